// plato_ref_shim.cpp — the reference's own engine path, compiled from its
// headers where they lie in the reference tree, behind a small C API.
//
// TEST INFRASTRUCTURE ONLY: the oracle's build compiles this file into
// oracle/_ref/libplato_ref.so when the reference tree is present; the CPU
// tests and the fixture script call it to pin the oracle's restatement
// (oracle/ref_cpu.c) to what the reference itself computes.  Nothing in the
// product links or calls it.
//
// The reference needs MPI, glog, gflags, libnuma, libhdfs, boost and yas,
// none of which this image has.  oracle/ref_shim/include holds stand-ins:
// a one-rank in-process MPI (every message the engine sends goes to the
// process itself, as under `mpirun -np 1`), glog macros whose lines this file
// captures, and declarations for the file-system and serialisation names that
// the engine path mentions but never calls on in-memory graphs.  The engine,
// the graph structures, the message passing and the algorithms are the
// reference's code, unmodified, compiled with __DUALMODE_DEBUG__ so that the
// engine logs its push/pull choice per call (plato/engine/dualmode.hpp:281-293).
//
// Graph construction follows create_dualmode_seq_from_path
// (plato/graph/structure.hpp:983-1086) step for step, with the edge cache
// filled from memory instead of read_from_files (load_edges_cache,
// structure.hpp:190-237, sets the same graph_info fields from the same
// bitmap): out-degrees from the cache, sequence_balanced_by_destination_t
// partition, bcsr_t::load_from_cache, then dcsc_t::load_from_graph with the
// RANDOM traversal.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "plato/graph/graph.hpp"
#include "plato/algo/pagerank/pagerank.hpp"
#include "plato/algo/ppr/personalized_pagerank.hpp"
#include "plato/algo/bfs/bfs.hpp"
#include "plato/algo/trustrank/trustrank.hpp"
#include "plato/algo/cgm/connected_component.hpp"
#include "plato/algo/hyperanf/hyperanf.hpp"

#include "shim_common.hpp"

DEFINE_int32(threads, -1, "threads (the reference's --threads)");

namespace plato {
void install_oneshot_signal_handlers() {}
}  // namespace plato

namespace plato_ref_shim {
std::mutex g_log_mu;
std::vector<std::string> g_lines;
}  // namespace plato_ref_shim

namespace {

using bcsr_spec_t = plato::bcsr_t<plato::empty_t, plato::sequence_balanced_by_destination_t>;
using dcsc_spec_t = plato::dcsc_t<plato::empty_t, plato::sequence_balanced_by_source_t>;

struct ref_graph {
  plato::graph_info_t info;
  std::unique_ptr<bcsr_spec_t> bcsr;
  std::unique_ptr<dcsc_spec_t> dcsc;
};

// mode trace from the engine's debug lines: bit i set = call i ran push-mode
uint64_t mode_trace(const std::vector<std::string>& lines) {
  uint64_t trace = 0;
  uint32_t n = 0;
  for (const auto& l : lines) {
    if (l.find("active_edges: ") != 0) continue;
    if (l.find("push-mode") != std::string::npos && n < 64) trace |= 1ull << n;
    ++n;
  }
  return trace;
}

}  // namespace

using namespace plato_ref_shim;

extern "C" {

// Edge list (caller ids, compact) -> the reference's BCSR + DCSC.
__attribute__((visibility("default"))) void* refp_graph_build(uint32_t vertices, uint64_t n,
                                                              const uint32_t* src, const uint32_t* dst,
                                                              int is_directed) {
  init_once();
  auto* g = new ref_graph();
  g->info.is_directed_ = is_directed != 0;
  std::shared_ptr<plato::edge_block_cache_t<plato::empty_t, plato::vid_t>> cache(
      new plato::edge_block_cache_t<plato::empty_t, plato::vid_t>());
  plato::bitmap_t<> v_bitmap(vertices > 0 ? vertices : 1);
  {
    constexpr uint64_t kBlock = 4096;
    std::vector<plato::edge_unit_t<plato::empty_t, plato::vid_t>> block;
    block.reserve(kBlock);
    for (uint64_t i = 0; i < n; ++i) {
      plato::edge_unit_t<plato::empty_t, plato::vid_t> e;
      e.src_ = src[i];
      e.dst_ = dst[i];
      block.push_back(e);
      v_bitmap.set_bit(src[i]);
      v_bitmap.set_bit(dst[i]);
      if (block.size() == kBlock || i + 1 == n) {
        cache->push_back(block.data(), block.size());
        block.clear();
      }
    }
  }
  g->info.edges_ = n;
  g->info.vertices_ = static_cast<plato::vid_t>(v_bitmap.count());
  g->info.max_v_i_ = static_cast<plato::vid_t>(v_bitmap.msb());
  (void)vertices;

  std::shared_ptr<plato::sequence_balanced_by_destination_t> part_bcsr;
  {
    std::vector<plato::vid_t> degrees = plato::generate_dense_out_degrees<plato::vid_t>(g->info, *cache);
    plato::eid_t edges = g->info.edges_;
    if (!g->info.is_directed_) edges *= 2;
    part_bcsr.reset(new plato::sequence_balanced_by_destination_t(degrees.data(), g->info.vertices_, edges, -1));
    part_bcsr->check_consistency();
  }
  g->bcsr.reset(new bcsr_spec_t(part_bcsr));
  if (g->bcsr->load_from_cache(g->info, *cache) != 0) {
    delete g;
    return nullptr;
  }
  cache = nullptr;
  std::shared_ptr<plato::sequence_balanced_by_source_t> part_dcsc(
      new plato::sequence_balanced_by_source_t(part_bcsr->offset_));
  g->dcsc.reset(new dcsc_spec_t(part_dcsc));
  plato::traverse_opts_t opts;
  opts.mode_ = plato::traverse_mode_t::RANDOM;
  if (g->dcsc->load_from_graph(g->info, *g->bcsr, true, opts) != 0) {
    delete g;
    return nullptr;
  }
  return g;
}

__attribute__((visibility("default"))) void refp_graph_free(void* h) { delete static_cast<ref_graph*>(h); }

// Threads the reference runs its OpenMP loops on (cluster_info_t::threads_,
// from --threads, OMP_NUM_THREADS or every configured CPU, base.hpp:194-202).
__attribute__((visibility("default"))) int refp_threads(void) {
  init_once();
  return plato::cluster_info_t::get_instance().threads_;
}

// graph_info_t of the built graph: {vertices, max_v_i, edges}
__attribute__((visibility("default"))) void refp_graph_info(void* h, uint32_t* vertices, uint32_t* max_v_i,
                                                            uint64_t* edges) {
  auto* g = static_cast<ref_graph*>(h);
  *vertices = g->info.vertices_;
  *max_v_i = g->info.max_v_i_;
  *edges = g->info.edges_;
}

// algo::pagerank (pagerank.hpp:60-149): ranks [max_v_i + 1] in the reference's
// units; *epochs = epochs logged, deltas [cap] = each epoch's logged delta.
__attribute__((visibility("default"))) int refp_pagerank(void* h, uint32_t iteration, double damping, double eps,
                                                         double* out, uint32_t* epochs, double* deltas,
                                                         uint32_t cap) {
  auto* g = static_cast<ref_graph*>(h);
  plato::algo::pagerank_opts_t opts;
  opts.iteration_ = iteration;
  opts.damping_ = damping;
  opts.eps_ = eps;
  start_capture();
  auto ranks = plato::algo::pagerank(*g->dcsc, g->info, opts);
  const auto lines = stop_capture();
  copy_out(ranks, g->info.max_v_i_ + 1, out);
  *epochs = epoch_deltas(lines, deltas, cap);
  return 0;
}

// algo::personalized_pagerank: pull-only (personalized_pagerank.hpp:40-134)
// or dual-mode (:137-275) when pushpull != 0.  Ranks [max_v_i + 1];
// *epochs = epochs logged.
__attribute__((visibility("default"))) int refp_ppr(void* h, uint32_t src, uint32_t iteration, double damping,
                                                    double eps, int pushpull, double* out, uint32_t* epochs) {
  auto* g = static_cast<ref_graph*>(h);
  plato::algo::personalized_pagerank_opts_t opts;
  opts.iteration_ = iteration;
  opts.damping_ = damping;
  opts.src_ = src;
  opts.eps_ = eps;
  start_capture();
  if (pushpull) {
    auto ranks = plato::algo::personalized_pagerank(*g->dcsc, *g->bcsr, g->info, opts);
    copy_out(ranks, g->info.max_v_i_ + 1, out);
  } else {
    auto ranks = plato::algo::personalized_pagerank(*g->dcsc, g->info, opts);
    copy_out(ranks, g->info.max_v_i_ + 1, out);
  }
  const auto lines = stop_capture();
  *epochs = epoch_deltas(lines, nullptr, 0);
  return 0;
}

// algo::trustrank with select_good_seeds (trustrank.hpp:88-259): good [V]
// 0/1 bytes; ranks [max_v_i + 1]; *epochs = the trust epochs (the last
// "[epoch-i]" lines after the selection PageRank's).  select_method 2 draws
// from std::random_device in the reference and is not offered here.
__attribute__((visibility("default"))) int refp_trustrank(void* h, const uint8_t* good, uint32_t seed_num,
                                                          uint32_t select_method, uint32_t iteration,
                                                          double damping, double eps, double* out,
                                                          uint32_t* epochs) {
  auto* g = static_cast<ref_graph*>(h);
  if (select_method > 1) return 1;
  plato::bitmap_t<> good_vertices(g->info.max_v_i_ + 1);
  for (uint32_t v = 0; v <= g->info.max_v_i_; ++v)
    if (good[v]) good_vertices.set_bit(v);
  plato::algo::trustrank_opts_t opts;
  opts.iteration_ = iteration;
  opts.damping_ = damping;
  opts.seed_num_ = seed_num;
  opts.select_method_ = select_method;
  opts.eps_ = eps;
  start_capture();
  auto ranks = plato::algo::trustrank(*g->dcsc, *g->bcsr, g->info, good_vertices, opts);
  const auto lines = stop_capture();
  copy_out(ranks, g->info.max_v_i_ + 1, out);
  // the trust loop's epochs follow the selection PageRank's (if any): count
  // the "[epoch-" lines after the last epoch-0 line
  uint32_t n = 0;
  for (const auto& l : lines) {
    if (l.rfind("[epoch-0]", 0) == 0) n = 0;
    if (l.rfind("[epoch-", 0) == 0) ++n;
  }
  *epochs = n;
  return 0;
}

// algo::breadth_first_search (bfs.hpp:55-155): returns the visited count;
// actives [cap] = the vertices activated per epoch (its "active_v[i] = n"
// lines), *epochs = epochs run, *trace = the engine's push/pull choice per
// epoch (bit i set = push).
__attribute__((visibility("default"))) uint64_t refp_bfs(void* h, uint32_t root, uint64_t* actives, uint32_t cap,
                                                         uint32_t* epochs, uint64_t* trace) {
  auto* g = static_cast<ref_graph*>(h);
  plato::algo::bfs_opts_t opts;
  opts.root_ = root;
  start_capture();
  const plato::vid_t visited = plato::algo::breadth_first_search(*g->dcsc, *g->bcsr, g->info, opts);
  const auto lines = stop_capture();
  uint32_t n = 0;
  for (const auto& l : lines) {
    int e = 0;
    unsigned long long a = 0;
    if (std::sscanf(l.c_str(), "active_v[%d] = %llu", &e, &a) == 2) {
      if (n < cap) actives[n] = a;
      ++n;
    }
  }
  *epochs = n;
  *trace = mode_trace(lines);
  return visited;
}

// connected_component_t::compute + summary (connected_component.hpp:173-340):
// labels [max_v_i + 1], component count, major label with its vertex and
// edge counts.
__attribute__((visibility("default"))) int refp_cc(void* h, uint32_t* labels, uint64_t* components,
                                                   uint32_t* major_label, uint64_t* major_vertices,
                                                   uint64_t* major_edges) {
  auto* g = static_cast<ref_graph*>(h);
  using engine_t = plato::dualmode_engine_t<dcsc_spec_t, bcsr_spec_t>;
  engine_t engine(std::shared_ptr<dcsc_spec_t>(g->dcsc.get(), [](dcsc_spec_t*) {}),
                  std::shared_ptr<bcsr_spec_t>(g->bcsr.get(), [](bcsr_spec_t*) {}), g->info);
  plato::algo::connected_component_t<dcsc_spec_t, bcsr_spec_t> cc(&engine, g->info);
  start_capture();
  cc.compute();
  stop_capture();
  copy_out_u32(*cc.get_labels(), g->info.max_v_i_ + 1, labels);
  *components = static_cast<uint64_t>(cc.get_num_components());
  *major_label = cc.get_major_label();
  *major_vertices = cc.get_major_vertices();
  const auto* info = cc.get_components_info();
  const auto it = info->find(cc.get_major_label());
  *major_edges = it == info->end() ? 0 : it->second.edges_;
  return 0;
}

// algo::hyperanf (hyperanf.hpp:83-195): the average distance, for register
// widths 6 and 8 (the template argument).
__attribute__((visibility("default"))) int refp_hyperanf(void* h, uint32_t bits, uint32_t iteration,
                                                         double* avg_distance) {
  auto* g = static_cast<ref_graph*>(h);
  plato::algo::hyperanf_opts_t opts;
  opts.iteration_ = iteration;
  opts.bits = bits;
  start_capture();
  if (bits == 6)
    *avg_distance = plato::algo::hyperanf<dcsc_spec_t, bcsr_spec_t, 6>(*g->dcsc, *g->bcsr, g->info, opts);
  else if (bits == 8)
    *avg_distance = plato::algo::hyperanf<dcsc_spec_t, bcsr_spec_t, 8>(*g->dcsc, *g->bcsr, g->info, opts);
  else {
    stop_capture();
    return 1;
  }
  stop_capture();
  return 0;
}

}  // extern "C"
