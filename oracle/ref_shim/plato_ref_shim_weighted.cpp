// plato_ref_shim_weighted.cpp — the reference's algo::weighted_pagerank
// (plato/algo/pagerank/weighted_pagerank.hpp:60-149) behind the oracle
// shim's C API (test infrastructure only; see plato_ref_shim.cpp).  It is
// built into a library of its own (oracle/_ref/libplato_ref_weighted.so):
// weighted_pagerank.hpp defines its own pagerank_opts_t, which pagerank.hpp
// also defines, and the reference's headers define non-inline functions, so
// each of its programs is a single translation unit.
#include <cstdint>
#include <memory>
#include <vector>

#include "plato/graph/graph.hpp"
#include "plato/algo/pagerank/weighted_pagerank.hpp"

#include "shim_common.hpp"

DEFINE_int32(threads, -1, "threads (the reference's --threads)");

namespace plato {
void install_oneshot_signal_handlers() {}
}  // namespace plato

namespace plato_ref_shim {
std::mutex g_log_mu;
std::vector<std::string> g_lines;
}  // namespace plato_ref_shim

using namespace plato_ref_shim;

namespace {

using wdcsc_spec_t = plato::dcsc_t<double, plato::sequence_balanced_by_source_t>;

// create_dcsc_seqs_from_path<double> (structure.hpp:471-555) from memory
struct ref_wgraph {
  plato::graph_info_t info;
  std::unique_ptr<wdcsc_spec_t> dcsc;
};

}  // namespace

extern "C" {

// Weighted graph: edges with a double weight each, as the weighted CLI loads them.
__attribute__((visibility("default"))) void* refp_wgraph_build(uint32_t vertices, uint64_t n, const uint32_t* src,
                                                               const uint32_t* dst, const double* w,
                                                               int is_directed) {
  init_once();
  auto* g = new ref_wgraph();
  g->info.is_directed_ = is_directed != 0;
  std::shared_ptr<plato::edge_block_cache_t<double, plato::vid_t>> cache(
      new plato::edge_block_cache_t<double, plato::vid_t>());
  plato::bitmap_t<> v_bitmap(vertices > 0 ? vertices : 1);
  std::vector<plato::edge_unit_t<double, plato::vid_t>> block;
  for (uint64_t i = 0; i < n; ++i) {
    plato::edge_unit_t<double, plato::vid_t> e;
    e.src_ = src[i];
    e.dst_ = dst[i];
    e.edata_ = w[i];
    block.push_back(e);
    v_bitmap.set_bit(src[i]);
    v_bitmap.set_bit(dst[i]);
    if (block.size() == 4096 || i + 1 == n) {
      cache->push_back(block.data(), block.size());
      block.clear();
    }
  }
  g->info.edges_ = n;
  g->info.vertices_ = static_cast<plato::vid_t>(v_bitmap.count());
  g->info.max_v_i_ = static_cast<plato::vid_t>(v_bitmap.msb());
  std::vector<plato::vid_t> degrees = plato::generate_dense_out_degrees<plato::vid_t>(g->info, *cache);
  plato::eid_t edges = g->info.edges_;
  if (!g->info.is_directed_) edges *= 2;
  std::shared_ptr<plato::sequence_balanced_by_source_t> part(
      new plato::sequence_balanced_by_source_t(degrees.data(), g->info.vertices_, edges, -1));
  part->check_consistency();
  g->dcsc.reset(new wdcsc_spec_t(part));
  if (g->dcsc->load_from_cache(g->info, *cache) != 0) {
    delete g;
    return nullptr;
  }
  return g;
}

__attribute__((visibility("default"))) void refp_wgraph_free(void* h) { delete static_cast<ref_wgraph*>(h); }

// algo::weighted_pagerank (weighted_pagerank.hpp:60-149), reference units.
__attribute__((visibility("default"))) int refp_weighted_pagerank(void* h, uint32_t iteration, double damping,
                                                                  double eps, double* out, uint32_t* epochs) {
  auto* g = static_cast<ref_wgraph*>(h);
  plato::algo::pagerank_opts_t opts;
  opts.iteration_ = iteration;
  opts.damping_ = damping;
  opts.eps_ = eps;
  start_capture();
  auto ranks = plato::algo::weighted_pagerank(*g->dcsc, g->info, opts);
  const auto lines = stop_capture();
  copy_out(ranks, g->info.max_v_i_ + 1, out);
  *epochs = epoch_deltas(lines, nullptr, 0);
  return 0;
}

}  // extern "C"
