// Connected components by label propagation on the dual-mode engine.
//
// Mirrors plato::algo::connected_component_t (plato/algo/cgm/connected_component.hpp):
//   compute (:173-245)  labels start as the vertex ids and every vertex is
//       active; each epoch runs foreach_edges with
//         push  signal sends (v, label[v]); the slot lowers label[dst] of every
//               out-neighbour with write_min and activates it
//         pull  signal takes the smallest label of v's in-neighbours (starting
//               from v's own id) and sends it when below v's id; the slot
//               lowers label[v] with write_min and activates v
//       and the engine's active-edge switch picks push or pull; the loop ends
//       after an epoch that lowered nothing.  The pull runs on the engine's
//       combined path: a vertex's 4-edge pieces in one warp fold to their
//       smallest label before one slot call (the reference's slot sees one
//       message per partition piece instead; write_min gives the same labels).
//   summary (:247-340)  component count (distinct labels), the largest
//       component ("major label"; ties here go to the smallest label, the
//       reference takes whichever its hash map visits first) with its vertex
//       count and its edges: in-edges whose source carries the label, halved
//       for undirected graphs.
// The functors are written for include/plato_b200/dualmode.cuh, the same
// header a user client of the engine includes.  Labels are caller ids:
// internal vertex v starts with its caller id, so the fixed point is the
// smallest caller id that reaches v (the component's smallest id when the
// graph is undirected) whatever the engine's internal numbering.
#include <exception>
#include <mutex>

#include "graph.cuh"
#include "plato_b200/dualmode.cuh"

namespace plato_b200 {
namespace {

struct cc_msg {  // connected_comp_msg_type_t (connected_component.hpp:40-45)
  vid_t src_;
  vid_t label_;
};

__global__ void k_cc_init(vid_t* labels, const vid_t* __restrict__ to_ext, uint32_t V) {
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < V;
       v += (uint64_t)gridDim.x * blockDim.x)
    labels[v] = to_ext ? to_ext[v] : static_cast<vid_t>(v);
}

// cnt[label] = vertices carrying it; roots (label == own caller id) count
// the components; best = max over labels of (count << 32 | ~label).  Lanes
// of a warp holding the same label add once for all of them (a large
// component's label would otherwise take one atomic per vertex on a single
// counter).
__global__ void k_cc_count(const vid_t* __restrict__ labels, const vid_t* __restrict__ to_ext,
                           uint32_t V, uint32_t* cnt, unsigned long long* roots) {
  const unsigned lane = threadIdx.x & 31;
  unsigned long long r = 0;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;  // a multiple of 32
  // the warp stays together: the trip count follows its first lane
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v - lane < V; v += stride) {
    const bool valid = v < V;
    const vid_t l = valid ? labels[v] : 0xFFFFFFFFu;
    const unsigned same = __match_any_sync(0xFFFFFFFFu, l);
    if (valid && lane == static_cast<unsigned>(__ffs(same) - 1))
      atomicAdd(&cnt[l], static_cast<uint32_t>(__popc(same)));
    r += (valid && l == (to_ext ? to_ext[v] : static_cast<vid_t>(v))) ? 1ull : 0ull;
  }
  r = warp_sum(r);
  if (lane == 0 && r) atomicAdd(roots, r);
}

__global__ void k_cc_major(const uint32_t* __restrict__ cnt, uint32_t V, unsigned long long* best) {
  unsigned long long b = 0;
  for (uint64_t l = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; l < V;
       l += (uint64_t)gridDim.x * blockDim.x)
    if (cnt[l]) b = max(b, (static_cast<unsigned long long>(cnt[l]) << 32) | (0xFFFFFFFFu - static_cast<uint32_t>(l)));
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) b = max(b, __shfl_xor_sync(0xffffffffu, b, o));
  if ((threadIdx.x & 31) == 0 && b) atomicMax(best, b);
}

// In-edges whose source carries `label` (connected_component.hpp:310-323).
__global__ void k_cc_edges(const uint32_t* __restrict__ in_adj, uint64_t E,
                           const vid_t* __restrict__ labels, vid_t label, unsigned long long* out) {
  unsigned long long c = 0;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < E;
       i += (uint64_t)gridDim.x * blockDim.x)
    c += (labels[in_adj[i]] == label);
  c = warp_sum(c);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(out, c);
}

int cc_impl(plato_graph* g, const plato_dualmode_opts* eo, plato_vid_t* labels_out,
            plato_cc_summary* summary, plato_run_stats* stats) {
  dualmode_engine_opts_t opts;
  if (eo) opts.push_threshold_ = eo->push_threshold;
  dualmode_engine_t engine(g, opts);
  const uint32_t V = engine.vertices();
  const vid_t* to_ext = g->relabeled ? g->to_ext.p : nullptr;
  auto labels = engine.alloc_v_state<vid_t>();
  k_cc_init<<<grid_for(V, 256), 256>>>(labels.data(), to_ext, V);
  check_cuda(cudaGetLastError(), "k_cc_init");
  count_launch();
  vid_t* L = labels.data();
  const out_edges_view oe = engine.out_edges();
  auto active_current = engine.alloc_v_subset();
  auto active_next = engine.alloc_v_subset();
  {
    std::vector<uint32_t> all((V + 31) / 32, 0xFFFFFFFFu);  // active_current.fill()
    if (V % 32) all.back() = (1u << (V % 32)) - 1u;
    check_cuda(cudaMemcpy(active_current.data(), all.data(), all.size() * 4, cudaMemcpyHostToDevice),
               "cc actives");
  }
  uint32_t epochs = 0, pushes = 0;
  uint64_t trace = 0;
  for (vid_t actives = V; actives != 0; ++epochs) {
    active_next.clear();
    const bitmap_t::view next = active_next.dev();
    actives = engine.foreach_edges<cc_msg, vid_t>(
        [L] __device__(const auto& context, vid_t v_i) { context.send(cc_msg{v_i, L[v_i]}); },
        [L, oe, next] __device__(int, cc_msg& msg) -> vid_t {
          vid_t activated = 0;
          const adj_unit_list_t nbrs = oe.neighbours(msg.src_);
          for (auto it = nbrs.begin_; nbrs.end_ != it; ++it) {
            const vid_t dst = it->neighbour_;
            if (msg.label_ < L[dst]) {
              atomicMin(L + dst, msg.label_);  // write_min (atomic.hpp:78-88)
              next.set_bit(dst);
              ++activated;
            }
          }
          return activated;
        },
        [L, to_ext] __device__(const auto& context, vid_t v_i, const adj_unit_list_t& adjs) {
          const vid_t self = to_ext ? to_ext[v_i] : v_i;  // the vertex's own id
          vid_t cur_label = self;
          for (auto it = adjs.begin_; adjs.end_ != it; ++it) {
            const vid_t l = L[it->neighbour_];
            if (l < cur_label) cur_label = l;
          }
          if (cur_label < self) context.send(mepa_ag_message_t<cc_msg>{v_i, cc_msg{v_i, cur_label}});
        },
        [L, next] __device__(int, mepa_ag_message_t<cc_msg>& msg) -> vid_t {
          if (msg.message_.label_ < L[msg.v_i_]) {
            atomicMin(L + msg.v_i_, msg.message_.label_);
            next.set_bit(msg.v_i_);
            return 1;
          }
          return 0;
        },
        active_current,
        // a vertex's pull messages fold to the smallest label before its slot
        make_combiner([] __device__(cc_msg& into, const cc_msg& from) {
          if (from.label_ < into.label_) into = from;
        }));
    count_launch(2);
    if (engine.last_was_push()) {
      ++pushes;
      if (epochs < 64) trace |= 1ull << epochs;
    }
    std::swap(active_current, active_next);
  }
  if (stats) {
    *stats = plato_run_stats{};
    stats->iterations = epochs;
    stats->push_iterations = pushes;
    stats->pull_iterations = epochs - pushes;
    stats->mode_trace = trace;
  }
  if (summary) {
    uint32_t* cnt = nullptr;
    unsigned long long* acc = nullptr;  // [0] roots, [1] best, [2] major edges
    dev_alloc(&cnt, 4ull * (V ? V : 1), "cc counts");
    dev_alloc(&acc, 3 * sizeof(unsigned long long), "cc summary");
    int rc = PLATO_OK;
    try {
      check_cuda(cudaMemset(cnt, 0, 4ull * V), "cc counts");
      check_cuda(cudaMemset(acc, 0, 3 * sizeof(unsigned long long)), "cc summary");
      k_cc_count<<<grid_for(V, 256), 256>>>(L, to_ext, V, cnt, acc);
      k_cc_major<<<grid_for(V, 256), 256>>>(cnt, V, acc + 1);
      check_cuda(cudaGetLastError(), "cc summary kernels");
      count_launch(2);
      unsigned long long h[3] = {0, 0, 0};
      check_cuda(cudaMemcpy(h, acc, 2 * sizeof(unsigned long long), cudaMemcpyDeviceToHost), "cc summary");
      const vid_t major = 0xFFFFFFFFu - static_cast<uint32_t>(h[1] & 0xFFFFFFFFull);
      const uint64_t E = g->stored_edges;
      if (V) {
        k_cc_edges<<<grid_for(E, 256), 256>>>(g->in_adj.p, E, L, major, acc + 2);
        check_cuda(cudaGetLastError(), "k_cc_edges");
        count_launch();
        check_cuda(cudaMemcpy(h + 2, acc + 2, sizeof(unsigned long long), cudaMemcpyDeviceToHost), "cc edges");
      }
      summary->components = h[0];
      summary->major_label = V ? major : 0;
      summary->major_vertices = h[1] >> 32;
      summary->major_edges = g->info.is_directed ? h[2] : h[2] / 2;
    } catch (const std::exception& e) {
      rc = set_error(PLATO_ECUDA, e.what());
    }
    dev_free(cnt);
    dev_free(acc);
    if (rc != PLATO_OK) return rc;
  }
  if (labels_out) {
    const std::vector<vid_t> h = engine.to_host(labels);
    std::copy(h.begin(), h.end(), labels_out);
  }
  return PLATO_OK;
}

}  // namespace
}  // namespace plato_b200

using namespace plato_b200;

extern "C" int plato_connected_components(plato_graph* g, const plato_dualmode_opts* engine_opts,
                                          plato_vid_t* labels, plato_cc_summary* summary,
                                          plato_run_stats* stats) {
  if (!g) return set_error(PLATO_EINVAL, "plato_connected_components: null graph");
  std::lock_guard<std::mutex> lock(g->mu);
  PLATO_CUDA_TRY(cudaSetDevice(g->device));
  PLATO_CUDA_TRY(cudaStreamSynchronize(g->stream));  // the engine runs on the default stream
  try {
    return cc_impl(g, engine_opts, labels, summary, stats);
  } catch (const std::exception& e) {
    return set_error(PLATO_ECUDA, std::string("plato_connected_components: ") + e.what());
  }
}
