// Breadth-first search with the dual-mode engine's push/pull switch.
//
// Mirrors algo::breadth_first_search (plato/algo/bfs/bfs.hpp:55-155) driven by
// dualmode_engine_t::foreach_edges (plato/engine/dualmode.hpp:245-297):
//   each epoch: active_edges = sum of out-degrees of the current frontier;
//   push iff active_edges / edges < push_threshold (edges doubled for
//   undirected graphs, dualmode.hpp:261-262), else pull.
//   push (bfs.hpp:97-118): each frontier vertex claims unvisited out-neighbours.
//   pull (bfs.hpp:119-136): each unvisited vertex takes the first in-neighbour
//   that is in the current frontier.
// A vertex first reached in epoch e has level e + 1 (root: 0).  Levels are
// unique; parents depend on claim order in push mode, as in the reference.
#include <new>

#include "graph.cuh"
#include "push.cuh"

namespace plato_b200 {

// Device-side level state.  mode: 1 = the next level runs push, 0 = pull.
struct bfs_control {
  int mode;
  int done;                  // the last level activated no vertex
  uint32_t level;            // levels run (epochs, bfs.hpp:92)
  uint32_t pushes;           // of which push
  unsigned long long visited;
  unsigned long long trace;  // bit i: level i ran push (first 64 levels)
};

struct bfs_workspace {
  push_frontier fr[2];
  dbuf<uint32_t> visited;
  dbuf<uint32_t> level, parent;
  dbuf<bfs_control> ctrl;
  bfs_control* h_ctrl = nullptr;  // pinned
  ~bfs_workspace() {
    if (h_ctrl) cudaFreeHost(h_ctrl);
  }
};

void destroy_bfs_workspace(bfs_workspace* ws) { delete ws; }

namespace {

// After a level: count it, fold the new frontier into the visited count and
// pick the next level's mode from its active-edge count (dualmode.hpp:264-279).
__global__ void k_bfs_control(frontier_view fn, bfs_control* c, double edges, double threshold) {
  if (threadIdx.x != 0 || c->done) return;
  const unsigned long long actives = fn.counters[0];
  if (c->mode == 1) c->pushes += 1;
  c->level += 1;
  c->visited += actives;
  if (actives == 0) {
    c->done = 1;
    return;
  }
  const int push = (static_cast<double>(fn.counters[2]) / edges) < threshold ? 1 : 0;
  c->mode = push;
  if (push && c->level < 64) c->trace |= 1ull << c->level;
}

__global__ void k_bfs_init(uint32_t V, uint32_t root, uint32_t invalid_parent, uint32_t* level,
                           uint32_t* parent, uint32_t* visited) {
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < V;
       v += (uint64_t)gridDim.x * blockDim.x) {
    level[v] = v == root ? 0u : PLATO_LEVEL_UNREACHED;
    parent[v] = v == root ? root : invalid_parent;
    if ((v & 31) == 0) {
      uint32_t w = 0;
      if ((root >> 5) == (v >> 5)) w = 1u << (root & 31);
      visited[v >> 5] = w;
    }
  }
}

// Push level: frontier chunks -> claim unvisited out-neighbours.
__global__ void __launch_bounds__(256) k_bfs_push(frontier_view cur, frontier_view next,
                                                  const uint64_t* __restrict__ out_off,
                                                  const uint32_t* __restrict__ out_adj,
                                                  const uint32_t* __restrict__ deg,
                                                  uint32_t* visited, uint32_t* level,
                                                  uint32_t* parent, uint32_t new_level,
                                                  const bfs_control* ctrl) {
  if (ctrl->done || ctrl->mode != 1) return;  // uniform: pull level or finished
  const unsigned long long nchunks = cur.counters[1];
  const unsigned lane = threadIdx.x & 31;
  const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t c = warp; c < nchunks; c += nwarps) {
    const uint2 ch = cur.chunks[c];
    const uint32_t u = ch.x;
    const uint64_t b = out_off[u] + static_cast<uint64_t>(ch.y) * kPushChunk;
    const uint64_t e_end = min(b + kPushChunk, out_off[u + 1]);
    for (uint64_t base = b; base < e_end; base += 32) {
      const uint64_t e = base + lane;
      uint32_t dst = 0;
      bool fresh = false;
      if (e < e_end) {
        dst = out_adj[e];
        const uint32_t bit = 1u << (dst & 31);
        if (!(visited[dst >> 5] & bit)) fresh = !(atomicOr(&visited[dst >> 5], bit) & bit);
        if (fresh) {
          level[dst] = new_level;
          parent[dst] = u;
          atomicOr(&next.bits[dst >> 5], bit);
        }
      }
      frontier_append_warp(next, fresh, dst, deg);
    }
  }
}

// Pull level: every unvisited vertex scans its in-edges for a frontier member.
__global__ void __launch_bounds__(256) k_bfs_pull(uint32_t V, frontier_view cur, frontier_view next,
                                                  const uint64_t* __restrict__ in_off,
                                                  const uint32_t* __restrict__ in_adj,
                                                  const uint32_t* __restrict__ deg,
                                                  uint32_t* visited, uint32_t* level,
                                                  uint32_t* parent, uint32_t new_level,
                                                  const bfs_control* ctrl) {
  if (ctrl->done || ctrl->mode != 0) return;  // uniform: push level or finished
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  const uint64_t nrounds = (V + stride - 1) / stride;
  for (uint64_t r = 0; r < nrounds; ++r) {  // warp-uniform trip count for the appends
    const uint64_t v = r * stride + blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    bool fresh = false;
    if (v < V && !test_bit(visited, static_cast<uint32_t>(v))) {
      const uint64_t b = in_off[v], e = in_off[v + 1];
      // four in-neighbours per step (ids, then bitmap tests, all in flight);
      // the first hit in CSC order is the parent, as in a one-by-one scan
      for (uint64_t i = b; i < e; i += 4) {
        const bool p1 = i + 1 < e, p2 = i + 2 < e, p3 = i + 3 < e;
        const uint32_t s0 = in_adj[i];
        const uint32_t s1 = p1 ? in_adj[i + 1] : 0u;
        const uint32_t s2 = p2 ? in_adj[i + 2] : 0u;
        const uint32_t s3 = p3 ? in_adj[i + 3] : 0u;
        const bool h0 = test_bit(cur.bits, s0);
        const bool h1 = p1 && test_bit(cur.bits, s1);
        const bool h2 = p2 && test_bit(cur.bits, s2);
        const bool h3 = p3 && test_bit(cur.bits, s3);
        if (h0 || h1 || h2 || h3) {
          const uint32_t s = h0 ? s0 : h1 ? s1 : h2 ? s2 : s3;
          fresh = true;
          level[v] = new_level;
          parent[v] = s;
          const uint32_t bit = 1u << (v & 31);
          atomicOr(&visited[v >> 5], bit);
          atomicOr(&next.bits[v >> 5], bit);
          break;
        }
      }
    }
    frontier_append_warp(next, fresh, static_cast<uint32_t>(v), deg);
  }
}

int ensure_bfs_ws(plato_graph* g) {
  if (!g->bfs_ws) {
    g->bfs_ws = new (std::nothrow) bfs_workspace();
    if (!g->bfs_ws) return set_error(PLATO_ENOMEM, "bfs workspace: host allocation failed");
  }
  bfs_workspace* ws = g->bfs_ws;
  const uint32_t V = g->info.vertices;
  PLATO_TRY(frontier_alloc(ws->fr[0], g));
  PLATO_TRY(frontier_alloc(ws->fr[1], g));
  PLATO_TRY(ws->visited.alloc((V + 31) / 32));
  PLATO_TRY(ws->level.alloc(V));
  PLATO_TRY(ws->parent.alloc(V));
  PLATO_TRY(ws->ctrl.alloc(1));
  if (!ws->h_ctrl)
    PLATO_CUDA_TRY(cudaMallocHost(reinterpret_cast<void**>(&ws->h_ctrl), sizeof(bfs_control)));
  return PLATO_OK;
}

// parent ids are internal; map to caller ids (the invalid marker stays).
__global__ void k_parents_to_external(const uint32_t* __restrict__ parent_int,
                                      const uint32_t* __restrict__ to_ext, uint32_t V,
                                      uint32_t invalid, uint32_t* parent_ext) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < V;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t p = parent_int[i];
    parent_ext[to_ext[i]] = (p == invalid) ? invalid : to_ext[p];
  }
}

int bfs_impl(plato_graph* g, const plato_bfs_opts* o, const plato_dualmode_opts* eo,
             cudaStream_t st, plato_run_stats* stats) {
  const uint32_t V = g->info.vertices;
  if (o->root >= V) return set_error(PLATO_EINVAL, "bfs: root out of range");
  const double threshold = eo ? eo->push_threshold : 0.05;
  PLATO_TRY(ensure_bfs_ws(g));
  bfs_workspace* ws = g->bfs_ws;
  uint32_t root = 0;
  PLATO_TRY(lookup_internal(g, o->root, &root, st));
  const uint32_t invalid_parent = g->info.max_v_i + 1;  // bfs.hpp:79
  k_bfs_init<<<grid_for(V, 256), 256, 0, st>>>(V, root, invalid_parent, ws->level.p, ws->parent.p,
                                                ws->visited.p);
  PLATO_LAUNCHED("k_bfs_init");
  PLATO_TRY(frontier_reset(ws->fr[0], V, st));
  PLATO_TRY(frontier_seed(ws->fr[0], g, root, st));
  PLATO_TRY(frontier_read(ws->fr[0], st));

  // Level loop with the engine switch on the device: after each level
  // k_bfs_control reads the new frontier's counters, decides push or pull for
  // the next level (dualmode.hpp:264-279) and flags the end (bfs.hpp:92, no
  // vertex activated).  The host enqueues levels in batches and polls between
  // batches; levels enqueued after the end return at once.
  const double edges = static_cast<double>(g->stored_edges);
  const bool first_push = (static_cast<double>(ws->fr[0].h_counters[2]) / edges) < threshold;
  const bfs_control init{first_push ? 1 : 0, 0, 0, 0, 1ull, first_push ? 1ull : 0ull};
  PLATO_CUDA_TRY(cudaMemcpyAsync(ws->ctrl.p, &init, sizeof(init), cudaMemcpyHostToDevice, st));
  const unsigned push_blocks = 148 * 16;
  const unsigned pull_blocks = grid_for(V, 256, 148 * 8);
  constexpr uint32_t kBatch = 4;
  uint32_t launched = 0;
  for (;;) {
    for (uint32_t k = 0; k < kBatch; ++k, ++launched) {
      const int cur = static_cast<int>(launched & 1u);
      push_frontier& fc = ws->fr[cur];
      push_frontier& fn = ws->fr[cur ^ 1];
      PLATO_TRY(frontier_reset(fn, V, st));
      k_bfs_push<<<push_blocks, 256, 0, st>>>(fc.view(), fn.view(), g->out_off.p, g->out_adj.p,
                                              g->out_deg.p, ws->visited.p, ws->level.p,
                                              ws->parent.p, launched + 1, ws->ctrl.p);
      PLATO_LAUNCHED("k_bfs_push");
      k_bfs_pull<<<pull_blocks, 256, 0, st>>>(V, fc.view(), fn.view(), g->in_off.p, g->in_adj.p,
                                              g->out_deg.p, ws->visited.p, ws->level.p,
                                              ws->parent.p, launched + 1, ws->ctrl.p);
      PLATO_LAUNCHED("k_bfs_pull");
      k_bfs_control<<<1, 32, 0, st>>>(fn.view(), ws->ctrl.p, edges, threshold);
      PLATO_LAUNCHED("k_bfs_control");
    }
    PLATO_CUDA_TRY(cudaMemcpyAsync(ws->h_ctrl, ws->ctrl.p, sizeof(bfs_control), cudaMemcpyDeviceToHost, st));
    PLATO_CUDA_TRY(cudaStreamSynchronize(st));
    if (ws->h_ctrl->done) break;
  }
  const bfs_control& c = *ws->h_ctrl;
  if (stats) {
    *stats = plato_run_stats{};
    stats->iterations = c.level;
    const uint32_t traced = std::min<uint32_t>(c.level, 64);
    const uint64_t mask = traced >= 64 ? ~0ull : ((1ull << traced) - 1);
    stats->push_iterations = c.pushes;
    stats->pull_iterations = c.level - c.pushes;
    stats->visited = c.visited;
    stats->mode_trace = c.trace & mask;
  }
  return PLATO_OK;
}

}  // namespace
}  // namespace plato_b200

using namespace plato_b200;

extern "C" int plato_bfs(plato_graph* g, const plato_bfs_opts* opts,
                         const plato_dualmode_opts* engine_opts, uint32_t* levels,
                         plato_vid_t* parents, plato_run_stats* stats) {
  if (!g || !opts) return set_error(PLATO_EINVAL, "plato_bfs: null argument");
  std::lock_guard<std::mutex> lock(g->mu);
  PLATO_CUDA_TRY(cudaSetDevice(g->device));
  cudaStream_t st = g->stream;
  PLATO_TRY(bfs_impl(g, opts, engine_opts, st, stats));
  const uint32_t V = g->info.vertices;
  bfs_workspace* ws = g->bfs_ws;
  if (levels || parents) {
    dbuf<uint32_t> ext;
    PLATO_TRY(ext.alloc(V));
    if (levels) {
      PLATO_TRY(scatter_to_external_u32(g, ws->level.p, ext.p, st));
      PLATO_CUDA_TRY(cudaMemcpyAsync(levels, ext.p, V * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
      PLATO_CUDA_TRY(cudaStreamSynchronize(st));
    }
    if (parents) {
      if (g->relabeled) {
        k_parents_to_external<<<grid_for(V, 256), 256, 0, st>>>(
            ws->parent.p, g->to_ext.p, V, g->info.max_v_i + 1, ext.p);
        PLATO_LAUNCHED("k_parents_to_external");
      } else {
        PLATO_CUDA_TRY(cudaMemcpyAsync(ext.p, ws->parent.p, V * sizeof(uint32_t),
                                       cudaMemcpyDeviceToDevice, st));
      }
      PLATO_CUDA_TRY(cudaMemcpyAsync(parents, ext.p, V * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
      PLATO_CUDA_TRY(cudaStreamSynchronize(st));
    }
  }
  return PLATO_OK;
}
