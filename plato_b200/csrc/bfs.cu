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
//
// One kernel launch per level (k_bfs_level): it runs the push or the pull
// step that the previous level chose, clears the frontier buffer that the
// level after next fills, and its last CTA to finish counts the new frontier
// and chooses the next level's mode (no CTA waits for another).  A search's
// start (root in, state cleared, root seeded, first mode chosen), its first
// 8 levels and the read of the control word are one CUDA graph per graph and
// threshold, so the host issues one launch where it issued 16 calls.
#include <algorithm>
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
  unsigned int arrived;      // CTAs of the running level that finished
};

struct bfs_workspace {
  push_frontier fr[3];  // current, next, and the one cleared for the level after
  dbuf<uint32_t> visited;
  dbuf<uint32_t> level, parent;
  dbuf<bfs_control> ctrl;
  bfs_control* h_ctrl = nullptr;  // pinned
  unsigned level_blocks = 0;      // one full wave of resident k_bfs_level CTAs
  dbuf<uint32_t> root;            // the search's root (internal id) on the device
  uint32_t* h_root = nullptr;     // pinned; copied to `root` by the start graph
  // start graph (see bfs_impl) and what it was captured with
  cudaGraphExec_t start = nullptr;
  double start_threshold = -1.0;
  const void* start_key = nullptr;
  ~bfs_workspace() {
    if (start) cudaGraphExecDestroy(start);
    if (h_ctrl) cudaFreeHost(h_ctrl);
    if (h_root) cudaFreeHost(h_root);
  }
};

void destroy_bfs_workspace(bfs_workspace* ws) { delete ws; }

namespace {

__global__ void k_bfs_init(uint32_t V, const uint32_t* __restrict__ root_p, uint32_t invalid_parent,
                           uint32_t* level, uint32_t* parent, uint32_t* visited) {
  const uint32_t root = *root_p;
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

struct bfs_level_args {
  frontier_view cur, next, spare;
  uint32_t V;
  const uint64_t* __restrict__ out_off;
  const uint32_t* __restrict__ out_adj;
  const uint32_t* __restrict__ out_deg;
  const uint64_t* __restrict__ in_off;
  const uint32_t* __restrict__ in_adj;
  uint32_t* visited;
  uint32_t* level;
  uint32_t* parent;
  uint32_t new_level;
  bfs_control* ctrl;
  double edges, threshold;
};

// Claims dst for parent u if nobody has (bfs.hpp:97-118: CAS on the parent);
// `word` is a recent read of dst's visited word (bits are only ever set, and
// the atomic decides).
__device__ __forceinline__ bool bfs_claim(const bfs_level_args& a, uint32_t u, uint32_t dst,
                                          uint32_t word) {
  const uint32_t bit = 1u << (dst & 31);
  if (word & bit) return false;
  if (atomicOr(&a.visited[dst >> 5], bit) & bit) return false;
  a.level[dst] = a.new_level;
  a.parent[dst] = u;
  atomicOr(&a.next.bits[dst >> 5], bit);
  return true;
}

constexpr uint32_t kPushLaneEdges = 8;  // chunks this short are walked by one lane

// Push step: frontier chunks -> claim unvisited out-neighbours.  With few
// chunks (at most four per warp) each warp walks one chunk, 32 edges a round.
// With many, a warp takes 32 chunks at a time, one per lane, interleaved over
// the chunk list (lane l of task t takes chunk l * tasks + t, so the chunks of
// one hub land on different warps); a lane walks a chunk of at most
// kPushLaneEdges edges itself (ids, then visited words, four at a time in
// flight), and the warp walks the longer chunks together.  Large push
// frontiers are mostly low-degree vertices with one short chunk each.
__device__ __forceinline__ void bfs_push_step(const bfs_level_args& a) {
  const unsigned long long nchunks = a.cur.counters[1];
  const unsigned lane = threadIdx.x & 31;
  const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  if (nchunks <= 4 * nwarps) {
    // few chunks (the first levels: hubs' long chunks): one chunk per warp,
    // so every chunk gets its own warp
    for (uint64_t c = warp; c < nchunks; c += nwarps) {
      const uint2 ch = a.cur.chunks[c];
      const uint64_t b = a.out_off[ch.x] + static_cast<uint64_t>(ch.y) * kPushChunk;
      const uint64_t e_end = min(b + kPushChunk, a.out_off[ch.x + 1]);
      for (uint64_t base = b; base < e_end; base += 32) {
        const uint64_t e = base + lane;
        uint32_t dst = 0;
        bool fresh = false;
        if (e < e_end) {
          dst = a.out_adj[e];
          fresh = bfs_claim(a, ch.x, dst, a.visited[dst >> 5]);
        }
        frontier_append_warp(a.next, fresh, dst, a.out_deg);
      }
    }
    return;
  }
  const uint64_t ntasks = (nchunks + 31) / 32;
  for (uint64_t t = warp; t < ntasks; t += nwarps) {  // warp-uniform
    const uint64_t c = static_cast<uint64_t>(lane) * ntasks + t;
    uint32_t u = 0;
    uint64_t b = 0, e_end = 0;
    if (c < nchunks) {
      const uint2 ch = a.cur.chunks[c];
      u = ch.x;
      b = a.out_off[u] + static_cast<uint64_t>(ch.y) * kPushChunk;
      e_end = min(b + kPushChunk, a.out_off[u + 1]);
    }
    const bool own = e_end - b <= kPushLaneEdges;  // lanes without a chunk too
    for (uint32_t s = 0; s < kPushLaneEdges; s += 4) {
      uint32_t d0 = 0, d1 = 0, d2 = 0, d3 = 0;
      bool f0 = false, f1 = false, f2 = false, f3 = false;
      if (own) {
        const uint64_t e = b + s;
        d0 = e < e_end ? a.out_adj[e] : 0u;
        d1 = e + 1 < e_end ? a.out_adj[e + 1] : 0u;
        d2 = e + 2 < e_end ? a.out_adj[e + 2] : 0u;
        d3 = e + 3 < e_end ? a.out_adj[e + 3] : 0u;
        // the four visited words in flight before the (rare) claims
        const uint32_t w0 = e < e_end ? a.visited[d0 >> 5] : ~0u;
        const uint32_t w1 = e + 1 < e_end ? a.visited[d1 >> 5] : ~0u;
        const uint32_t w2 = e + 2 < e_end ? a.visited[d2 >> 5] : ~0u;
        const uint32_t w3 = e + 3 < e_end ? a.visited[d3 >> 5] : ~0u;
        f0 = e < e_end && bfs_claim(a, u, d0, w0);
        f1 = e + 1 < e_end && bfs_claim(a, u, d1, w1);
        f2 = e + 2 < e_end && bfs_claim(a, u, d2, w2);
        f3 = e + 3 < e_end && bfs_claim(a, u, d3, w3);
      }
      frontier_append_warp(a.next, f0, d0, a.out_deg);
      frontier_append_warp(a.next, f1, d1, a.out_deg);
      frontier_append_warp(a.next, f2, d2, a.out_deg);
      frontier_append_warp(a.next, f3, d3, a.out_deg);
    }
    unsigned big = __ballot_sync(0xffffffffu, !own);
    while (big) {  // warp-uniform
      const int l = __ffs(big) - 1;
      big &= big - 1;
      const uint32_t uu = __shfl_sync(0xffffffffu, u, l);
      const uint64_t bb = __shfl_sync(0xffffffffu, b, l);
      const uint64_t ee = __shfl_sync(0xffffffffu, e_end, l);
      for (uint64_t base = bb; base < ee; base += 32) {
        const uint64_t e = base + lane;
        uint32_t dst = 0;
        bool fresh = false;
        if (e < ee) {
          dst = a.out_adj[e];
          fresh = bfs_claim(a, uu, dst, a.visited[dst >> 5]);
        }
        frontier_append_warp(a.next, fresh, dst, a.out_deg);
      }
    }
  }
}

// Pull step: every unvisited vertex takes the first in-neighbour (CSC order)
// that is in the current frontier.  A thread per row tests the row's first
// four in-edges (all ids, then all bitmap probes, in flight together); most
// rows of a pull level stop there.  The rows still open are finished by
// their warp, one row at a time, in rounds of 32 in-edges whose first hit is
// found with a ballot, so the parent equals that of a one-by-one scan.
__device__ __forceinline__ void bfs_pull_step(const bfs_level_args& a, append_smem& app) {
  const unsigned lane = threadIdx.x & 31;
  const uint32_t* cur = a.cur.bits;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  const uint64_t rounds = (a.V + stride - 1) / stride;
  // the next row's visited bit and offsets are loaded one round ahead (only
  // this thread can mark its own rows visited during a pull step)
  uint64_t v_next = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  bool todo_next = false;
  uint64_t b_next = 0, e_next = 0;
  if (v_next < a.V && !test_bit(a.visited, static_cast<uint32_t>(v_next))) {
    todo_next = true;
    b_next = a.in_off[v_next];
    e_next = a.in_off[v_next + 1];
  }
  for (uint64_t r = 0; r < rounds; ++r) {  // warp-uniform trip count
    const uint64_t v64 = v_next;
    const uint32_t v = static_cast<uint32_t>(v64);
    const bool todo = todo_next;
    const uint64_t b = b_next;
    uint64_t e = e_next;
    v_next = v64 + stride;
    todo_next = false;
    if (v_next < a.V && !test_bit(a.visited, static_cast<uint32_t>(v_next))) {
      todo_next = true;
      b_next = a.in_off[v_next];
      e_next = a.in_off[v_next + 1];
    }
    bool found = false, open = false;
    uint32_t par = 0;
    uint64_t next_edge = 0;
    if (todo) {
      const bool p0 = b < e, p1 = b + 1 < e, p2 = b + 2 < e, p3 = b + 3 < e;
      const uint32_t s0 = p0 ? a.in_adj[b] : 0u;
      const uint32_t s1 = p1 ? a.in_adj[b + 1] : 0u;
      const uint32_t s2 = p2 ? a.in_adj[b + 2] : 0u;
      const uint32_t s3 = p3 ? a.in_adj[b + 3] : 0u;
      const bool h0 = p0 && test_bit(cur, s0);
      const bool h1 = p1 && test_bit(cur, s1);
      const bool h2 = p2 && test_bit(cur, s2);
      const bool h3 = p3 && test_bit(cur, s3);
      found = h0 || h1 || h2 || h3;
      par = h0 ? s0 : h1 ? s1 : h2 ? s2 : s3;
      next_edge = b + 4;
      open = !found && next_edge < e;
    }
    unsigned open_rows = __ballot_sync(0xffffffffu, open);
    while (open_rows) {  // warp-uniform
      const int l = __ffs(open_rows) - 1;
      open_rows &= open_rows - 1;
      const uint64_t rb = __shfl_sync(0xffffffffu, next_edge, l);
      const uint64_t re = __shfl_sync(0xffffffffu, e, l);
      for (uint64_t i = rb + lane; i - lane < re; i += 32) {
        const uint32_t sv = i < re ? a.in_adj[i] : 0u;
        const unsigned hit = __ballot_sync(0xffffffffu, i < re && test_bit(cur, sv));
        if (hit) {
          const uint32_t p = __shfl_sync(0xffffffffu, sv, __ffs(hit) - 1);
          if (lane == static_cast<unsigned>(l)) {
            found = true;
            par = p;
          }
          break;
        }
      }
    }
    if (found) {
      a.level[v] = a.new_level;
      a.parent[v] = par;
    }
    // A warp's rows of a round are 32 consecutive ids on one bitmap word that
    // no other thread touches during a pull step: one plain update per warp.
    const unsigned fm = __ballot_sync(0xffffffffu, found);
    if (lane == 0 && fm) {
      a.visited[v >> 5] |= fm;
      a.next.bits[v >> 5] |= fm;
    }
    frontier_append_block(a.next, found, v, a.out_deg, app);  // block-uniform: same rounds everywhere
  }
}

__global__ void __launch_bounds__(256, 8) k_bfs_level(bfs_level_args a) {
  __shared__ bool s_last;
  __shared__ append_smem s_app;
  bfs_control* c = a.ctrl;
  if (c->done) return;  // uniform: the search ended at an earlier level
  const int mode = c->mode;
  // the level after next writes into `spare`; nothing reads it in this level
  const uint32_t words = (a.V + 31) / 32;
  for (uint32_t w = blockIdx.x * blockDim.x + threadIdx.x; w < words; w += gridDim.x * blockDim.x)
    a.spare.bits[w] = 0;
  if (blockIdx.x == 0 && threadIdx.x < 3) a.spare.counters[threadIdx.x] = 0;

  if (mode == 1)
    bfs_push_step(a);
  else
    bfs_pull_step(a, s_app);

  // the last CTA to finish sees every append (fence + ticket) and decides
  // the next level (dualmode.hpp:264-279; bfs.hpp:92 ends on no activation)
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    s_last = atomicAdd(&c->arrived, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!s_last || threadIdx.x != 0) return;
  __threadfence();
  c->arrived = 0;
  const unsigned long long actives = atomicAdd(&a.next.counters[0], 0ull);
  const unsigned long long active_edges = atomicAdd(&a.next.counters[2], 0ull);
  if (mode == 1) c->pushes += 1;
  c->level += 1;
  c->visited += actives;
  if (actives == 0) {
    c->done = 1;
    return;
  }
  const int push = (static_cast<double>(active_edges) / a.edges) < a.threshold ? 1 : 0;
  c->mode = push;
  if (push && c->level < 64) c->trace |= 1ull << c->level;
}

int ensure_bfs_ws(plato_graph* g) {
  if (!g->bfs_ws) {
    g->bfs_ws = new (std::nothrow) bfs_workspace();
    if (!g->bfs_ws) return set_error(PLATO_ENOMEM, "bfs workspace: host allocation failed");
  }
  bfs_workspace* ws = g->bfs_ws;
  const uint32_t V = g->info.vertices;
  for (push_frontier& f : ws->fr) PLATO_TRY(frontier_alloc(f, g));
  PLATO_TRY(ws->visited.alloc((V + 31) / 32));
  PLATO_TRY(ws->level.alloc(V));
  PLATO_TRY(ws->parent.alloc(V));
  PLATO_TRY(ws->ctrl.alloc(1));
  PLATO_TRY(ws->root.alloc(1));
  if (!ws->h_ctrl)
    PLATO_CUDA_TRY(cudaMallocHost(reinterpret_cast<void**>(&ws->h_ctrl), sizeof(bfs_control)));
  if (!ws->h_root)
    PLATO_CUDA_TRY(cudaMallocHost(reinterpret_cast<void**>(&ws->h_root), sizeof(uint32_t)));
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

// Control word of the first level (bfs.hpp:86-96): push iff the root's
// out-degree over the stored edges is below the threshold (dualmode.hpp:261-279),
// decided on the device from the seeded frontier's degree sum.
__global__ void k_bfs_start(bfs_control* c, const unsigned long long* counters, double edges,
                            double threshold) {
  const bool push = (static_cast<double>(counters[2]) / edges) < threshold;
  *c = bfs_control{push ? 1 : 0, 0, 0, 0, 1ull, push ? 1ull : 0ull, 0u};
}

constexpr uint32_t kFirstBatch = 8;  // RMAT searches end within about 8 levels
constexpr uint64_t kStartKernels = 3 + kFirstBatch;  // init, seed, start, levels

// k_frontier_seed for a root held on the device (the start graph's copy).
__global__ void k_frontier_seed_at(frontier_view f, const uint32_t* __restrict__ vp,
                                   const uint32_t* __restrict__ deg) {
  // one warp
  const uint32_t v = *vp;
  const bool take = (threadIdx.x == 0);
  if (take) atomicOr(&f.bits[v >> 5], 1u << (v & 31));
  frontier_append_warp(f, take, v, deg);
}

// A launch inside a capture: its error is checked, and it is counted once
// per replay of the graph instead of at capture.
#define BFS_CAPTURED(name)                                                                  \
  do {                                                                                      \
    cudaError_t bfs_e_ = cudaGetLastError();                                                \
    if (bfs_e_ != cudaSuccess)                                                              \
      return set_error(PLATO_ECUDA, std::string("launch of ") + (name) + " failed: " +     \
                                        cudaGetErrorString(bfs_e_));                       \
  } while (0)

// The start graph's work (captured by bfs_impl): the root copied in from
// pinned memory, level / parent / visited cleared with the root set, the
// frontiers reset and seeded with the root, the first level's mode
// (bfs.hpp:86-96), kFirstBatch levels and the control word copied out.
int enqueue_start(plato_graph* g, bfs_workspace* ws, bfs_level_args a, uint32_t invalid_parent,
                  cudaStream_t st) {
  const uint32_t V = g->info.vertices;
  PLATO_CUDA_TRY(cudaMemcpyAsync(ws->root.p, ws->h_root, sizeof(uint32_t), cudaMemcpyHostToDevice, st));
  k_bfs_init<<<grid_for(V, 256), 256, 0, st>>>(V, ws->root.p, invalid_parent, ws->level.p, ws->parent.p,
                                                ws->visited.p);
  BFS_CAPTURED("k_bfs_init");
  PLATO_TRY(frontier_reset(ws->fr[0], V, st));
  PLATO_TRY(frontier_reset(ws->fr[1], V, st));
  k_frontier_seed_at<<<1, 32, 0, st>>>(ws->fr[0].view(), ws->root.p, g->out_deg.p);
  BFS_CAPTURED("k_frontier_seed_at");
  k_bfs_start<<<1, 1, 0, st>>>(ws->ctrl.p, ws->fr[0].counters.p, a.edges, a.threshold);
  BFS_CAPTURED("k_bfs_start");
  for (uint32_t launched = 0; launched < kFirstBatch; ++launched) {
    a.cur = ws->fr[launched % 3].view();
    a.next = ws->fr[(launched + 1) % 3].view();
    a.spare = ws->fr[(launched + 2) % 3].view();
    a.new_level = launched + 1;
    k_bfs_level<<<ws->level_blocks, 256, 0, st>>>(a);
    BFS_CAPTURED("k_bfs_level");
  }
  PLATO_CUDA_TRY(cudaMemcpyAsync(ws->h_ctrl, ws->ctrl.p, sizeof(bfs_control), cudaMemcpyDeviceToHost, st));
  return PLATO_OK;
}

int bfs_impl(plato_graph* g, const plato_bfs_opts* o, const plato_dualmode_opts* eo,
             cudaStream_t st, plato_run_stats* stats) {
  const uint32_t V = g->info.vertices;
  if (o->root >= V) return set_error(PLATO_EINVAL, "bfs: root out of range");
  const double threshold = eo ? eo->push_threshold : 0.05;
  PLATO_TRY(ensure_bfs_ws(g));
  bfs_workspace* ws = g->bfs_ws;
  const std::vector<uint32_t>* to_int = nullptr;  // host copy, fetched once per graph
  PLATO_TRY(host_to_internal(g, &to_int, st));
  const uint32_t root = to_int ? (*to_int)[o->root] : o->root;
  const uint32_t invalid_parent = g->info.max_v_i + 1;  // bfs.hpp:79
  const double edges = static_cast<double>(g->stored_edges);
  if (ws->level_blocks == 0) {  // one full wave of resident CTAs; the steps stride over their work
    int sms = 0, per_sm = 0;
    PLATO_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, g->device));
    PLATO_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_bfs_level, 256, 0));
    ws->level_blocks = static_cast<unsigned>(sms) * static_cast<unsigned>(std::max(per_sm, 1));
  }
  bfs_level_args a{};
  a.V = V;
  a.out_off = g->out_off.p;
  a.out_adj = g->out_adj.p;
  a.out_deg = g->out_deg.p;
  a.in_off = g->in_off.p;
  a.in_adj = g->in_adj.p;
  a.visited = ws->visited.p;
  a.level = ws->level.p;
  a.parent = ws->parent.p;
  a.ctrl = ws->ctrl.p;
  a.edges = edges;
  a.threshold = threshold;
  // The start graph: root in, state cleared, root seeded, first mode (decided
  // on the device from the seeded frontier's degree sum), the first
  // kFirstBatch levels and the control word out.  Levels enqueued after the
  // end return at once.  Captured once per graph and threshold; the buffers
  // it names never move (grow-only, sized by V), and the key below catches it
  // if they ever do.
  const void* key = ws->level.p;
  if (!ws->start || ws->start_threshold != threshold || ws->start_key != key) {
    if (ws->start) cudaGraphExecDestroy(ws->start);
    ws->start = nullptr;
    cudaGraph_t graph = nullptr;
    PLATO_CUDA_TRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    const int rc = enqueue_start(g, ws, a, invalid_parent, st);
    const cudaError_t ec = cudaStreamEndCapture(st, &graph);
    if (rc != PLATO_OK) {
      if (graph) cudaGraphDestroy(graph);
      return rc;
    }
    if (ec != cudaSuccess) return set_error(PLATO_ECUDA, std::string("bfs: capture failed: ") + cudaGetErrorString(ec));
    const cudaError_t ei = cudaGraphInstantiate(&ws->start, graph, 0);
    cudaGraphDestroy(graph);
    if (ei != cudaSuccess) {
      ws->start = nullptr;
      return set_error(PLATO_ECUDA, std::string("bfs: graph instantiation failed: ") + cudaGetErrorString(ei));
    }
    ws->start_threshold = threshold;
    ws->start_key = key;
  }
  *ws->h_root = root;  // read by the graph's first node
  PLATO_CUDA_TRY(cudaGraphLaunch(ws->start, st));
  count_launch(kStartKernels);
  PLATO_CUDA_TRY(cudaStreamSynchronize(st));
  // Rare deeper searches: more levels in batches, one poll each.
  for (uint32_t launched = kFirstBatch; !ws->h_ctrl->done;) {
    for (uint32_t k = 0; k < 4; ++k, ++launched) {
      a.cur = ws->fr[launched % 3].view();
      a.next = ws->fr[(launched + 1) % 3].view();
      a.spare = ws->fr[(launched + 2) % 3].view();
      a.new_level = launched + 1;
      k_bfs_level<<<ws->level_blocks, 256, 0, st>>>(a);
      PLATO_LAUNCHED("k_bfs_level");
    }
    PLATO_CUDA_TRY(cudaMemcpyAsync(ws->h_ctrl, ws->ctrl.p, sizeof(bfs_control), cudaMemcpyDeviceToHost, st));
    PLATO_CUDA_TRY(cudaStreamSynchronize(st));
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
