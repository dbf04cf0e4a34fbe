// Push-mode frontier: the device form of the reference's active-vertex subset
// (bitmap_t, plato/util/bitmap.hpp:43-350) plus the work list that
// broadcast_message walks (plato/graph/message_passing.hpp:286-335).
//
// A frontier holds
//   bits     membership bitmap, 32-bit words (ballot friendly),
//   queue    members in insertion order,
//   chunks   work items (vertex, k): edges [out_off[v] + k*C, min(+C, out_off[v+1]))
//            of a member, C = kPushChunk, so a hub's out-edges spread over
//            many warps and no warp walks more than C edges,
//   counters [0] members, [1] chunks, [2] sum of member out-degrees
//            (= active_edges of dualmode.hpp:264-277).
// Members are appended with warp-aggregated atomics: one atomic per warp for
// the queue slot, one for the chunk range, one for the degree sum.
#pragma once

#include "common.cuh"
#include "graph.cuh"

namespace plato_b200 {

constexpr uint32_t kPushChunk = 256;

struct frontier_view {
  uint32_t* bits;
  uint32_t* queue;
  uint2* chunks;
  unsigned long long* counters;
};

struct push_frontier {
  uint32_t V = 0;
  dbuf<uint32_t> bits;
  dbuf<uint32_t> queue;
  dbuf<uint2> chunks;
  dbuf<unsigned long long> counters;
  unsigned long long* h_counters = nullptr;  // pinned [3]
  push_frontier() = default;
  push_frontier(const push_frontier&) = delete;
  push_frontier& operator=(const push_frontier&) = delete;
  ~push_frontier() {
    if (h_counters) cudaFreeHost(h_counters);
  }
  frontier_view view() { return frontier_view{bits.p, queue.p, chunks.p, counters.p}; }
};

__device__ __forceinline__ bool test_bit(const uint32_t* bits, uint32_t v) {
  return (bits[v >> 5] >> (v & 31)) & 1u;
}

// Warp-collective append of the lanes with `take` set (all 32 lanes call).
__device__ __forceinline__ void frontier_append_warp(frontier_view f, bool take, uint32_t v,
                                                     const uint32_t* __restrict__ deg) {
  const unsigned lane = threadIdx.x & 31;
  const unsigned m = __ballot_sync(0xffffffffu, take);
  if (m == 0) return;
  const unsigned leader = __ffs(m) - 1;
  unsigned long long base = 0;
  if (lane == leader) base = atomicAdd(&f.counters[0], static_cast<unsigned long long>(__popc(m)));
  base = __shfl_sync(0xffffffffu, base, leader);
  const uint32_t dg = take ? deg[v] : 0u;
  if (take) f.queue[base + __popc(m & ((1u << lane) - 1u))] = v;
  // chunk range: warp inclusive scan of the chunk counts
  const uint32_t nch = (dg + kPushChunk - 1) / kPushChunk;
  uint32_t inc = nch;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t t = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= static_cast<unsigned>(o)) inc += t;
  }
  const uint32_t tot = __shfl_sync(0xffffffffu, inc, 31);
  unsigned long long cbase = 0;
  if (lane == leader && tot) cbase = atomicAdd(&f.counters[1], static_cast<unsigned long long>(tot));
  cbase = __shfl_sync(0xffffffffu, cbase, leader);
  for (uint32_t k = 0; k < nch; ++k) f.chunks[cbase + (inc - nch) + k] = make_uint2(v, k);
  const unsigned long long dsum = warp_sum(static_cast<unsigned long long>(dg));
  if (lane == leader && dsum) atomicAdd(&f.counters[2], dsum);
}

// Block-collective append (every thread of the block calls, the same number
// of times): warps reserve their slots with shared-memory atomics and one
// thread per block takes the block's ranges from the global counters, so the
// counters see one atomic per block and call instead of one per warp.
struct append_smem {
  unsigned long long base_q, base_c, dsum;
  uint32_t cnt_q, cnt_c;
};

__device__ __forceinline__ void frontier_append_block(frontier_view f, bool take, uint32_t v,
                                                      const uint32_t* __restrict__ deg,
                                                      append_smem& sm) {
  const unsigned lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    sm.cnt_q = 0;
    sm.cnt_c = 0;
    sm.dsum = 0;
  }
  __syncthreads();
  const unsigned m = __ballot_sync(0xffffffffu, take);
  const uint32_t dg = take ? deg[v] : 0u;
  const uint32_t nch = (dg + kPushChunk - 1) / kPushChunk;
  uint32_t inc = nch;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t t = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= static_cast<unsigned>(o)) inc += t;
  }
  const uint32_t tot = __shfl_sync(0xffffffffu, inc, 31);
  const unsigned long long dsum = warp_sum(static_cast<unsigned long long>(dg));
  uint32_t wq = 0, wc = 0;
  if (lane == 0 && m) {
    wq = atomicAdd(&sm.cnt_q, static_cast<uint32_t>(__popc(m)));
    if (tot) wc = atomicAdd(&sm.cnt_c, tot);
    if (dsum) atomicAdd(&sm.dsum, dsum);
  }
  wq = __shfl_sync(0xffffffffu, wq, 0);
  wc = __shfl_sync(0xffffffffu, wc, 0);
  __syncthreads();
  if (threadIdx.x == 0) {
    if (sm.cnt_q) sm.base_q = atomicAdd(&f.counters[0], static_cast<unsigned long long>(sm.cnt_q));
    if (sm.cnt_c) sm.base_c = atomicAdd(&f.counters[1], static_cast<unsigned long long>(sm.cnt_c));
    if (sm.dsum) atomicAdd(&f.counters[2], sm.dsum);
  }
  __syncthreads();
  if (take) {
    f.queue[sm.base_q + wq + __popc(m & ((1u << lane) - 1u))] = v;
    for (uint32_t k = 0; k < nch; ++k) f.chunks[sm.base_c + wc + (inc - nch) + k] = make_uint2(v, k);
  }
}

static __global__ void k_frontier_seed(frontier_view f, uint32_t v, const uint32_t* __restrict__ deg) {
  // one warp
  const bool take = (threadIdx.x == 0);
  if (take) atomicOr(&f.bits[v >> 5], 1u << (v & 31));
  frontier_append_warp(f, take, v, deg);
}

inline int frontier_alloc(push_frontier& f, const plato_graph* g) {
  const uint32_t V = g->info.vertices;
  f.V = V;
  PLATO_TRY(f.bits.alloc((V + 31) / 32));
  PLATO_TRY(f.queue.alloc(V));
  PLATO_TRY(f.chunks.alloc(static_cast<size_t>(V) + g->stored_edges / kPushChunk + 1));
  PLATO_TRY(f.counters.alloc(3));
  if (!f.h_counters)
    PLATO_CUDA_TRY(cudaMallocHost(reinterpret_cast<void**>(&f.h_counters), 3 * sizeof(unsigned long long)));
  return PLATO_OK;
}

inline int frontier_reset(push_frontier& f, uint32_t V, cudaStream_t st) {
  PLATO_CUDA_TRY(cudaMemsetAsync(f.bits.p, 0, ((V + 31) / 32) * sizeof(uint32_t), st));
  PLATO_CUDA_TRY(cudaMemsetAsync(f.counters.p, 0, 3 * sizeof(unsigned long long), st));
  return PLATO_OK;
}

inline int frontier_seed(push_frontier& f, const plato_graph* g, uint32_t v, cudaStream_t st) {
  k_frontier_seed<<<1, 32, 0, st>>>(f.view(), v, g->out_deg.p);
  PLATO_LAUNCHED("k_frontier_seed");
  return PLATO_OK;
}

// Copies the counters to the host (synchronises `st`).
inline int frontier_read(push_frontier& f, cudaStream_t st) {
  PLATO_CUDA_TRY(cudaMemcpyAsync(f.h_counters, f.counters.p, 3 * sizeof(unsigned long long),
                                 cudaMemcpyDeviceToHost, st));
  PLATO_CUDA_TRY(cudaStreamSynchronize(st));
  return PLATO_OK;
}

inline int frontier_active_edges(push_frontier& f, cudaStream_t st, uint64_t* active_edges) {
  PLATO_TRY(frontier_read(f, st));
  *active_edges = f.h_counters[2];
  return PLATO_OK;
}

// PPR push epoch (personalized_pagerank.hpp:225-239): every member u adds
// x[u] to y[dst] for its out-edges and marks dst active in the same frontier.
// The epoch walks the members it started with (the chunk count read before
// the launch).  In the reference the slot sets bits in the bitmap the
// broadcast is still scanning, so a vertex reached this epoch may be walked
// in it or not by thread timing; it holds x == 0, so the ranks are the same,
// and the order taken here is the one that leaves the active-edge count, and
// so the push/pull switch epoch, independent of timing.
static __global__ void __launch_bounds__(256) k_ppr_push(frontier_view f, unsigned long long nchunks,
                                                  const uint64_t* __restrict__ out_off,
                                                  const uint32_t* __restrict__ out_adj,
                                                  const uint32_t* __restrict__ deg,
                                                  const float* __restrict__ x, float* y) {
  const unsigned lane = threadIdx.x & 31;
  const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t c = warp; c < nchunks; c += nwarps) {
    const uint2 ch = f.chunks[c];
    const uint32_t u = ch.x;
    const uint64_t b = out_off[u] + static_cast<uint64_t>(ch.y) * kPushChunk;
    const uint64_t e_end = min(b + kPushChunk, out_off[u + 1]);
    const float xu = x[u];
    for (uint64_t base = b; base < e_end; base += 32) {
      const uint64_t e = base + lane;
      const bool valid = e < e_end;
      uint32_t dst = 0;
      bool fresh = false;
      if (valid) {
        dst = out_adj[e];
        atomicAdd(&y[dst], xu);
        const uint32_t bit = 1u << (dst & 31);
        if (!(f.bits[dst >> 5] & bit)) fresh = !(atomicOr(&f.bits[dst >> 5], bit) & bit);
      }
      frontier_append_warp(f, fresh, dst, deg);
    }
  }
}

inline int frontier_push_scatter(push_frontier& f, const plato_graph* g, const float* x, float* y,
                                 cudaStream_t st) {
  // the chunk count was read by the preceding frontier_active_edges()
  const unsigned long long nchunks = f.h_counters[1];
  if (nchunks == 0) return PLATO_OK;
  const unsigned blocks = grid_for(nchunks * 32, 256, 148 * 16);
  k_ppr_push<<<blocks, 256, 0, st>>>(f.view(), nchunks, g->out_off.p, g->out_adj.p, g->out_deg.p,
                                     x, y);
  PLATO_LAUNCHED("k_ppr_push");
  return PLATO_OK;
}

}  // namespace plato_b200
