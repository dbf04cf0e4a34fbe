// Persistent warp-granular pull gather with hub ranks staged in shared memory.
//
// Same contract as k_pull_merge (pull_merge.cuh): y(v) = sum over in-edges of
// x[src], then the fused rank update of pagerank.hpp:118-135.  Differences:
//
//  * One 1024-thread CTA per SM.  Internal ids are sorted by descending
//    out-degree (PLATO_GRAPH_RELABEL), so x[0, H) holds the most-gathered
//    ranks; each CTA copies them to shared memory once per launch and gathers
//    with src < H read shared memory instead of L2.
//  * Work unit = one warp tile of 32*IPT merge items (Merrill & Garland merge
//    path).  Each warp walks a contiguous range of tiles and carries the
//    partial sum of the row that is still open at a tile boundary in a
//    register, so rows only need a cross-warp join at range boundaries.
//  * No block barriers after the hub copy: warps stage their own tile in a
//    private shared-memory slice, merge (IPT items per lane, odd IPT so lane
//    strides spread over banks), join row pieces with a warp segmented scan,
//    and finalise rows warp-cooperatively (coalesced deg / x / x' accesses).
//  * Source ids of the next tile are loaded while the current tile is merged.
//
// Rows that begin in an earlier range and end in range w are completed by
// k_pull_warp_fixup from the per-range carries, summed in range order, so the
// result is deterministic.
#pragma once

#include "common.cuh"
#include "pull_merge.cuh"

namespace plato_b200 {

template <int IPT>
struct pull_warp_cfg {
  static constexpr int kItems = 32 * IPT;
  static constexpr int kWarps = 32;  // 1024 threads
  static constexpr size_t kSliceBytes = (static_cast<size_t>(kItems) * 10 + 15) / 16 * 16;
  static constexpr size_t kSlices = kWarps * kSliceBytes;
  static size_t smem_bytes(uint32_t hub) { return (static_cast<size_t>(hub) * 4 + 15) / 16 * 16 + kSlices; }
};

struct pull_warp_args {
  const uint32_t* trow;   // [T+1] warp tile start rows
  const uint64_t* tedge;  // [T+1] warp tile start edges
  uint32_t T;
  uint64_t E;
  const uint64_t* off;
  const uint32_t* adj;
  const float* x;
  uint32_t H;             // x[0, H) staged in shared memory
  float* rcarry;          // [W] partial of the row open at the end of range w
  float* rhead;           // [W] range w's part of its first row when that row began earlier
  double* partials;       // [gridDim.x]
  const float* w = nullptr;  // per-edge weights (CSC order) of a weighted pull, else unused
};

__device__ __forceinline__ uint32_t warp_range_begin(uint32_t T, uint32_t w, uint32_t W) {
  return static_cast<uint32_t>(static_cast<uint64_t>(T) * w / W);
}

// kWeighted: y(v) = sum over in-edges of x[src] * w[edge] (weighted_pagerank.hpp:112-118
// with x = rank / out-weight-sum), the weights read alongside the ids.
template <int IPT, class Update, bool kWeighted = false>
__global__ void __launch_bounds__(1024, 1) k_pull_warp(pull_warp_args a, Update upd) {
  using C = pull_warp_cfg<IPT>;
  constexpr int ITEMS = C::kItems;
  extern __shared__ __align__(16) unsigned char smem[];
  float* s_hub = reinterpret_cast<float*>(smem);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  unsigned char* slice = smem + (static_cast<size_t>(a.H) * 4 + 15) / 16 * 16 + wid * C::kSliceBytes;
  float* s_val = reinterpret_cast<float*>(slice);
  float* s_y = s_val + ITEMS;
  uint16_t* s_rowend = reinterpret_cast<uint16_t*>(s_y + ITEMS);
  __shared__ double s_red[32];
  if (upd.skip()) return;  // device epoch control: nothing left to run

  {
    const float4* src4 = reinterpret_cast<const float4*>(a.x);
    float4* dst4 = reinterpret_cast<float4*>(s_hub);
    const uint32_t n4 = a.H / 4;
    for (uint32_t i = threadIdx.x; i < n4; i += blockDim.x) dst4[i] = __ldg(src4 + i);
    for (uint32_t i = n4 * 4 + threadIdx.x; i < a.H; i += blockDim.x) s_hub[i] = __ldg(a.x + i);
  }
  __syncthreads();

  const uint32_t W = gridDim.x * C::kWarps;
  const uint32_t w = blockIdx.x * C::kWarps + wid;
  const uint32_t tb = warp_range_begin(a.T, w, W), te = warp_range_begin(a.T, w + 1, W);
  double dl = 0.0;
  float wcarry = 0.f;
  if (tb < te) {
    const uint32_t row0 = a.trow[tb];
    const bool range_spans = a.off[row0] < a.tedge[tb];
    uint32_t i0 = row0, i1 = a.trow[tb + 1];
    uint64_t j0 = a.tedge[tb], j1 = a.tedge[tb + 1];
    uint32_t ids[IPT];
    float wts[IPT];
#pragma unroll
    for (int k = 0; k < IPT; ++k) {
      const uint64_t e = j0 + lane + 32 * k;
      ids[k] = e < a.E ? __ldg(a.adj + e) : 0u;
      if constexpr (kWeighted) wts[k] = e < a.E ? __ldg(a.w + e) : 0.f;
    }
    for (uint32_t t = tb; t < te; ++t) {
      const int nrows = static_cast<int>(i1 - i0);
      const int nnz = static_cast<int>(j1 - j0);
      // gathers + row ends of this tile
      float vals[IPT];
#pragma unroll
      for (int k = 0; k < IPT; ++k) {
        const uint32_t s = ids[k];
        vals[k] = (lane + 32 * k < nnz) ? (s < a.H ? s_hub[s] : __ldg(a.x + s)) : 0.f;
        if constexpr (kWeighted) vals[k] *= wts[k];
      }
      uint32_t re[IPT];
#pragma unroll
      for (int k = 0; k < IPT; ++k) {
        const int r = lane + 32 * k;
        re[k] = (r < nrows) ? static_cast<uint32_t>(__ldg(a.off + i0 + r + 1) - j0) : 0u;
      }
      // prefetch the next tile's coordinates and source ids
      uint32_t ni1 = i1;
      uint64_t nj1 = j1;
      if (t + 1 < te) {
        ni1 = a.trow[t + 2];
        nj1 = a.tedge[t + 2];
#pragma unroll
        for (int k = 0; k < IPT; ++k) {
          const uint64_t e = j1 + lane + 32 * k;
          ids[k] = e < a.E ? __ldg(a.adj + e) : 0u;
          if constexpr (kWeighted) wts[k] = e < a.E ? __ldg(a.w + e) : 0.f;
        }
      }
#pragma unroll
      for (int k = 0; k < IPT; ++k) {
        const int e = lane + 32 * k;
        if (e < nnz) s_val[e] = vals[k];
        if (e < nrows) s_rowend[e] = static_cast<uint16_t>(re[k]);
      }
      __syncwarp();

      // merge IPT items per lane
      const int total = nrows + nnz;
      const int diag = min(lane * IPT, total);
      int lo = max(diag - nnz, 0), hi = min(diag, nrows);
      while (lo < hi) {
        const int p = (lo + hi) >> 1;
        if (static_cast<int>(s_rowend[p]) <= diag - p - 1)
          lo = p + 1;
        else
          hi = p;
      }
      int ii = lo, jj = diag - lo;
      const int head = ii;
      const int nitems = min(IPT, total - diag);
      float sum = (lane == 0) ? wcarry : 0.f, head_sum = 0.f;
      bool head_done = false;
#pragma unroll
      for (int k = 0; k < IPT; ++k) {
        if (k < nitems) {
          if (ii < nrows && jj >= static_cast<int>(s_rowend[ii])) {
            if (ii == head) {
              head_done = true;
              head_sum = sum;
            } else {
              s_y[ii] = sum;
            }
            sum = 0.f;
            ++ii;
          } else {
            sum += s_val[jj];
            ++jj;
          }
        }
      }
      // warp segmented scan of (open row, partial) over lanes
      uint32_t key = static_cast<uint32_t>(ii);
      float val = sum;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t k2 = __shfl_up_sync(0xffffffffu, key, o);
        const float v2 = __shfl_up_sync(0xffffffffu, val, o);
        if (lane >= o && k2 == key) val = v2 + val;
      }
      const uint32_t pkey = __shfl_up_sync(0xffffffffu, key, 1);
      const float pval = __shfl_up_sync(0xffffffffu, val, 1);
      const bool first_partial = range_spans && i0 == row0;  // row 0 began before this range
      if (head_done) {
        const float y = ((lane > 0 && pkey == static_cast<uint32_t>(head)) ? pval : 0.f) + head_sum;
        if (head == 0 && first_partial)
          a.rhead[w] = y;
        else
          s_y[head] = y;
      }
      wcarry = __shfl_sync(0xffffffffu, val, 31);
      __syncwarp();
      for (int r = lane; r < nrows; r += 32) {
        if (r == 0 && first_partial) continue;
        dl += upd.apply(i0 + r, s_y[r]);
      }
      __syncwarp();
      i0 = i1;
      j0 = j1;
      i1 = ni1;
      j1 = nj1;
    }
  }
  if (lane == 0) a.rcarry[w] = (tb < te) ? wcarry : 0.f;
  dl = block_sum<1024>(dl, s_red);
  if (threadIdx.x == 0) a.partials[blockIdx.x] = dl;
}

// Rows that began before range w and end inside it: rhead[w] plus the carries
// of the preceding ranges that end inside the same row, in range order.
template <class Update>
__global__ void __launch_bounds__(256) k_pull_warp_fixup(pull_warp_args a, uint32_t W, Update upd) {
  __shared__ double s_red[32];
  if (upd.skip()) return;
  double dl = 0.0;
  const uint32_t w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= 1 && w < W) {
    const uint32_t tb = warp_range_begin(a.T, w, W), te = warp_range_begin(a.T, w + 1, W);
    if (tb < te) {
      const uint32_t r0 = a.trow[tb];
      if (a.off[r0] < a.tedge[tb] && a.trow[te] > r0) {
        uint32_t wf = w - 1;
        while (wf > 0 && a.trow[warp_range_begin(a.T, wf, W)] == r0) --wf;
        float y = 0.f;
        for (uint32_t u = wf; u < w; ++u) y += a.rcarry[u];
        y += a.rhead[w];
        dl = upd.apply(r0, y);
      }
    }
  }
  dl = block_sum<256>(dl, s_red);
  if (threadIdx.x == 0) a.partials[blockIdx.x] = dl;
}

}  // namespace plato_b200
