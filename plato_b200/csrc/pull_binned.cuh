// Degree-binned pull gather with the rank update fused (the PageRank / PPR
// pull epoch: aggregate_message over the in-edges, message_passing.hpp:88-144,
// with the update of pagerank.hpp:118-135).
//
// The engine numbers vertices by descending in-degree, so the CSC columns fall
// into three contiguous bins, each with its own work granularity:
//   long   in-degree > kMidMax: one warp per work item, an item being a whole
//          row or a kLongPiece-edge piece of a hub row; lanes stride the edges
//          with four id loads and four rank gathers in flight each; pieces of
//          one hub row are summed in piece order by k_pull_hubs.
//   mid    kShortMax < in-degree <= kMidMax: 8 lanes per row.
//   short  in-degree <= kShortMax (empty rows included): one thread per row.
// Kernels run a fixed grid (a few CTAs per SM) and stride over their work, so
// each writes one delta partial per CTA.  Per-edge work is an id load, a
// gather and an add; no shared memory is used besides the delta reduction,
// so L1 keeps the most-gathered ranks (high in-degree goes with high
// out-degree in these graphs, and those ranks sit at the front of x); the
// streamed arrays (ids, offsets, degrees, old ranks) are read with
// evict-first loads so they do not push those ranks out of L1 and L2.  Every
// row is summed in a fixed order, so results are bit-for-bit reproducible.
#pragma once

#include "common.cuh"
#include "pull_merge.cuh"

namespace plato_b200 {

constexpr uint32_t kShortMax = 4;
constexpr uint32_t kMidMax = 32;
constexpr uint32_t kLongPiece = 4096;

struct pull_plan_view {
  uint32_t n_long, n_mid, V;      // rows [0,n_long) long, [n_long, n_long+n_mid) mid, rest short
  uint32_t n_items;               // long work items
  const uint2* items;             // (row, piece)
  uint32_t n_hubs;                // rows of the long bin with more than one piece
  const uint32_t* hub_rows;       // [n_hubs]
  const uint32_t* hub_item0;      // [n_hubs] first item of the row
  const uint32_t* hub_pieces;     // [n_hubs]
  float* piece_sum;               // [n_items]
};

template <class Update>
__global__ void __launch_bounds__(256, 8) k_pull_long(pull_plan_view pv, const uint64_t* __restrict__ off,
                                                   const uint32_t* __restrict__ adj,
                                                   const float* __restrict__ x, Update upd,
                                                   double* __restrict__ partials) {
  __shared__ double s_red[32];
  if (upd.skip()) return;
  const unsigned lane = threadIdx.x & 31;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  double dl = 0.0;
  for (uint32_t item = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; item < pv.n_items;
       item += nwarps) {
    const uint2 it = pv.items[item];
    const uint64_t rb = __ldcs(off + it.x), re = __ldcs(off + it.x + 1);
    const uint64_t b = rb + static_cast<uint64_t>(it.y) * kLongPiece;
    const uint64_t e = min(b + kLongPiece, re);
    float s0 = 0.f, s1 = 0.f, s2 = 0.f, s3 = 0.f;
    uint64_t i = b + lane;
    for (; i + 96 < e; i += 128) {
      const uint32_t a0 = __ldcs(adj + i), a1 = __ldcs(adj + i + 32), a2 = __ldcs(adj + i + 64),
                     a3 = __ldcs(adj + i + 96);
      s0 += __ldg(x + a0);
      s1 += __ldg(x + a1);
      s2 += __ldg(x + a2);
      s3 += __ldg(x + a3);
    }
    for (; i < e; i += 32) s0 += __ldg(x + __ldcs(adj + i));
    float s = (s0 + s1) + (s2 + s3);
    s = warp_sum(s);
    if (lane == 0) {
      if (re - rb <= kLongPiece)
        dl += upd.apply(it.x, s);
      else
        pv.piece_sum[item] = s;
    }
  }
  dl = block_sum<256>(dl, s_red);
  if (threadIdx.x == 0) partials[blockIdx.x] = dl;
}

template <class Update>
__global__ void __launch_bounds__(256) k_pull_hubs(pull_plan_view pv, Update upd,
                                                   double* __restrict__ partials) {
  __shared__ double s_red[32];
  if (upd.skip()) return;
  double dl = 0.0;
  for (uint32_t h = blockIdx.x * blockDim.x + threadIdx.x; h < pv.n_hubs; h += gridDim.x * blockDim.x) {
    const uint32_t i0 = pv.hub_item0[h], n = pv.hub_pieces[h];
    float y = 0.f;
    for (uint32_t k = 0; k < n; ++k) y += pv.piece_sum[i0 + k];
    dl += upd.apply(pv.hub_rows[h], y);
  }
  dl = block_sum<256>(dl, s_red);
  if (threadIdx.x == 0) partials[blockIdx.x] = dl;
}

template <class Update>
__global__ void __launch_bounds__(256) k_pull_mid(pull_plan_view pv, const uint64_t* __restrict__ off,
                                                  const uint32_t* __restrict__ adj,
                                                  const float* __restrict__ x, Update upd,
                                                  double* __restrict__ partials) {
  __shared__ double s_red[32];
  if (upd.skip()) return;
  const unsigned sub = threadIdx.x & 7;
  const uint32_t ngroups = (gridDim.x * blockDim.x) >> 3;
  // warp-uniform trip count: the shuffles below need all 32 lanes
  const uint32_t g0 = (blockIdx.x * blockDim.x + threadIdx.x) >> 3;
  const uint32_t rounds = (pv.n_mid + ngroups - 1) / ngroups;
  double dl = 0.0;
  for (uint32_t k = 0; k < rounds; ++k) {
    const uint32_t r = g0 + k * ngroups;
    const bool valid = r < pv.n_mid;
    float s = 0.f;
    uint32_t v = 0;
    if (valid) {
      v = pv.n_long + r;
      const uint64_t b = __ldcs(off + v), e = __ldcs(off + v + 1);
      for (uint64_t i = b + sub; i < e; i += 8) s += __ldg(x + __ldcs(adj + i));
    }
    s += __shfl_xor_sync(0xffffffffu, s, 4);
    s += __shfl_xor_sync(0xffffffffu, s, 2);
    s += __shfl_xor_sync(0xffffffffu, s, 1);
    if (valid && sub == 0) dl += upd.apply(v, s);
  }
  dl = block_sum<256>(dl, s_red);
  if (threadIdx.x == 0) partials[blockIdx.x] = dl;
}

template <class Update>
__global__ void __launch_bounds__(256) k_pull_short(pull_plan_view pv, const uint64_t* __restrict__ off,
                                                    const uint32_t* __restrict__ adj,
                                                    const float* __restrict__ x, Update upd,
                                                    double* __restrict__ partials) {
  __shared__ double s_red[32];
  if (upd.skip()) return;
  const uint32_t base = pv.n_long + pv.n_mid;
  double dl = 0.0;
  for (uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; base + r < pv.V;
       r += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t v = static_cast<uint32_t>(base + r);
    const uint64_t b = __ldcs(off + v), e = __ldcs(off + v + 1);
    float s = 0.f;
    for (uint64_t i = b; i < e; ++i) s += __ldg(x + __ldcs(adj + i));
    dl += upd.apply(v, s);
  }
  dl = block_sum<256>(dl, s_red);
  if (threadIdx.x == 0) partials[blockIdx.x] = dl;
}

// Device-side epoch control (the eps early exit of pagerank.hpp:137-139
// without a host round trip).  ctrl[0] = mode of the next epoch (0 normal,
// 1 final, 2 done), ctrl[1] = epochs run; delta[0] = last non-final delta
// (scaled to the reference's units by `scale`).
static __global__ void __launch_bounds__(1024) k_epoch_control(const double* __restrict__ partials,
                                                               uint32_t n, int* ctrl, double* delta,
                                                               double scale, double eps,
                                                               uint32_t iteration) {
  __shared__ double s_red[32];
  const int mode = ctrl[0];
  if (mode == 2) return;  // block-uniform
  const uint32_t per = (n + 1023) / 1024;
  const uint32_t b = threadIdx.x * per, e = min(n, b + per);
  double s = 0.0;
  for (uint32_t i = b; i < e; ++i) s += partials[i];
  s = block_sum<1024>(s, s_red);
  if (threadIdx.x == 0) {
    const int ran = ctrl[1] + 1;
    ctrl[1] = ran;
    if (mode == 1) {
      ctrl[0] = 2;
    } else {
      const double dlt = s * scale;
      delta[0] = dlt;
      if ((eps > 0.0 && dlt < eps) || static_cast<uint32_t>(ran) >= iteration - 1) ctrl[0] = 1;
    }
  }
}

}  // namespace plato_b200
