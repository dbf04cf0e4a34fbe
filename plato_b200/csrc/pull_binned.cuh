// Degree-binned pull gather with the rank update fused (the PageRank / PPR
// pull epoch: aggregate_message over the in-edges, message_passing.hpp:88-144,
// with the update of pagerank.hpp:118-135).
//
// The engine numbers vertices by descending in-degree, so the CSC columns fall
// into contiguous bins, each with its own work granularity:
//   long   in-degree > 64: one warp per work unit, a unit being a
//          kLongPiece-edge piece of a hub row or a group of up to 32
//          consecutive rows; the id loads of the next round of 128 edges
//          overlap the rank gathers of this one; pieces of one hub row are
//          summed in piece order by k_pull_hubs.
//   rows   33..64, 17..32, 5..16: k_pull_rows with 16, 8 or 4 lanes per
//          row, each row in one round of four edges per lane, rounds
//          pipelined the same way.
//   short  in-degree <= kShortMax (empty rows included): one thread per row.
// Kernels run a fixed grid (a few CTAs per SM) and stride over their work, so
// each writes one delta partial per CTA.  Per-edge work is an id load, a
// gather and an add; no shared memory is used besides the delta reduction,
// so L1 keeps the most-gathered ranks (high in-degree goes with high
// out-degree in these graphs, and those ranks sit at the front of x); the
// streamed arrays (ids, offsets, degrees, old ranks) are read with
// evict-first loads so they do not push those ranks out of L1 and L2.  Every
// row is summed in a fixed order, so results are bit-for-bit reproducible.
// With kW (weighted PageRank, weighted_pagerank.hpp:112-118) each gathered
// value is multiplied by its edge's weight, read like the ids from w (CSC
// order), pipelined with them.
#pragma once

#include "common.cuh"
#include "pull_merge.cuh"

namespace plato_b200 {

constexpr uint32_t kShortMax = 4;
constexpr uint32_t kRowsMax[3] = {64, 32, 16};  // k_pull_rows<16>, <8>, <4>: in-degree <= 4 * LPR
constexpr uint32_t kLongPiece = 4096;

struct pull_plan_view {
  uint32_t n_long, short_begin, V;  // rows [0,n_long) long, [short_begin, V) short
  uint32_t n_items;               // long work items
  const uint2* items;             // long-bin units (see k_pull_long)
  uint32_t n_hubs;                // rows of the long bin with more than one piece
  const uint32_t* hub_rows;       // [n_hubs]
  const uint32_t* hub_item0;      // [n_hubs] first item of the row
  const uint32_t* hub_pieces;     // [n_hubs]
  float* piece_sum;               // [n_items]
};

// Long-bin work units (pull_plan_view::items), hub pieces first:
//   (row, kPieceFlag | k)  edges [k*kLongPiece, (k+1)*kLongPiece) of a hub row
//   (row0, n)              rows [row0, row0+n), n <= 32, at most kGroupEdges
//                          edges in all unless n == 1
constexpr uint32_t kPieceFlag = 0x80000000u;
constexpr uint32_t kGroupRows = 32;
constexpr uint32_t kGroupEdges = 4096;

// Ids of one round: edges [i, i+128) of the current segment clipped to e,
// lane l taking i+l, i+l+32, i+l+64, i+l+96.
struct round_ids {
  uint32_t a0, a1, a2, a3;
  __device__ __forceinline__ void load(const uint32_t* __restrict__ ab, uint32_t j, uint32_t e) {
    a0 = j < e ? __ldcs(ab + j) : 0u;
    a1 = j + 32 < e ? __ldcs(ab + j + 32) : 0u;
    a2 = j + 64 < e ? __ldcs(ab + j + 64) : 0u;
    a3 = j + 96 < e ? __ldcs(ab + j + 96) : 0u;
  }
};

// Weights of one round, at the same positions as round_ids.
struct round_w {
  float w0, w1, w2, w3;
  __device__ __forceinline__ void load(const float* __restrict__ wb, uint32_t j, uint32_t e) {
    w0 = j < e ? __ldcs(wb + j) : 0.f;
    w1 = j + 32 < e ? __ldcs(wb + j + 32) : 0.f;
    w2 = j + 64 < e ? __ldcs(wb + j + 64) : 0.f;
    w3 = j + 96 < e ? __ldcs(wb + j + 96) : 0.f;
  }
};

// One warp per unit.  A unit's segments (one hub piece, or up to 32 whole
// rows) are walked in rounds of 128 edges, software-pipelined one round
// deep: the ids of the next round (possibly of the next row) are loaded
// before the ranks of this round are gathered, so an id load and a gather
// overlap instead of running back to back.  Lane j keeps the sum of segment
// j and applies the update of row row0+j, so the offsets, degrees and old
// ranks of a group are read with one coalesced access each.
template <class Update, bool kW = false>
__global__ void __launch_bounds__(256, 8) k_pull_long(pull_plan_view pv, const uint64_t* __restrict__ off,
                                                   const uint32_t* __restrict__ adj,
                                                   const float* __restrict__ x, Update upd,
                                                   double* __restrict__ partials,
                                                   const float* __restrict__ w) {
  __shared__ double s_red[32];
  if (upd.skip()) return;
  const unsigned lane = threadIdx.x & 31;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  double dl = 0.0;
  uint32_t unit = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  uint2 it = unit < pv.n_items ? pv.items[unit] : make_uint2(0, 0);
  for (; unit < pv.n_items; unit += nwarps) {
    const uint32_t un = unit + nwarps;
    const uint2 it_next = un < pv.n_items ? pv.items[un] : make_uint2(0, 0);
    const bool piece = (it.y & kPieceFlag) != 0;
    const uint32_t nseg = piece ? 1u : it.y;
    uint64_t base;
    uint32_t sb = 0, se = 0;  // this lane's segment, relative to base
    if (piece) {
      const uint64_t rb = __ldcs(off + it.x), re = __ldcs(off + it.x + 1);
      base = rb + static_cast<uint64_t>(it.y & ~kPieceFlag) * kLongPiece;
      if (lane == 0) se = static_cast<uint32_t>(min(static_cast<uint64_t>(kLongPiece), re - base));
    } else {
      uint64_t lo = 0, hi = 0;
      if (lane < nseg) {
        lo = __ldcs(off + it.x + lane);
        hi = __ldcs(off + it.x + lane + 1);
      }
      base = __shfl_sync(0xffffffffu, lo, 0);
      sb = static_cast<uint32_t>(lo - base);
      se = static_cast<uint32_t>(hi - base);
    }
    const bool mine = !piece && lane < nseg;
    const typename Update::operands ops = upd.load(mine ? it.x + lane : it.x);
    const uint32_t* ab = adj + base;
    const float* wb = kW ? w + base : nullptr;
    uint32_t k = 0;
    uint32_t i = __shfl_sync(0xffffffffu, sb, 0), e = __shfl_sync(0xffffffffu, se, 0);
    round_ids cur;
    cur.load(ab, i + lane, e);
    round_w cw{0.f, 0.f, 0.f, 0.f};
    if constexpr (kW) cw.load(wb, i + lane, e);
    float s = 0.f, res = 0.f;
    for (;;) {
      // cursor of the next round (warp-uniform)
      uint32_t kn = k, in = i + 128, en = e;
      if (in >= e) {
        kn = k + 1;
        const uint32_t src = kn < nseg ? kn : 0;
        in = __shfl_sync(0xffffffffu, sb, src);
        en = __shfl_sync(0xffffffffu, se, src);
      }
      const bool more = kn < nseg;
      round_ids nxt{0u, 0u, 0u, 0u};
      round_w nw{0.f, 0.f, 0.f, 0.f};
      if (more) {
        nxt.load(ab, in + lane, en);
        if constexpr (kW) nw.load(wb, in + lane, en);
      }
      const uint32_t j = i + lane;
      float g0 = j < e ? __ldg(x + cur.a0) : 0.f;
      float g1 = j + 32 < e ? __ldg(x + cur.a1) : 0.f;
      float g2 = j + 64 < e ? __ldg(x + cur.a2) : 0.f;
      float g3 = j + 96 < e ? __ldg(x + cur.a3) : 0.f;
      if constexpr (kW) {
        g0 *= cw.w0;
        g1 *= cw.w1;
        g2 *= cw.w2;
        g3 *= cw.w3;
        cw = nw;
      }
      s += (g0 + g1) + (g2 + g3);
      if (kn != k) {
        const float t = warp_sum(s);
        if (lane == k) res = t;
        s = 0.f;
      }
      if (!more) break;
      cur = nxt;
      k = kn;
      i = in;
      e = en;
    }
    if (piece) {
      if (lane == 0) pv.piece_sum[unit] = res;
    } else if (mine) {
      dl += upd.apply(it.x + lane, res, ops);
    }
    it = it_next;
  }
  dl = block_sum<256>(dl, s_red);
  if (threadIdx.x == 0) partials[blockIdx.x] = dl;
}

template <class Update>
__global__ void __launch_bounds__(256) k_pull_hubs(pull_plan_view pv, Update upd,
                                                   double* __restrict__ partials) {
  __shared__ double s_red[32];
  if (upd.skip()) return;
  // one warp per hub row: lane l sums pieces l, l+32, ..., then a butterfly
  // (a fixed order, so the row sum is reproducible)
  const unsigned lane = threadIdx.x & 31;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  double dl = 0.0;
  for (uint32_t h = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; h < pv.n_hubs; h += nwarps) {
    const uint32_t i0 = pv.hub_item0[h], n = pv.hub_pieces[h];
    float y = 0.f;
    for (uint32_t k = lane; k < n; k += 32) y += pv.piece_sum[i0 + k];
    y = warp_sum(y);
    if (lane == 0) dl += upd.apply(pv.hub_rows[h], y);
  }
  dl = block_sum<256>(dl, s_red);
  if (threadIdx.x == 0) partials[blockIdx.x] = dl;
}

// Ids of one single-round row: edges b+q, b+q+LPR, b+q+2*LPR, b+q+3*LPR
// clipped to e (lane q of the row's LPR lanes).
template <int LPR>
struct row_ids {
  uint32_t a0, a1, a2, a3;
  __device__ __forceinline__ void load(const uint32_t* __restrict__ ab, uint32_t j, uint32_t e) {
    a0 = j < e ? __ldcs(ab + j) : 0u;
    a1 = j + LPR < e ? __ldcs(ab + j + LPR) : 0u;
    a2 = j + 2 * LPR < e ? __ldcs(ab + j + 2 * LPR) : 0u;
    a3 = j + 3 * LPR < e ? __ldcs(ab + j + 3 * LPR) : 0u;
  }
};

// Rank gather of the row bins: the first kHotRanks ranks (the most gathered,
// at the front of x on a relabelled graph) through L1 as usual, the others
// without allocating L1 lines, so that cold ranks do not evict hot ones
// (k_pull_rows16/8/4 0.195 -> 0.184 ms per epoch at RMAT s24; the long bin
// loses with the same split, 0.598 -> 0.610 ms, and keeps plain loads).
constexpr uint32_t kHotRanks = 65536;
__device__ __forceinline__ float ld_rank_rows(const float* __restrict__ x, uint32_t s) {
  if (s < kHotRanks) return __ldg(x + s);
  float v;
  asm("ld.global.nc.L1::no_allocate.f32 %0, [%1];" : "=f"(v) : "l"(x + s));
  return v;
}

template <int LPR>
struct row_w {
  float w0, w1, w2, w3;
  __device__ __forceinline__ void load(const float* __restrict__ wb, uint32_t j, uint32_t e) {
    w0 = j < e ? __ldcs(wb + j) : 0.f;
    w1 = j + LPR < e ? __ldcs(wb + j + LPR) : 0.f;
    w2 = j + 2 * LPR < e ? __ldcs(wb + j + 2 * LPR) : 0.f;
    w3 = j + 3 * LPR < e ? __ldcs(wb + j + 3 * LPR) : 0.f;
  }
};

// Rows [r0, r1) whose in-degree is at most 4*LPR.  One warp per unit of 32
// consecutive rows; a round gives each row LPR lanes with four edges each, so
// it covers 32/LPR rows and a unit takes LPR rounds.  The ids of the next
// round are loaded while the ranks of this round are gathered; the offsets of
// the warp's next unit and the update operands of this unit are loaded at the
// start of the unit.  Lane j ends up with the sum of row row0+j, so offsets,
// operands and new ranks move with one coalesced access each.
template <int LPR, class Update, bool kW = false>
__global__ void __launch_bounds__(256, 8) k_pull_rows(uint32_t r0, uint32_t r1, const uint64_t* __restrict__ off,
                                                   const uint32_t* __restrict__ adj,
                                                   const float* __restrict__ x, Update upd,
                                                   double* __restrict__ partials,
                                                   const float* __restrict__ w) {
  static_assert(LPR == 4 || LPR == 8 || LPR == 16, "k_pull_rows: 4, 8 or 16 lanes per row");
  constexpr uint32_t RPR = 32 / LPR;  // rows per round
  __shared__ double s_red[32];
  if (upd.skip()) return;
  const unsigned lane = threadIdx.x & 31, slot = lane / LPR, q = lane % LPR;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  const uint32_t n_units = (r1 - r0 + 31) / 32;
  double dl = 0.0;
  uint32_t unit = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  uint64_t lo = 0, hi = 0;
  if (unit < n_units && r0 + unit * 32 + lane < r1) {
    lo = __ldcs(off + r0 + unit * 32 + lane);
    hi = __ldcs(off + r0 + unit * 32 + lane + 1);
  }
  for (; unit < n_units; unit += nwarps) {
    const uint32_t row0 = r0 + unit * 32, un = unit + nwarps;
    uint64_t lo_n = 0, hi_n = 0;
    if (un < n_units && r0 + un * 32 + lane < r1) {
      lo_n = __ldcs(off + r0 + un * 32 + lane);
      hi_n = __ldcs(off + r0 + un * 32 + lane + 1);
    }
    const bool mine = row0 + lane < r1;
    const typename Update::operands ops = upd.load(mine ? row0 + lane : row0);
    const uint64_t base = __shfl_sync(0xffffffffu, lo, 0);
    const uint32_t sb = mine ? static_cast<uint32_t>(lo - base) : 0u;
    const uint32_t se = mine ? static_cast<uint32_t>(hi - base) : 0u;
    const uint32_t* ab = adj + base;
    const float* wb = kW ? w + base : nullptr;
    uint32_t b = __shfl_sync(0xffffffffu, sb, slot), e = __shfl_sync(0xffffffffu, se, slot);
    row_ids<LPR> cur;
    cur.load(ab, b + q, e);
    row_w<LPR> cw{0.f, 0.f, 0.f, 0.f};
    if constexpr (kW) cw.load(wb, b + q, e);
    float res = 0.f;
#pragma unroll 1
    for (uint32_t t = 0; t < LPR; ++t) {  // 32 rows / RPR rows per round = LPR rounds
      uint32_t bn = 0, en = 0;
      row_ids<LPR> nxt{0u, 0u, 0u, 0u};
      row_w<LPR> nw{0.f, 0.f, 0.f, 0.f};
      if (t + 1 < LPR) {
        bn = __shfl_sync(0xffffffffu, sb, (t + 1) * RPR + slot);
        en = __shfl_sync(0xffffffffu, se, (t + 1) * RPR + slot);
        nxt.load(ab, bn + q, en);
        if constexpr (kW) nw.load(wb, bn + q, en);
      }
      const uint32_t j = b + q;
      float g0 = j < e ? ld_rank_rows(x, cur.a0) : 0.f;
      float g1 = j + LPR < e ? ld_rank_rows(x, cur.a1) : 0.f;
      float g2 = j + 2 * LPR < e ? ld_rank_rows(x, cur.a2) : 0.f;
      float g3 = j + 3 * LPR < e ? ld_rank_rows(x, cur.a3) : 0.f;
      if constexpr (kW) {
        g0 *= cw.w0;
        g1 *= cw.w1;
        g2 *= cw.w2;
        g3 *= cw.w3;
        cw = nw;
      }
      float s = (g0 + g1) + (g2 + g3);
#pragma unroll
      for (int o = LPR / 2; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
      // row t*RPR + k sits in lanes k*LPR..; lane L collects row L in round L / RPR
      const float v = __shfl_sync(0xffffffffu, s, (lane % RPR) * LPR);
      if (lane / RPR == t) res = v;
      cur = nxt;
      b = bn;
      e = en;
    }
    if (mine) dl += upd.apply(row0 + lane, res, ops);
    lo = lo_n;
    hi = hi_n;
  }
  dl = block_sum<256>(dl, s_red);
  if (threadIdx.x == 0) partials[blockIdx.x] = dl;
}

template <class Update, bool kW = false>
__global__ void __launch_bounds__(256) k_pull_short(pull_plan_view pv, const uint64_t* __restrict__ off,
                                                    const uint32_t* __restrict__ adj,
                                                    const float* __restrict__ x, Update upd,
                                                    double* __restrict__ partials,
                                                    const float* __restrict__ w) {
  __shared__ double s_red[32];
  if (upd.skip()) return;
  const uint32_t base = pv.short_begin;
  double dl = 0.0;
  for (uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; base + r < pv.V;
       r += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t v = static_cast<uint32_t>(base + r);
    // at most kShortMax edges: all id loads, then all gathers, predicated
    static_assert(kShortMax <= 4, "k_pull_short covers a row in one round of 4");
    const uint64_t b = __ldcs(off + v), e = __ldcs(off + v + 1);
    const bool p0 = b < e, p1 = b + 1 < e, p2 = b + 2 < e, p3 = b + 3 < e;
    const uint32_t a0 = p0 ? __ldcs(adj + b) : 0u;
    const uint32_t a1 = p1 ? __ldcs(adj + b + 1) : 0u;
    const uint32_t a2 = p2 ? __ldcs(adj + b + 2) : 0u;
    const uint32_t a3 = p3 ? __ldcs(adj + b + 3) : 0u;
    float g0 = p0 ? __ldg(x + a0) : 0.f, g1 = p1 ? __ldg(x + a1) : 0.f;
    float g2 = p2 ? __ldg(x + a2) : 0.f, g3 = p3 ? __ldg(x + a3) : 0.f;
    if constexpr (kW) {
      g0 *= p0 ? __ldcs(w + b) : 0.f;
      g1 *= p1 ? __ldcs(w + b + 1) : 0.f;
      g2 *= p2 ? __ldcs(w + b + 2) : 0.f;
      g3 *= p3 ? __ldcs(w + b + 3) : 0.f;
    }
    const float s = (g0 + g1) + (g2 + g3);
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
