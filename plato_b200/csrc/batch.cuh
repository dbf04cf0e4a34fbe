// Batched multi-source personalized PageRank: one pull sweep serves many
// queries (columns) at once.
//
// Semantics per column q (seed set S_q) follow algo::trustrank
// (plato/algo/trustrank/trustrank.hpp:197-245) with explicit seeds:
//   init      x = (1/|S_q|) / deg on seeds (1/|S_q| when deg == 0), 0 elsewhere
//   epoch     y = sum over in-edges of x;  r = tele_q(v) + d * y,
//             tele_q(v) = (1-d)/|S_q| on seeds, 0 elsewhere;
//             x' = r / deg (deg > 0) or r; delta_q = sum |x' - x| * deg
//   stop      after a non-final epoch with delta_q < eps, or at epoch
//             max_iterations - 1, the next epoch is the final one and stores r
//             (pagerank.hpp:118-140).
//
// Layout (HBM): the V x K state is stored tile-major, X[tile][v][kt], one
// tile = kt consecutive columns, so one sweep over a tile touches a dense
// V x kt block (kt*4 bytes per vertex, whole L2 sectors) and the vertex-row
// gather of an edge is one coalesced kt-float load.  Each column tile is one
// launch of k_batch_pull over the same merge-path tiles as the scalar pull
// kernel; a group of GL lanes owns a run of merge items and each lane holds
// VEC columns (kt = GL * VEC).  Column states live on the device, so a whole
// iteration is a fixed launch sequence that is captured in a CUDA graph.
#pragma once

#include "graph.cuh"

namespace plato_b200 {

enum : uint8_t { COL_FREE = 0, COL_LIVE = 1, COL_FINAL = 2, COL_DONE = 3 };

// Merge items per CTA by column-tile width.  2048 below kt 128; 3072 at kt
// 128, where a group's row pieces are wider (one B200, queries/s against
// 2048: RMAT s22 K = 256 / 1024 +0.2% / +1.1%, RMAT s24 K = 128 +1.3%; at
// kt 64 RMAT s22 K = 64 -1.2%).  1024 was 5-9% slower; 4096 (41 KB of shared
// memory) leaves fewer CTAs per SM and loses 10%.
constexpr int batch_tile_items(int kt) { return kt >= 128 ? 3072 : 2048; }
// Row gathers in flight per lane and CTAs per SM of k_batch_pull: 4 at 5 CTAs
// beat 8 at 4 (K = 64: 103.6 -> 100.9 ms per batch at RMAT s22; 6 or 8 at 5
// CTAs spill and lose 7%).
constexpr int kBatchInflight = 4;
constexpr int kBatchMinBlocks = 5;

struct seed_index_view {
  const uint32_t* off;   // [V+1] by internal vertex
  const uint32_t* col;   // [S] global column
  const float* tele;     // [S] (1-d)/|S_q|
};

struct batch_pass {
  const uint32_t* trow;
  const uint64_t* tedge;
  uint32_t T;
  uint32_t V;
  uint32_t rows;         // partial rows per column tile: T + fixup blocks
  const uint64_t* off;
  const uint32_t* adj;
  const uint32_t* deg;
  const float* X;   // column tile ct at X + ct * V * kt: [V][kt]
  float* Xn;
  const uint8_t* state;  // [K] column states
  seed_index_view seeds;
  uint32_t col_base;     // global column of the tile's first column (set per tile)
  float d;
  float* tcarry;         // per column tile: [T][kt]
  float* thead;          // per column tile: [T][kt]
  double* partials;      // per column tile: [rows][kt]
  uint32_t hot_rows;     // rows gathered with normal L2 priority; the colder rest evict first
};

// Pointers of column tile blockIdx.y (grids are (tiles, column tiles)).
template <int KT>
__device__ __forceinline__ batch_pass batch_tile_view(const batch_pass& p) {
  batch_pass q = p;
  const size_t ct = blockIdx.y;
  q.X += ct * p.V * KT;
  q.Xn += ct * p.V * KT;
  q.state += ct * KT;
  q.col_base = static_cast<uint32_t>(ct * KT);
  q.tcarry += ct * p.T * KT;
  q.thead += ct * p.T * KT;
  q.partials += ct * p.rows * KT;
  return q;
}

template <int VEC>
__device__ __forceinline__ void ldvec(const float* p, float (&a)[VEC]) {
  if constexpr (VEC == 1) {
    a[0] = __ldg(p);
  } else if constexpr (VEC == 2) {
    const float2 t = __ldg(reinterpret_cast<const float2*>(p));
    a[0] = t.x;
    a[1] = t.y;
  } else {
    const float4 t = __ldg(reinterpret_cast<const float4*>(p));
    a[0] = t.x;
    a[1] = t.y;
    a[2] = t.z;
    a[3] = t.w;
  }
}

// 16-byte load with an L2 cache policy (createpolicy).  k_batch_pull gathers
// every row through one range policy: the hottest rows (the first hot_rows
// vertices: on a relabelled graph the highest in-degrees, which on these
// graphs are also the most gathered; half of L2 for one column tile, as the
// tiles of a launch run one after another) at normal priority, all colder
// rows evict-first, so they do not push the hot rows out of L2.  Against
// plain loads for every row the split gained 2-8%; making it by address (one
// load form, no compare per gather) instead of choosing between a plain and
// an evict-first load per row gained another 4-14% (one B200, queries/s,
// RMAT s22 K = 64 / 256 / 1024: 630 / 753 / 773 -> 716 / 792 / 818; RMAT
// s24 K = 64 / 128: 158.5 / 173 -> 171 / 179).  Choosing between two policy
// registers per gather gains nothing.
__device__ __forceinline__ void ld4_pol(const float* p, float (&a)[4], uint64_t pol) {
  asm("ld.global.nc.L2::cache_hint.v4.f32 {%0,%1,%2,%3}, [%4], %5;"
      : "=f"(a[0]), "=f"(a[1]), "=f"(a[2]), "=f"(a[3])
      : "l"(p), "l"(pol));
}

// Evict-first variant for the state streams (old row read once, new row
// written once): they must not push the hot gathered rows out of L2.
template <int VEC>
__device__ __forceinline__ void ldvec_cs(const float* p, float (&a)[VEC]) {
  if constexpr (VEC == 4) {
    const float4 t = __ldcs(reinterpret_cast<const float4*>(p));
    a[0] = t.x;
    a[1] = t.y;
    a[2] = t.z;
    a[3] = t.w;
  } else {
#pragma unroll
    for (int c = 0; c < VEC; ++c) a[c] = __ldcs(p + c);
  }
}

// Per-lane column flags, fixed for a launch (batch_finalize's fast paths).
enum : uint32_t { kLaneRunning = 1u, kLaneLive = 2u, kLaneAll = 4u };
template <int VEC>
__device__ __forceinline__ uint32_t lane_flags_of(const uint8_t (&st)[VEC]) {
  bool running = false, live = false, all = true;
#pragma unroll
  for (int c = 0; c < VEC; ++c) {
    const bool w = st[c] == COL_LIVE || st[c] == COL_FINAL;
    running |= w;
    live |= st[c] == COL_LIVE;
    all &= w;
  }
  return (running ? kLaneRunning : 0u) | (live ? kLaneLive : 0u) | (all ? kLaneAll : 0u);
}

// Update of one vertex row for this lane's VEC columns.
template <int GL, int VEC>
__device__ __forceinline__ void batch_finalize(const batch_pass& p, uint32_t v,
                                               const float (&y)[VEC], const uint8_t (&st)[VEC],
                                               int lane_g, uint32_t lane_flags, float (&dl)[VEC]) {
  constexpr int KT = GL * VEC;
  if (!(lane_flags & kLaneRunning)) return;  // nothing of this lane's columns is read or written
  float tele[VEC];
#pragma unroll
  for (int c = 0; c < VEC; ++c) tele[c] = 0.f;
  const uint32_t s0 = p.seeds.off[v], s1 = p.seeds.off[v + 1];
  for (uint32_t e = s0; e < s1; ++e) {
    const uint32_t c = p.seeds.col[e] - p.col_base - static_cast<uint32_t>(lane_g * VEC);
#pragma unroll
    for (int k = 0; k < VEC; ++k)
      if (c == static_cast<uint32_t>(k)) tele[k] += p.seeds.tele[e];
  }
  const uint32_t dg = p.deg[v];
  const size_t base = static_cast<size_t>(v) * KT + lane_g * VEC;
  float old[VEC];
  if (lane_flags & kLaneLive) {  // only a live column's delta needs its old value
    ldvec_cs<VEC>(p.X + base, old);
  } else {
#pragma unroll
    for (int c = 0; c < VEC; ++c) old[c] = 0.f;
  }
  // old[c] is dead once its delta is taken: it holds the value to store
#pragma unroll
  for (int c = 0; c < VEC; ++c) {
    const float r = fmaf(p.d, y[c], tele[c]);
    if (st[c] == COL_LIVE) {
      float xv, dlt;
      if (dg > 0) {
        const float fd = static_cast<float>(dg);
        xv = r / fd;
        dlt = fabsf(xv - old[c]) * fd;
      } else {
        xv = r;
        dlt = fabsf(xv - old[c]);
      }
      old[c] = xv;
      dl[c] += dlt;
    } else {
      old[c] = r;
    }
  }
  if constexpr (VEC == 4) {
    if (lane_flags & kLaneAll) {  // every column of the lane is written: one 16-byte store
      __stcs(reinterpret_cast<float4*>(p.Xn + base), make_float4(old[0], old[1], old[2], old[3]));
      return;
    }
  }
#pragma unroll
  for (int c = 0; c < VEC; ++c)
    if (st[c] == COL_LIVE || st[c] == COL_FINAL) __stcs(p.Xn + base + c, old[c]);
}

// Merge-path search in shared memory: first coordinate of diagonal `diag`.
__device__ __forceinline__ void merge_search(const uint32_t* s_rowend, int nrows, int nnz, int diag,
                                             int& row, int& edge) {
  int lo = max(diag - nnz, 0), hi = min(diag, nrows);
  while (lo < hi) {
    const int piv = (lo + hi) >> 1;
    if (static_cast<int>(s_rowend[piv]) <= diag - piv - 1)
      lo = piv + 1;
    else
      hi = piv;
  }
  row = lo;
  edge = diag - lo;
}

template <int GL, int VEC>
__global__ void __launch_bounds__(256, kBatchMinBlocks) k_batch_pull(batch_pass p0) {
  constexpr int KT = GL * VEC, NG = 256 / GL, TILE = batch_tile_items(KT), IPG = TILE / NG;
  const batch_pass p = batch_tile_view<KT>(p0);
  // The row ends and staged source ids are dead once the gathers are done, so
  // the per-lane delta partials reuse their space; the head row's sums wait in
  // shared memory instead of registers.  Less shared memory leaves more L1 to
  // the gathers and the freed registers end a spill (K = 64 batch at RMAT s22:
  // 100.9 -> 96.7 ms).
  constexpr int kRaw = (2 * TILE * 4 > NG * KT * 8) ? 2 * TILE * 4 : NG * KT * 8;
  __shared__ __align__(16) unsigned char s_raw[kRaw];
  uint32_t* s_rowend = reinterpret_cast<uint32_t*>(s_raw);
  uint32_t* s_src = s_rowend + TILE;
  double* s_dl = reinterpret_cast<double*>(s_raw);
  __shared__ uint32_t s_ckey[NG];
  __shared__ float s_cval[NG * KT];
  __shared__ float s_hacc[NG * KT];
  // One L2 policy for every row gather, by address: normal priority for the
  // hot rows [0, hot_rows) of this column tile, evict-first past them (range
  // sizes are 32-bit: rows past 4 GB of a tile keep the default priority).
  uint64_t pol;
  {
    const uint64_t tile_bytes = static_cast<uint64_t>(p.V) * KT * 4;
    const uint32_t total = static_cast<uint32_t>(tile_bytes < 0xFFFFFF00ull ? tile_bytes : 0xFFFFFF00ull);
    const uint64_t hot_bytes = static_cast<uint64_t>(p.hot_rows) * KT * 4;
    const uint32_t primary = static_cast<uint32_t>(hot_bytes < total ? hot_bytes : total);
    asm("createpolicy.range.global.L2::evict_normal.L2::evict_first.b64 %0, [%1], %2, %3;"
        : "=l"(pol)
        : "l"(p.X), "r"(primary), "r"(total));
  }

  const int lane_g = threadIdx.x % GL, g = threadIdx.x / GL;
  uint8_t st[VEC];
  int mine = 0;
#pragma unroll
  for (int c = 0; c < VEC; ++c) {
    st[c] = p.state[lane_g * VEC + c];
    mine |= (st[c] == COL_LIVE || st[c] == COL_FINAL);
  }
  if (!__syncthreads_or(mine)) return;  // every column of this tile is idle
  const uint32_t lflags = lane_flags_of<VEC>(st);

  const uint32_t t = blockIdx.x;
  const uint32_t i0 = p.trow[t], i1 = p.trow[t + 1];
  const uint64_t j0 = p.tedge[t], j1 = p.tedge[t + 1];
  const int nrows = static_cast<int>(i1 - i0), nnz = static_cast<int>(j1 - j0);
  const bool spans = p.off[i0] < j0;
  for (int r = threadIdx.x; r < nrows; r += 256)
    s_rowend[r] = static_cast<uint32_t>(p.off[i0 + r + 1] - j0);
  for (int e = threadIdx.x; e < nnz; e += 256) s_src[e] = __ldcs(p.adj + j0 + e);
  __syncthreads();

  const int total = nrows + nnz;
  const int d0 = min(g * IPG, total), d1 = min(d0 + IPG, total);
  int ra, ja, rb, jb;
  merge_search(s_rowend, nrows, nnz, d0, ra, ja);
  merge_search(s_rowend, nrows, nnz, d1, rb, jb);
  const int head = ra;
  bool head_done = false;
  float acc[VEC];
  float dl[VEC];  // this lane's rows only; the CTA sums them in double
#pragma unroll
  for (int c = 0; c < VEC; ++c) {
    acc[c] = 0.f;
    dl[c] = 0.f;
  }
  const float* xl = p.X + lane_g * VEC;
  int jj = ja;
  for (int r = ra; r <= rb; ++r) {
    const int e_end = (r < rb) ? static_cast<int>(s_rowend[r]) : jb;
    // The update's old row is prefetched into L2 while the row's gathers run,
    // so batch_finalize does not wait a DRAM latency for it.  With the flags
    // taken once and the 16-byte store of the update, on one B200 (queries/s,
    // RMAT s22 K = 64 / 256 / 1024, RMAT s24 K = 64 / 128): 616 / 703 / 718,
    // 150.6 / 161.5 -> 634 / 731 / 742, 153.6 / 164.6.
    if ((lflags & kLaneLive) && r < rb && r != head)
      asm volatile("prefetch.global.L2 [%0];" ::"l"(p.X + static_cast<size_t>(i0 + r) * KT + lane_g * VEC));
    // rounds of kBatchInflight row gathers in flight per lane; the last
    // round of a row is predicated instead of a serial tail, so a row costs
    // one gather latency per kBatchInflight in-edges.  A lane whose columns
    // are all finished or free loads nothing (its part of the row is never
    // fetched), so a tile costs less as its columns converge.
    for (; jj < e_end; jj += kBatchInflight) {
      const int n = mine ? e_end - jj : 0;
      float a[kBatchInflight][VEC];
#pragma unroll
      for (int u = 0; u < kBatchInflight; ++u) {
        if (u < n) {
          const uint32_t src = s_src[jj + u];
          static_assert(VEC == 4, "row gathers are 16-byte loads");
          ld4_pol(xl + static_cast<size_t>(src) * KT, a[u], pol);
        } else {
#pragma unroll
          for (int c = 0; c < VEC; ++c) a[u][c] = 0.f;
        }
      }
      static_assert(kBatchInflight == 4, "the row sum below adds four gathers");
#pragma unroll
      for (int c = 0; c < VEC; ++c) acc[c] += (a[0][c] + a[1][c]) + (a[2][c] + a[3][c]);
    }
    jj = e_end;  // the last round may step past the row's end
    if (r < rb) {
      if (r == head) {
        head_done = true;
#pragma unroll
        for (int c = 0; c < VEC; ++c) s_hacc[g * KT + lane_g * VEC + c] = acc[c];
      } else {
        batch_finalize<GL, VEC>(p, i0 + r, acc, st, lane_g, lflags, dl);
      }
#pragma unroll
      for (int c = 0; c < VEC; ++c) acc[c] = 0.f;
    }
  }
  if (lane_g == 0) s_ckey[g] = static_cast<uint32_t>(rb);
#pragma unroll
  for (int c = 0; c < VEC; ++c) s_cval[g * KT + lane_g * VEC + c] = acc[c];
  __syncthreads();

  if (head_done) {
    float y[VEC];
#pragma unroll
    for (int c = 0; c < VEC; ++c) y[c] = s_hacc[g * KT + lane_g * VEC + c];
    for (int g2 = g - 1; g2 >= 0 && s_ckey[g2] == static_cast<uint32_t>(head); --g2) {
#pragma unroll
      for (int c = 0; c < VEC; ++c) y[c] += s_cval[g2 * KT + lane_g * VEC + c];
    }
    if (head == 0 && spans) {
#pragma unroll
      for (int c = 0; c < VEC; ++c) p.thead[static_cast<size_t>(t) * KT + lane_g * VEC + c] = y[c];
    } else {
      batch_finalize<GL, VEC>(p, i0 + head, y, st, lane_g, lflags, dl);
    }
  }
  if (g == NG - 1) {
    float y[VEC];
#pragma unroll
    for (int c = 0; c < VEC; ++c) y[c] = 0.f;
    for (int g2 = NG - 1; g2 >= 0 && s_ckey[g2] == static_cast<uint32_t>(nrows); --g2) {
#pragma unroll
      for (int c = 0; c < VEC; ++c) y[c] += s_cval[g2 * KT + lane_g * VEC + c];
    }
#pragma unroll
    for (int c = 0; c < VEC; ++c) p.tcarry[static_cast<size_t>(t) * KT + lane_g * VEC + c] = y[c];
  }
#pragma unroll
  for (int c = 0; c < VEC; ++c) s_dl[g * KT + lane_g * VEC + c] = dl[c];
  __syncthreads();
  for (int c = threadIdx.x; c < KT; c += 256) {
    double s = 0.0;
    for (int g2 = 0; g2 < NG; ++g2) s += s_dl[g2 * KT + c];
    p.partials[static_cast<size_t>(t) * KT + c] = s;
  }
}

// Rows split across CTAs: one group of GL lanes per tile.
template <int GL, int VEC>
__global__ void __launch_bounds__(256) k_batch_fixup(batch_pass p0) {
  constexpr int KT = GL * VEC, NG = 256 / GL;
  const batch_pass p = batch_tile_view<KT>(p0);
  __shared__ double s_dl[NG * KT];
  const int lane_g = threadIdx.x % GL, g = threadIdx.x / GL;
  uint8_t st[VEC];
  int mine = 0;
#pragma unroll
  for (int c = 0; c < VEC; ++c) {
    st[c] = p.state[lane_g * VEC + c];
    mine |= (st[c] == COL_LIVE || st[c] == COL_FINAL);
  }
  if (!__syncthreads_or(mine)) return;
  const uint32_t lflags = lane_flags_of<VEC>(st);
  float dl[VEC];
#pragma unroll
  for (int c = 0; c < VEC; ++c) dl[c] = 0.f;
  const uint32_t t = blockIdx.x * NG + g;
  if (t >= 1 && t < p.T) {
    const uint32_t i0 = p.trow[t];
    if (p.trow[t + 1] > i0 && p.off[i0] < p.tedge[t]) {
      uint32_t tf = t - 1;
      while (tf > 0 && p.trow[tf] == i0) --tf;
      float y[VEC];
#pragma unroll
      for (int c = 0; c < VEC; ++c) y[c] = 0.f;
      for (uint32_t u = tf; u < t; ++u) {
#pragma unroll
        for (int c = 0; c < VEC; ++c) y[c] += p.tcarry[static_cast<size_t>(u) * KT + lane_g * VEC + c];
      }
#pragma unroll
      for (int c = 0; c < VEC; ++c) y[c] += p.thead[static_cast<size_t>(t) * KT + lane_g * VEC + c];
      batch_finalize<GL, VEC>(p, i0, y, st, lane_g, lflags, dl);
    }
  }
#pragma unroll
  for (int c = 0; c < VEC; ++c) s_dl[g * KT + lane_g * VEC + c] = dl[c];
  __syncthreads();
  for (int c = threadIdx.x; c < KT; c += 256) {
    double s = 0.0;
    for (int g2 = 0; g2 < NG; ++g2) s += s_dl[g2 * KT + c];
    p.partials[(static_cast<size_t>(p.T) + blockIdx.x) * KT + c] = s;
  }
}

// delta[q] = sum over rows of the column tile's partials[row][c] in row order;
// grid (kt, column tiles), q = blockIdx.y * kt + blockIdx.x.  Also clears the
// live-column count that k_batch_states (the next launch) accumulates.
static __global__ void __launch_bounds__(256) k_batch_delta(const double* __restrict__ partials,
                                                            uint32_t rows, uint32_t kt,
                                                            const uint8_t* __restrict__ state,
                                                            double* __restrict__ delta,
                                                            uint32_t* __restrict__ live_count) {
  __shared__ double s_red[32];
  if (blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0) *live_count = 0u;
  const uint32_t c = blockIdx.x;
  const uint32_t q = blockIdx.y * kt + c;
  if (state[q] != COL_LIVE) return;  // block-uniform
  const double* pt = partials + static_cast<size_t>(blockIdx.y) * rows * kt;
  const uint32_t per = (rows + 255) / 256;
  const uint32_t b = threadIdx.x * per, e = min(rows, b + per);
  double acc = 0.0;
  for (uint32_t i = b; i < e; ++i) acc += pt[static_cast<size_t>(i) * kt + c];
  acc = block_sum<256>(acc, s_red);
  if (threadIdx.x == 0) delta[q] = acc;
}

// Column state machine after one iteration (see the header comment).
static __global__ void k_batch_states(uint32_t K, uint8_t* state, uint32_t* iters, uint8_t* parity,
                               const double* __restrict__ delta, uint32_t max_iterations,
                               double eps, int written_parity, uint32_t* live_count,
                               uint32_t* retired, uint32_t* retired_count) {
  for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < K; q += gridDim.x * blockDim.x) {
    const uint8_t s = state[q];
    if (s == COL_LIVE) {
      const uint32_t it = ++iters[q];
      if (it >= max_iterations - 1 || (eps > 0.0 && delta[q] < eps)) state[q] = COL_FINAL;
      atomicAdd(live_count, 1u);
    } else if (s == COL_FINAL) {
      ++iters[q];
      state[q] = COL_DONE;
      parity[q] = static_cast<uint8_t>(written_parity);
      const uint32_t slot = atomicAdd(retired_count, 1u);
      retired[slot] = q;
    }
  }
}

}  // namespace plato_b200
