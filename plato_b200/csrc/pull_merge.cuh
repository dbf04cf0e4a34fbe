// Pull-mode gather over the CSC with the rank update fused in the epilogue.
//
// This is the device form of the reference's pull path for the rank
// algorithms: aggregate_message over the DCSC (plato/graph/message_passing.hpp:88-144)
// with the signal "rank_sum = sum of curt_rank[src] over in-edges"
// (pagerank.hpp:104-116) followed by the per-vertex update
// (pagerank.hpp:118-135):  r = teleport(v) + d * y;  x = r / deg  (deg > 0),
// delta += |x - x_old| * deg  (|x - x_old| when deg == 0); the last epoch keeps r.
//
// Load balance: merge-path tiling (Merrill & Garland, SC'16).  Tile t owns
// `items` consecutive merge items of the two sorted lists (row ends, edge
// indices), so every CTA handles the same amount of work whatever the degree
// distribution.  A tile stages its row ends and gathered x[src] in shared
// memory, each thread merges IPT items, a block-wide segmented scan joins row
// pieces split across threads, and rows split across tiles are joined by a
// second small kernel that sums the per-tile pieces in tile order.  All sums
// have a fixed order, so results are bit-for-bit reproducible.
#pragma once

#include "common.cuh"

namespace plato_b200 {

// Teleport terms of the three rank algorithms.
struct teleport_uniform {  // pagerank.hpp:120,127 (normalised: (1-d)/V)
  float base;
  __device__ __forceinline__ float operator()(uint32_t) const { return base; }
};
struct teleport_single {  // personalized_pagerank.hpp:105,113: (v == src ? 1-d : 0)
  uint32_t src;
  float val;
  __device__ __forceinline__ float operator()(uint32_t v) const { return v == src ? val : 0.f; }
};

struct teleport_seeds {  // trustrank.hpp:226-245: (seed ? (1-d)/|S| : 0)
  const uint32_t* bits;  // seed bitmap, 32-bit words
  float val;
  __device__ __forceinline__ float operator()(uint32_t v) const {
    return ((bits[v >> 5] >> (v & 31)) & 1u) ? val : 0.f;
  }
};

template <class Teleport>
struct rank_update {
  const float* __restrict__ x;    // current state
  float* __restrict__ xn;         // next state
  const uint32_t* __restrict__ deg;
  Teleport tele;
  float d;
  int final_epoch;
  // When set, the epoch kind is read from the device: 0 normal, 1 final
  // (store r), 2 done (the kernels return at once); see k_epoch_control.
  const int* mode = nullptr;

  __device__ __forceinline__ bool skip() const { return mode && *mode == 2; }

  __device__ __forceinline__ bool storing_rank() const { return mode ? (*mode == 1) : (final_epoch != 0); }

  // The inputs of apply() that do not depend on the gathered sum; a kernel
  // may load them before its gathers so that their latency overlaps.
  struct operands {
    uint32_t dg;
    float xo;
  };
  __device__ __forceinline__ operands load(uint32_t v) const {
    if (storing_rank()) return {0u, 0.f};
    return {__ldcs(deg + v), __ldcs(x + v)};
  }

  __device__ __forceinline__ double apply(uint32_t v, float y) const { return apply(v, y, load(v)); }

  __device__ __forceinline__ double apply(uint32_t v, float y, operands o) const {
    const float r = fmaf(d, y, tele(v));
    if (storing_rank()) {
      xn[v] = r;
      return 0.0;
    }
    const uint32_t dg = o.dg;
    const float xo = o.xo;
    float xv, dl;
    if (dg > 0) {
      const float fd = static_cast<float>(dg);
      xv = r / fd;
      dl = fabsf(xv - xo) * fd;
    } else {
      xv = r;
      dl = fabsf(xv - xo);
    }
    xn[v] = xv;
    return static_cast<double>(dl);
  }
};

template <int NT, int IPT>
struct pull_merge_cfg {
  static constexpr int kTile = NT * IPT;
  // rowend + gathered values + row results (uint32/float each) + scan arrays
  static constexpr size_t kSmem = 3ull * kTile * 4 + 2ull * NT * 4 + 2ull * (NT / 32) * 4 + 32 * 8;
};

// Block-wide inclusive segmented scan over (key, val) with non-decreasing keys:
// (ka, va) . (kb, vb) = (kb, ka == kb ? va + vb : vb).
template <int NT>
__device__ __forceinline__ void seg_scan(uint32_t& key, float& val, uint32_t* s_wkey,
                                         float* s_wval) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t k2 = __shfl_up_sync(0xffffffffu, key, o);
    const float v2 = __shfl_up_sync(0xffffffffu, val, o);
    if (lane >= o && k2 == key) val = v2 + val;
  }
  if (lane == 31) {
    s_wkey[wid] = key;
    s_wval[wid] = val;
  }
  __syncthreads();
  if (wid == 0) {
    constexpr int NW = NT / 32;
    uint32_t k = lane < NW ? s_wkey[lane] : 0xFFFFFFFFu;
    float v = lane < NW ? s_wval[lane] : 0.f;
#pragma unroll
    for (int o = 1; o < NW; o <<= 1) {
      const uint32_t k2 = __shfl_up_sync(0xffffffffu, k, o);
      const float v2 = __shfl_up_sync(0xffffffffu, v, o);
      if (lane >= o && k2 == k) v = v2 + v;
    }
    if (lane < NW) {
      s_wkey[lane] = k;
      s_wval[lane] = v;
    }
  }
  __syncthreads();
  if (wid > 0 && s_wkey[wid - 1] == key) val = s_wval[wid - 1] + val;
}

template <int NT, int IPT, class Update>
__global__ void __launch_bounds__(NT) k_pull_merge(
    const uint32_t* __restrict__ trow, const uint64_t* __restrict__ tedge,
    const uint64_t* __restrict__ off, const uint32_t* __restrict__ adj,
    const float* __restrict__ x, Update upd, float* __restrict__ tile_carry,
    float* __restrict__ tile_head, double* __restrict__ partials) {
  constexpr int TILE = NT * IPT;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  uint32_t* s_rowend = reinterpret_cast<uint32_t*>(smem_raw);
  float* s_val = reinterpret_cast<float*>(s_rowend + TILE);
  float* s_y = s_val + TILE;
  uint32_t* s_key = reinterpret_cast<uint32_t*>(s_y + TILE);
  float* s_inc = reinterpret_cast<float*>(s_key + NT);
  uint32_t* s_wkey = reinterpret_cast<uint32_t*>(s_inc + NT);
  float* s_wval = reinterpret_cast<float*>(s_wkey + NT / 32);
  double* s_red = reinterpret_cast<double*>(
      (reinterpret_cast<uintptr_t>(s_wval + NT / 32) + 7) & ~uintptr_t(7));

  const uint32_t t = blockIdx.x;
  const uint32_t i0 = trow[t], i1 = trow[t + 1];
  const uint64_t j0 = tedge[t], j1 = tedge[t + 1];
  const int nrows = static_cast<int>(i1 - i0);
  const int nnz = static_cast<int>(j1 - j0);
  const bool spans = (nrows > 0 || nnz > 0) && off[i0] < j0;

  for (int r = threadIdx.x; r < nrows; r += NT)
    s_rowend[r] = static_cast<uint32_t>(off[i0 + r + 1] - j0);
  {
    uint32_t srcs[IPT];
#pragma unroll
    for (int k = 0; k < IPT; ++k) {
      const int e = threadIdx.x + k * NT;
      srcs[k] = (e < nnz) ? __ldg(adj + j0 + e) : 0u;
    }
#pragma unroll
    for (int k = 0; k < IPT; ++k) {
      const int e = threadIdx.x + k * NT;
      if (e < nnz) s_val[e] = __ldg(x + srcs[k]);
    }
  }
  __syncthreads();

  const int total = nrows + nnz;
  const int diag = min(static_cast<int>(threadIdx.x) * IPT, total);
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
  float sum = 0.f, head_sum = 0.f;
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

  uint32_t key = static_cast<uint32_t>(ii);
  float val = sum;
  seg_scan<NT>(key, val, s_wkey, s_wval);
  s_key[threadIdx.x] = key;
  s_inc[threadIdx.x] = val;
  __syncthreads();
  if (head_done) {
    float cin = 0.f;
    if (threadIdx.x > 0 && s_key[threadIdx.x - 1] == static_cast<uint32_t>(head))
      cin = s_inc[threadIdx.x - 1];
    const float y = cin + head_sum;
    if (head == 0 && spans)
      tile_head[t] = y;
    else
      s_y[head] = y;
  }
  if (threadIdx.x == NT - 1) tile_carry[t] = (key == static_cast<uint32_t>(nrows)) ? val : 0.f;
  __syncthreads();

  double dl = 0.0;
  for (int r = threadIdx.x; r < nrows; r += NT) {
    if (r == 0 && spans) continue;
    dl += upd.apply(i0 + r, s_y[r]);
  }
  dl = block_sum<NT>(dl, s_red);
  if (threadIdx.x == 0) partials[t] = dl;
}

// Rows that began in an earlier tile and end in tile t: y = sum of the
// carries of the tiles the row passed through (in tile order) + tile t's head.
template <class Update>
__global__ void __launch_bounds__(256) k_pull_fixup(
    const uint32_t* __restrict__ trow, const uint64_t* __restrict__ tedge,
    const uint64_t* __restrict__ off, uint32_t T, Update upd,
    const float* __restrict__ tile_carry, const float* __restrict__ tile_head,
    double* __restrict__ partials) {
  __shared__ double s_red[32];
  double dl = 0.0;
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 1 && t < T) {
    const uint32_t i0 = trow[t];
    if (trow[t + 1] > i0 && off[i0] < tedge[t]) {
      uint32_t tf = t - 1;
      while (tf > 0 && trow[tf] == i0) --tf;
      float y = 0.f;
      for (uint32_t u = tf; u < t; ++u) y += tile_carry[u];
      y += tile_head[t];
      dl = upd.apply(i0, y);
    }
  }
  dl = block_sum<256>(dl, s_red);
  if (threadIdx.x == 0) partials[blockIdx.x] = dl;
}

// delta = sum of partials in index order (one block, fixed tree) -> out[0].
static __global__ void __launch_bounds__(1024) k_sum_partials(const double* __restrict__ p, uint32_t n,
                                                       double* __restrict__ out) {
  __shared__ double s_red[32];
  const uint32_t per = (n + 1023) / 1024;
  const uint32_t b = threadIdx.x * per, e = min(n, b + per);
  double s = 0.0;
  for (uint32_t i = b; i < e; ++i) s += p[i];
  s = block_sum<1024>(s, s_red);
  if (threadIdx.x == 0) out[0] = s;
}

}  // namespace plato_b200
