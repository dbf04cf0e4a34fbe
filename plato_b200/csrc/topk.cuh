// Exact on-device top-k of rank columns (radix select on 64-bit keys).
//
// key(v) = (bits(rank) << 32) | (0xFFFFFFFF - caller_id(v)): ranks are >= 0,
// so the float bits order like the values, and equal ranks order by smaller
// caller id first; every key is unique, so the k largest keys are exactly the
// top-k with a deterministic tie-break.  Per column, 8-bit digits are fixed
// from the top until the keys at or above the current prefix number at most
// kCandCap; those candidates are collected and sorted in shared memory.
// Columns are read in place from the tile-major state (see batch.cuh).
#pragma once

#include "common.cuh"

namespace plato_b200 {

constexpr uint32_t kCandCap = 2048;
constexpr uint32_t kTopkMax = 1024;

struct topk_col {
  unsigned long long prefix;  // fixed high bits (low bits zero)
  uint32_t known;             // number of fixed bits
  uint32_t remaining;         // keys still needed inside the current bin
  uint32_t done;              // 1 = candidate bound found
  uint32_t count;             // candidates collected
};

struct topk_job {
  const float* buf[2];       // the two state buffers
  const uint8_t* parity;     // [K] buffer holding each column's result
  const uint32_t* cols;      // [n] global columns to process
  uint32_t n;
  uint32_t V;
  uint32_t kt;               // columns per tile (state layout)
  const uint32_t* to_ext;    // internal -> caller id (nullptr = identity)
  topk_col* st;              // [n]
  uint32_t* hist;            // [n][256], zero on entry
  unsigned long long* cand;  // [n][kCandCap]
};

__device__ __forceinline__ unsigned long long topk_key(const topk_job& j, uint32_t q, uint32_t v) {
  const uint32_t tile = q / j.kt, c = q % j.kt;
  const float val = j.buf[j.parity[q]][(static_cast<size_t>(tile) * j.V + v) * j.kt + c];
  const uint32_t ext = j.to_ext ? j.to_ext[v] : v;
  return (static_cast<unsigned long long>(__float_as_uint(val)) << 32) |
         static_cast<unsigned long long>(0xFFFFFFFFu - ext);
}

static __global__ void k_topk_init(topk_job j, uint32_t k) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < j.n; i += gridDim.x * blockDim.x) {
    topk_col s;
    s.prefix = 0ull;
    s.known = 0;
    s.remaining = k;
    s.done = (j.V <= kCandCap) ? 1u : 0u;  // everything fits: bound 0
    s.count = 0;
    j.st[i] = s;
  }
}

// Histogram of the next digit for job columns [c0, c0 + 32), one lane per column.
static __global__ void __launch_bounds__(256) k_topk_hist(topk_job j, uint32_t c0) {
  __shared__ uint32_t h[32][256];
  for (int i = threadIdx.x; i < 32 * 256; i += 256) (&h[0][0])[i] = 0u;
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const uint32_t ci = c0 + lane;
  const bool active = ci < j.n && !j.st[ci].done;
  unsigned long long pre = 0;
  uint32_t known = 0, q = 0;
  if (active) {
    pre = j.st[ci].prefix;
    known = j.st[ci].known;
    q = j.cols[ci];
  }
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  if (active) {
    for (uint32_t v = warp; v < j.V; v += nwarps) {
      const unsigned long long key = topk_key(j, q, v);
      if (known == 0 || (key >> (64 - known)) == (pre >> (64 - known)))
        atomicAdd(&h[lane][(key >> (56 - known)) & 0xFFu], 1u);
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < 32 * 256; i += 256) {
    const uint32_t col = static_cast<uint32_t>(i >> 8);
    const uint32_t cnt = (&h[0][0])[i];
    if (cnt && c0 + col < j.n) atomicAdd(&j.hist[(c0 + col) * 256 + (i & 255)], cnt);
  }
}

// Fix the next digit of each unfinished column (one thread per column);
// counts the columns that still need another pass into *undone.
static __global__ void k_topk_pick(topk_job j, uint32_t k, uint32_t* undone) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < j.n; i += gridDim.x * blockDim.x) {
    topk_col s = j.st[i];
    if (s.done) continue;
    uint32_t* h = j.hist + static_cast<size_t>(i) * 256;
    uint32_t cum = 0, digit = 0, eq = 0;
    for (int dgt = 255; dgt >= 0; --dgt) {
      const uint32_t c = h[dgt];
      if (cum + c >= s.remaining) {
        digit = static_cast<uint32_t>(dgt);
        eq = c;
        break;
      }
      cum += c;
    }
    for (int dgt = 0; dgt < 256; ++dgt) h[dgt] = 0u;
    s.prefix |= static_cast<unsigned long long>(digit) << (56 - s.known);
    s.known += 8;
    s.remaining -= cum;
    const uint32_t ge = (k - s.remaining) + eq;  // keys >= prefix
    if (ge <= kCandCap || s.known >= 64)
      s.done = 1;
    else
      atomicAdd(undone, 1u);
    j.st[i] = s;
  }
}

// Collect every key >= the column's bound (at most kCandCap of them).
static __global__ void __launch_bounds__(256) k_topk_collect(topk_job j, uint32_t c0) {
  const int lane = threadIdx.x & 31;
  const uint32_t ci = c0 + lane;
  if (ci >= j.n) return;  // lanes of a warp only diverge here, no warp collectives below
  const unsigned long long bound = j.st[ci].known ? j.st[ci].prefix : 0ull;
  const uint32_t q = j.cols[ci];
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t v = warp; v < j.V; v += nwarps) {
    const unsigned long long key = topk_key(j, q, v);
    if (key >= bound) {
      const uint32_t slot = atomicAdd(&j.st[ci].count, 1u);
      if (slot < kCandCap) j.cand[static_cast<size_t>(ci) * kCandCap + slot] = key;
    }
  }
}

// Sort each column's candidates (descending) and emit the first k as
// (caller id, rank); slots beyond V hold id 0xFFFFFFFF and rank 0.
static __global__ void __launch_bounds__(1024) k_topk_sort(topk_job j, uint32_t k, uint32_t* out_ids,
                                                           float* out_vals) {
  __shared__ unsigned long long s[kCandCap];
  const uint32_t ci = blockIdx.x;
  const uint32_t n = min(j.st[ci].count, kCandCap);
  for (uint32_t i = threadIdx.x; i < kCandCap; i += blockDim.x)
    s[i] = (i < n) ? j.cand[static_cast<size_t>(ci) * kCandCap + i] : 0ull;
  __syncthreads();
  // bitonic sort, descending
  for (uint32_t size = 2; size <= kCandCap; size <<= 1) {
    for (uint32_t stride = size >> 1; stride > 0; stride >>= 1) {
      for (uint32_t i = threadIdx.x; i < kCandCap; i += blockDim.x) {
        const uint32_t pr = i ^ stride;
        if (pr > i) {
          const bool desc = (i & size) == 0;
          const unsigned long long a = s[i], b = s[pr];
          if (desc ? (a < b) : (a > b)) {
            s[i] = b;
            s[pr] = a;
          }
        }
      }
      __syncthreads();
    }
  }
  for (uint32_t r = threadIdx.x; r < k; r += blockDim.x) {
    uint32_t id = 0xFFFFFFFFu;
    float val = 0.f;
    if (r < n) {
      const unsigned long long key = s[r];
      id = 0xFFFFFFFFu - static_cast<uint32_t>(key & 0xFFFFFFFFull);
      val = __uint_as_float(static_cast<uint32_t>(key >> 32));
    }
    out_ids[static_cast<size_t>(ci) * k + r] = id;
    out_vals[static_cast<size_t>(ci) * k + r] = val;
  }
}

}  // namespace plato_b200
