// HyperLogLog register propagation: algo::hyperanf and nstepdegrees_t.
//
// Reference behaviour followed:
//   plato/util/hash.hpp:33-88          murmurhash3 of the 4-byte vertex id
//   plato/util/hyperloglog.hpp:32-142  hyperloglog_t<P>: 2^P one-byte
//       registers; add (index = top P hash bits, rank = 1 + leading zeros of
//       the rest, capped at 33 - P), merge = register-wise max, estimate
//       (raw HLL with the small-range linear counting and large-range
//       corrections)
//   plato/algo/hyperanf/hyperanf.hpp:83-195  every vertex starts with its own
//       id; each epoch merges the in-neighbours' registers as they stood
//       before the epoch; ANF = sum of the estimates; stop when the ANF grows
//       by less than DBL_EPSILON; average distance from the ANF series
//   plato/algo/nstepdegrees/nstepdegrees.hpp:160-402  per phase (in, then
//       out): covered = targets, spread the coverage `step` hops against the
//       counting direction, propagate registers `step` epochs over covered
//       vertices only, degree = (uint32)estimate - 1 per target
//   plato/engine/dualmode.hpp:245-297  push iff the forward out-degrees of the
//       actives over the stored edges < push_threshold.  As in the reference,
//       the push slots scatter over the forward out-edges even while the
//       engine is reversed (nstepdegrees.hpp:217-229, 316-327), and reversed
//       pull epochs walk the out-edges (dualmode.hpp:302-308).
//
// Layout in HBM: registers are rows of m = 2^P bytes, row v at v * m
// (internal vertex order), in two buffers (cur, nxt).  An epoch reads cur and
// writes nxt only for rows that change now or changed in the previous epoch
// (the rows whose nxt copy lags); every other row is already equal in both
// buffers, so the buffers swap without a copy.  Estimates are kept per
// vertex (double) and recomputed only for changed rows; the register sum is
// accumulated exactly as fixed point (sum of 2^(32 - r)), so each estimate
// equals the reference's bit for bit up to the final log of the linear
// counting branch.
//
// Gather kernels: rows are destinations; a team of T lanes owns one row and
// each lane holds VEC 16-byte register words of a slice of T*VEC*16 bytes,
// merging source rows with per-byte max (__vmaxu4), several source rows in
// flight.  Rows with many sources go to a block-per-row kernel.  Sources are
// filtered by a bitmap (the previous epoch's changed rows): merging only the
// rows that changed gives the same registers as merging every in-neighbour
// whenever push and pull walk the same direction (any unchanged row was
// merged in an earlier epoch), and it is exactly the push slot's rule.
// Push epochs (few changed rows) scatter those rows over their out-edges
// instead (k_hll_scatter), so their cost follows the actives' edges rather
// than every row's sources.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <exception>
#include <mutex>
#include <utility>
#include <vector>

#include <cub/device/device_select.cuh>
#include <thrust/iterator/counting_iterator.h>

#include "graph.cuh"
#include "profile.cuh"

namespace plato_b200 {
namespace {

constexpr uint32_t kHllSeed = 0x5f61767au;  // hyperloglog.hpp:64
constexpr int kHllThreads = 256;
constexpr uint32_t kSumBlocks = 148u * 4u;
constexpr uint32_t kNoVertex = 0xFFFFFFFFu;
// Rows with more sources than hub_deg = clamp(kHubBytes / m, kHubMinDeg,
// kHubMaxDeg) go to the block-per-row kernel (measured on RMAT s22: 2048 at
// 64-byte rows, 512 from 256-byte rows up).
constexpr uint32_t kHubBytes = 131072u;
constexpr uint32_t kHubMinDeg = 512u;
constexpr uint32_t kHubMaxDeg = 2048u;

__device__ __forceinline__ uint32_t rotl32(uint32_t x, int r) { return (x << r) | (x >> (32 - r)); }

// MurmurHash3_x86_32 (Austin Appleby's published algorithm) of one 4-byte
// little-endian key, as hash.hpp:33-88 computes it for len = 4.
__device__ __forceinline__ uint32_t murmur3_u32(uint32_t k) {
  k *= 0xcc9e2d51u;
  k = rotl32(k, 15);
  k *= 0x1b873593u;
  uint32_t h = kHllSeed ^ k;
  h = rotl32(h, 13);
  h = h * 5u + 0xe6546b64u;
  h ^= 4u;
  h ^= h >> 16;
  h *= 0x85ebca6bu;
  h ^= h >> 13;
  h *= 0xc2b2ae35u;
  h ^= h >> 16;
  return h;
}

// alpha * m^2 of hyperloglog_t<P>::estimate (hyperloglog.hpp:77-93).
double hll_alpha_mm(uint32_t P) {
  const double m = static_cast<double>(1u << P);
  double a;
  switch (P) {
    case 4: a = 0.673; break;
    case 5: a = 0.697; break;
    case 6: a = 0.709; break;
    default: a = 0.7213 / (1.0 + 1.079 / m); break;
  }
  return a * (m * m);
}

// hyperloglog_t<P>::estimate (hyperloglog.hpp:94-112) from the exact
// register sum sumfx = sum of 2^(32 - r) and the count of zero registers.
__device__ __forceinline__ double hll_estimate(uint32_t P, double alpha_mm,
                                               unsigned long long sumfx, uint32_t zeros) {
  const double m = static_cast<double>(1u << P);
  const double sum = static_cast<double>(sumfx) * 0x1p-32;  // exact (< 2^53)
  double est = alpha_mm / sum;
  if (est <= 5.0 / 2.0 * m) {
    if (zeros) est = m * log(m / static_cast<double>(zeros));
  } else if (est > (1.0 / 30.0) * 4294967296.0) {
    est = -4294967296.0 * log(1.0 - (est / 4294967296.0));
  }
  return est;
}

__device__ __forceinline__ bool test_bit(const uint32_t* b, uint32_t v) {
  return (__ldg(b + (v >> 5)) >> (v & 31)) & 1u;
}

// Per-byte max of two words whose bytes are below 128 (registers never
// exceed 33 - P <= 29): bytes where a >= b get a 0x80 flag from a
// borrow-free subtraction, widened to a byte mask that selects a or b.
// (Measured on B200 against __vmaxu4: equal or faster at every width.)
__device__ __forceinline__ uint32_t bmax(uint32_t a, uint32_t b) {
  const uint32_t d = ((a | 0x80808080u) - b) & 0x80808080u;
  const uint32_t m = (d - (d >> 7)) | d;
  return (a & m) | (b & ~m);
}
__device__ __forceinline__ uint4 vmax4(uint4 a, uint4 b) {
  return make_uint4(bmax(a.x, b.x), bmax(a.y, b.y), bmax(a.z, b.z), bmax(a.w, b.w));
}
// Even and odd bytes of a word widened to 16-bit lanes, and back.
__device__ __forceinline__ uint32_t even_bytes(uint32_t w) { return __byte_perm(w, 0u, 0x4240); }
__device__ __forceinline__ uint32_t odd_bytes(uint32_t w) { return __byte_perm(w, 0u, 0x4341); }
__device__ __forceinline__ uint32_t join_bytes(uint32_t e, uint32_t o) { return __byte_perm(e, o, 0x6240); }

__device__ __forceinline__ bool differs(uint4 a, uint4 b) {
  return ((a.x ^ b.x) | (a.y ^ b.y) | (a.z ^ b.z) | (a.w ^ b.w)) != 0u;
}

__device__ __forceinline__ uint4 ldg4(const uint8_t* p) {
  return __ldg(reinterpret_cast<const uint4*>(p));
}

__device__ __forceinline__ void acc_regs(uint4 w, unsigned long long& s, uint32_t& z) {
  const uint32_t ws[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
  for (int i = 0; i < 4; ++i) {
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const uint32_t r = (ws[i] >> (8 * k)) & 0xFFu;
      s += 1ull << (32 - r);  // r <= 33 - P <= 29 for registers made by add
      z += (r == 0u);
    }
  }
}

__device__ __forceinline__ uint4 shfl_xor4(unsigned mask, uint4 v, int o) {
  return make_uint4(__shfl_xor_sync(mask, v.x, o), __shfl_xor_sync(mask, v.y, o),
                    __shfl_xor_sync(mask, v.z, o), __shfl_xor_sync(mask, v.w, o));
}

struct gather_args {
  const uint64_t* off;        // [V+1] sources of row v: adj[off[v], off[v+1])
  const uint32_t* adj;
  const uint32_t* filter;     // a source is merged only when its bit is set; null = every source
  const uint32_t* covered;    // rows that may change; null = every row
  const uint32_t* stale;      // rows whose nxt copy lags cur (changed last epoch); null = none
  const uint8_t* cur;
  uint8_t* nxt;
  uint32_t* changed;          // out: bitmap of rows changed this epoch (zeroed before)
  double* est;                // per-row estimate, rewritten for changed rows
  const uint32_t* fwd_outdeg; // forward out-degree (the engine's switch weight)
  unsigned long long* counters;  // [0] changed rows, [1] their forward out-degrees, [2] hub cursor
  const uint32_t* hubs;       // rows with more than hub_deg sources
  uint32_t n_hubs;
  uint32_t V;
  uint32_t P;
  uint32_t m;                 // bytes per row (1 << P)
  uint32_t passes;            // m / slice bytes
  uint32_t hub_deg;
  double alpha_mm;
};

// Source rows in flight per lane: 8 / VEC (VEC 16-byte words each), at least
// one (measured on B200: 16 rows lost occupancy to registers at every width).
constexpr int kRowsInFlight = 8;
__host__ __device__ constexpr int unroll_for(int vec) {
  return kRowsInFlight / vec < 1 ? 1 : kRowsInFlight / vec;
}

// Source ids a team stages per round (in shared memory, after the filter).
constexpr int kChunk = 32;

// Merges the filtered sources adj[c0, e) of one slice into agg; the team
// takes kChunk ids per round, rounds `stride` ids apart.  Each round the
// team's lanes load kChunk / T ids each (the next round's are loaded before
// this round's rows), keep those that pass the filter compacted in s_ids,
// then gather their rows UNR at a time.  Team-uniform control flow; returns
// whether any source passed the filter.
template <int T, int VEC>
__device__ __forceinline__ bool team_merge(const gather_args& a, uint64_t c0, uint64_t e,
                                           uint64_t stride, size_t col, int tl, int tb,
                                           unsigned tmask, uint32_t* s_ids, uint4 (&agg)[VEC]) {
  constexpr int K = kChunk / T;
  constexpr int UNR = unroll_for(VEC);
  // Up to 2 words per lane, the merge keeps even and odd bytes apart as 16-bit
  // lanes (__vmaxu2, two per word) and joins them once at the end; wider
  // slices keep the byte max (the split doubles the accumulator registers).
  constexpr bool kSplit = VEC <= 2;
  bool any = false;
  uint4 ev[VEC], od[VEC];
#pragma unroll
  for (int q = 0; q < VEC; ++q) ev[q] = od[q] = make_uint4(0u, 0u, 0u, 0u);
  uint32_t nid[K];
#pragma unroll
  for (int j = 0; j < K; ++j) {
    const uint64_t i = c0 + static_cast<uint64_t>(j) * T + tl;
    nid[j] = i < e ? __ldg(a.adj + i) : kNoVertex;
  }
  for (uint64_t c = c0; c < e; c += stride) {
    uint32_t ids[K];
#pragma unroll
    for (int j = 0; j < K; ++j) {
      ids[j] = nid[j];
      const uint64_t i = c + stride + static_cast<uint64_t>(j) * T + tl;
      nid[j] = i < e ? __ldg(a.adj + i) : kNoVertex;
    }
    uint32_t n = 0;
#pragma unroll
    for (int j = 0; j < K; ++j) {
      const bool ok = ids[j] != kNoVertex && (!a.filter || test_bit(a.filter, ids[j]));
      const unsigned bal = __ballot_sync(tmask, ok) >> tb;
      if (ok) s_ids[n + __popc(bal & ((1u << tl) - 1u))] = ids[j];
      n += __popc(bal);
    }
    __syncwarp(tmask);
    any |= n != 0u;
    for (uint32_t k = 0; k < n; k += UNR) {
      uint4 r[UNR][VEC];
#pragma unroll
      for (int j = 0; j < UNR; ++j) {
        const bool has = k + j < n;
        const uint32_t src = has ? s_ids[k + j] : 0u;
#pragma unroll
        for (int q = 0; q < VEC; ++q)
          r[j][q] = has ? ldg4(a.cur + static_cast<size_t>(src) * a.m + col + q * T * 16)
                        : make_uint4(0u, 0u, 0u, 0u);
      }
      if constexpr (kSplit) {
#pragma unroll
        for (int j = 0; j < UNR; ++j)
#pragma unroll
          for (int q = 0; q < VEC; ++q) {
            ev[q].x = __vmaxu2(ev[q].x, even_bytes(r[j][q].x));
            ev[q].y = __vmaxu2(ev[q].y, even_bytes(r[j][q].y));
            ev[q].z = __vmaxu2(ev[q].z, even_bytes(r[j][q].z));
            ev[q].w = __vmaxu2(ev[q].w, even_bytes(r[j][q].w));
            od[q].x = __vmaxu2(od[q].x, odd_bytes(r[j][q].x));
            od[q].y = __vmaxu2(od[q].y, odd_bytes(r[j][q].y));
            od[q].z = __vmaxu2(od[q].z, odd_bytes(r[j][q].z));
            od[q].w = __vmaxu2(od[q].w, odd_bytes(r[j][q].w));
          }
      } else {
#pragma unroll
        for (int j = 0; j < UNR; ++j)
#pragma unroll
          for (int q = 0; q < VEC; ++q) agg[q] = vmax4(agg[q], r[j][q]);
      }
    }
    __syncwarp(tmask);  // s_ids is rewritten next round
  }
  if constexpr (kSplit) {
#pragma unroll
    for (int q = 0; q < VEC; ++q)
      agg[q] = vmax4(agg[q], make_uint4(join_bytes(ev[q].x, od[q].x), join_bytes(ev[q].y, od[q].y),
                                        join_bytes(ev[q].z, od[q].z), join_bytes(ev[q].w, od[q].w)));
  }
  return any;
}

template <int T, int VEC>
__device__ __forceinline__ void load_own(const gather_args& a, uint32_t v, size_t col, uint4 (&own)[VEC]) {
  const uint8_t* p = a.cur + static_cast<size_t>(v) * a.m + col;
#pragma unroll
  for (int q = 0; q < VEC; ++q) own[q] = ldg4(p + q * T * 16);
}

// Applies agg to row v's slice at `col` (own = its current registers): nxt =
// max(cur, agg), written when it changed or the row is stale; accumulates the
// new slice's register sum.
template <int T, int VEC>
__device__ __forceinline__ bool team_apply(const gather_args& a, uint32_t v, size_t col, bool stale,
                                           unsigned tmask, const uint4 (&own)[VEC], const uint4 (&agg)[VEC],
                                           unsigned long long& sfx, uint32_t& zeros) {
  uint8_t* dst = a.nxt + static_cast<size_t>(v) * a.m + col;
  uint4 nw[VEC];
  bool ch = false;
#pragma unroll
  for (int q = 0; q < VEC; ++q) {
    nw[q] = vmax4(own[q], agg[q]);
    ch |= differs(own[q], nw[q]);
  }
  ch = __any_sync(tmask, ch);
  if (ch || stale) {
#pragma unroll
    for (int q = 0; q < VEC; ++q) *reinterpret_cast<uint4*>(dst + q * T * 16) = nw[q];
  }
#pragma unroll
  for (int q = 0; q < VEC; ++q) acc_regs(nw[q], sfx, zeros);
  return ch;
}

// One epoch over the rows with at most hub_deg sources: a team of T lanes per
// row (grid-strided over rows).
template <int T, int VEC>
__global__ void __launch_bounds__(kHllThreads, 4) k_hll_rows(gather_args a) {
  constexpr int SLICE = T * VEC * 16;
  const int lane = threadIdx.x & 31;
  const int tl = lane & (T - 1);
  const int tb = lane - tl;
  const unsigned tmask = T == 32 ? 0xFFFFFFFFu : (((1u << T) - 1u) << tb);
  const uint64_t team = (blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x) / T;
  const uint64_t nteams = static_cast<uint64_t>(gridDim.x) * blockDim.x / T;
  __shared__ uint32_t s_stage[kHllThreads / T][kChunk];
  uint32_t* s_ids = s_stage[threadIdx.x / T];
  unsigned long long n_chg = 0, deg_chg = 0;
  uint64_t nb = 0, ne = 0;
  if (team < a.V) {
    nb = __ldg(a.off + team);
    ne = __ldg(a.off + team + 1);
  }
  for (uint64_t vv = team; vv < a.V; vv += nteams) {
    const uint32_t v = static_cast<uint32_t>(vv);
    const uint64_t b = nb, e = ne;
    if (vv + nteams < a.V) {  // the next row's offsets, one latency early
      nb = __ldg(a.off + vv + nteams);
      ne = __ldg(a.off + vv + nteams + 1);
    }
    if (a.covered && !test_bit(a.covered, v)) continue;
    if (e - b > a.hub_deg) continue;
    const bool stale = a.stale && test_bit(a.stale, v);
    bool row_changed = false;
    unsigned long long sfx = 0;
    uint32_t zeros = 0;
    for (uint32_t pass = 0; pass < a.passes; ++pass) {
      const size_t col = static_cast<size_t>(pass) * SLICE + static_cast<size_t>(tl) * 16;
      uint4 agg[VEC], own[VEC];
#pragma unroll
      for (int q = 0; q < VEC; ++q) {
        agg[q] = make_uint4(0u, 0u, 0u, 0u);
        own[q] = agg[q];
      }
      if (e > b || stale) load_own<T, VEC>(a, v, col, own);  // in flight during the merge
      const bool any = team_merge<T, VEC>(a, b, e, kChunk, col, tl, tb, tmask, s_ids, agg);
      if (!any && !stale) break;  // same scan every pass: nothing to merge, nxt is current
      row_changed |= team_apply<T, VEC>(a, v, col, stale, tmask, own, agg, sfx, zeros);
    }
    if (row_changed) {
#pragma unroll
      for (int o = T / 2; o > 0; o >>= 1) {
        sfx += __shfl_xor_sync(tmask, sfx, o);
        zeros += __shfl_xor_sync(tmask, zeros, o);
      }
      if (tl == 0) {
        a.est[v] = hll_estimate(a.P, a.alpha_mm, sfx, zeros);
        atomicOr(a.changed + (v >> 5), 1u << (v & 31));
        ++n_chg;
        deg_chg += __ldg(a.fwd_outdeg + v);
      }
    }
  }
  n_chg = warp_sum(n_chg);
  deg_chg = warp_sum(deg_chg);
  if (lane == 0 && n_chg) {
    atomicAdd(a.counters, n_chg);
    atomicAdd(a.counters + 1, deg_chg);
  }
}

// One epoch over the rows with more than hub_deg sources: a block per row,
// its kHllThreads / T teams splitting the sources, then a max-reduction over
// the teams (shuffles inside a warp, shared memory across warps).
template <int T, int VEC>
__global__ void __launch_bounds__(kHllThreads, 3) k_hll_hubs(gather_args a) {
  constexpr int SLICE = T * VEC * 16;
  constexpr int kWarps = kHllThreads / 32;
  constexpr int kTeams = kHllThreads / T;
  __shared__ uint4 part[kWarps][T * VEC];
  __shared__ uint32_t s_stage[kTeams][kChunk];
  uint32_t* s_ids = s_stage[threadIdx.x / T];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int tl = lane & (T - 1);
  const int tb = lane - tl;
  const unsigned tmask = T == 32 ? 0xFFFFFFFFu : (((1u << T) - 1u) << tb);
  const uint64_t team_first = static_cast<uint64_t>(threadIdx.x / T) * kChunk;
  __shared__ uint32_t s_next;
  unsigned long long n_chg = 0, deg_chg = 0;
  for (;;) {
    // hubs are listed heaviest first (ascending internal ids); blocks take the
    // next one as they finish
    if (threadIdx.x == 0) s_next = atomicAdd(reinterpret_cast<unsigned int*>(a.counters + 2), 1u);
    __syncthreads();
    const uint32_t h = s_next;
    __syncthreads();
    if (h >= a.n_hubs) break;
    const uint32_t v = a.hubs[h];
    if (a.covered && !test_bit(a.covered, v)) continue;
    const uint64_t b = __ldg(a.off + v), e = __ldg(a.off + v + 1);
    const bool stale = a.stale && test_bit(a.stale, v);
    bool row_changed = false;
    unsigned long long sfx = 0;
    uint32_t zeros = 0;
    for (uint32_t pass = 0; pass < a.passes; ++pass) {
      const size_t col = static_cast<size_t>(pass) * SLICE + static_cast<size_t>(tl) * 16;
      uint4 agg[VEC];
#pragma unroll
      for (int q = 0; q < VEC; ++q) agg[q] = make_uint4(0u, 0u, 0u, 0u);
      bool any = team_merge<T, VEC>(a, b + team_first, e, static_cast<uint64_t>(kTeams) * kChunk, col,
                                    tl, tb, tmask, s_ids, agg);
#pragma unroll
      for (int o = T; o < 32; o <<= 1)
#pragma unroll
        for (int q = 0; q < VEC; ++q) agg[q] = vmax4(agg[q], shfl_xor4(0xFFFFFFFFu, agg[q], o));
      if (lane < T) {
#pragma unroll
        for (int q = 0; q < VEC; ++q) part[warp][q * T + tl] = agg[q];
      }
      any = __syncthreads_or(any);
      if (!any && !stale) break;  // block-uniform
      if (warp == 0 && lane < T) {
#pragma unroll
        for (int q = 0; q < VEC; ++q) {
          uint4 x = part[0][q * T + tl];
#pragma unroll
          for (int w = 1; w < kWarps; ++w) x = vmax4(x, part[w][q * T + tl]);
          agg[q] = x;
        }
        uint4 own[VEC];
        load_own<T, VEC>(a, v, col, own);
        row_changed |= team_apply<T, VEC>(a, v, col, stale, tmask, own, agg, sfx, zeros);
      }
      __syncthreads();  // part is rewritten by the next pass or row
    }
    if (warp == 0 && lane < T && row_changed) {
#pragma unroll
      for (int o = T / 2; o > 0; o >>= 1) {
        sfx += __shfl_xor_sync(tmask, sfx, o);
        zeros += __shfl_xor_sync(tmask, zeros, o);
      }
      if (lane == 0) {
        a.est[v] = hll_estimate(a.P, a.alpha_mm, sfx, zeros);
        atomicOr(a.changed + (v >> 5), 1u << (v & 31));
        ++n_chg;
        deg_chg += __ldg(a.fwd_outdeg + v);
      }
    }
  }
  if (threadIdx.x == 0 && n_chg) {
    atomicAdd(a.counters, n_chg);
    atomicAdd(a.counters + 1, deg_chg);
  }
}

// Rows of covered vertices (every vertex when covered is null) get their own
// id added to an empty register row in both buffers (hyperanf.hpp:111-121,
// nstepdegrees.hpp:303-312); other rows stay zero.
__global__ void k_hll_init(uint8_t* A, uint8_t* B, double* est, const uint32_t* covered,
                           const uint32_t* to_ext, uint32_t V, uint32_t P, double alpha_mm) {
  const uint32_t m = 1u << P, Q = 32u - P;
  for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < V;
       i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
    const uint32_t v = static_cast<uint32_t>(i);
    if (covered && !test_bit(covered, v)) continue;
    const uint32_t h = murmur3_u32(to_ext ? to_ext[v] : v);
    const uint32_t idx = h >> Q;
    const uint32_t lz = static_cast<uint32_t>(__clz(static_cast<int>(h << P)));
    const uint32_t r = (lz < Q ? lz : Q) + 1u;
    A[static_cast<size_t>(v) * m + idx] = static_cast<uint8_t>(r);
    B[static_cast<size_t>(v) * m + idx] = static_cast<uint8_t>(r);
    const unsigned long long sfx = (static_cast<unsigned long long>(m - 1u) << 32) + (1ull << (32 - r));
    est[v] = hll_estimate(P, alpha_mm, sfx, m - 1u);
  }
}

// One spread epoch (nstepdegrees.hpp:198-247): every row not yet covered with
// a source whose `active` bit is set joins `covered` and `next`.  A warp per
// row, 32 sources per step, first hit ends the row.
__global__ void __launch_bounds__(kHllThreads) k_hll_spread(
    const uint64_t* __restrict__ off, const uint32_t* __restrict__ adj,
    const uint32_t* __restrict__ active, uint32_t* covered, uint32_t* next,
    const uint32_t* __restrict__ fwd_outdeg, uint32_t V, unsigned long long* counters) {
  const int lane = threadIdx.x & 31;
  const uint64_t w0 = (blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x) >> 5;
  const uint64_t nw = (static_cast<uint64_t>(gridDim.x) * blockDim.x) >> 5;
  unsigned long long n = 0, deg = 0;
  for (uint64_t vv = w0; vv < V; vv += nw) {
    const uint32_t v = static_cast<uint32_t>(vv);
    if ((covered[v >> 5] >> (v & 31)) & 1u) continue;  // only this warp changes v's bit
    const uint64_t b = off[v], e = off[v + 1];
    bool hit = false;
    for (uint64_t c = b; c < e && !hit; c += 32) {
      const bool ok = c + lane < e && test_bit(active, adj[c + lane]);
      hit = __any_sync(0xFFFFFFFFu, ok);
    }
    if (hit && lane == 0) {
      atomicOr(covered + (v >> 5), 1u << (v & 31));
      atomicOr(next + (v >> 5), 1u << (v & 31));
      ++n;
      deg += fwd_outdeg[v];
    }
  }
  n = warp_sum(n);
  deg = warp_sum(deg);
  if (lane == 0 && n) {
    atomicAdd(counters, n);
    atomicAdd(counters + 1, deg);
  }
}

// One push-mode spread epoch (nstepdegrees.hpp:217-229): the active sources
// scatter over their forward out-edges and mark every destination not yet
// covered in `next`; a warp walks one active source's edges 32 at a time,
// sources found by scanning the active bitmap.  `covered` is only read here
// (the reference merges the epoch's actives into it afterwards, k_bits_or),
// and a destination counts once, when its bit goes from 0 to 1.
__global__ void __launch_bounds__(kHllThreads) k_hll_spread_push(
    const uint64_t* __restrict__ out_off, const uint32_t* __restrict__ out_adj,
    const uint32_t* __restrict__ active, const uint32_t* __restrict__ covered, uint32_t* next,
    const uint32_t* __restrict__ fwd_outdeg, uint32_t words, unsigned long long* counters) {
  const int lane = threadIdx.x & 31;
  const uint64_t w0 = (blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x) >> 5;
  const uint64_t nw = (static_cast<uint64_t>(gridDim.x) * blockDim.x) >> 5;
  unsigned long long n = 0, deg = 0;
  for (uint64_t w = w0; w < words; w += nw) {
    uint32_t bits = __ldg(active + w);  // warp-uniform
    while (bits) {
      const uint32_t u = static_cast<uint32_t>(w * 32 + (__ffs(bits) - 1));
      bits &= bits - 1u;
      const uint64_t b = __ldg(out_off + u), e = __ldg(out_off + u + 1);
      for (uint64_t c = b + lane; c < e; c += 32) {
        const uint32_t dst = __ldg(out_adj + c);
        const uint32_t bit = 1u << (dst & 31);
        if (!(__ldg(covered + (dst >> 5)) & bit)) {
          const uint32_t old = atomicOr(next + (dst >> 5), bit);
          if (!(old & bit)) {
            ++n;
            deg += __ldg(fwd_outdeg + dst);
          }
        }
      }
    }
  }
  n = warp_sum(n);
  deg = warp_sum(deg);
  if (lane == 0 && n) {
    atomicAdd(counters, n);
    atomicAdd(counters + 1, deg);
  }
}

// a |= b over `words` bitmap words.
__global__ void k_bits_or(uint32_t* a, const uint32_t* __restrict__ b, uint32_t words) {
  for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < words;
       i += static_cast<uint64_t>(gridDim.x) * blockDim.x)
    a[i] |= b[i];
}

// Push-mode propagation epoch (hyperanf.hpp:133-147, nstepdegrees.hpp:316-327):
// the rows of the active sources scatter over their forward out-edges into
// nxt with a per-byte max, in three launches.
//   k_hll_sync_rows  nxt = cur for the stale rows (those that changed last
//                    epoch), so every row a source may raise starts equal in
//                    both buffers;
//   k_hll_scatter    a warp per active source, 32 register words a step:
//                    rows of at most 32 words serve 32 / W destinations at
//                    once; a word is raised with compare-and-swap (register
//                    values only grow, so a stale read never skips a raise);
//                    a destination whose row rose gets its changed bit;
//   k_hll_finish     estimate, count and forward out-degree of each changed
//                    row.
// Rows outside `covered` (when given) are never written.
__device__ __forceinline__ uint32_t bitmap_word(const uint32_t* bits, uint64_t w, uint32_t V) {
  if (bits) return __ldg(bits + w);
  const uint64_t lo = w * 32;
  return V - lo >= 32 ? 0xFFFFFFFFu : ((1u << (V - lo)) - 1u);
}

__global__ void __launch_bounds__(kHllThreads) k_hll_sync_rows(const uint32_t* __restrict__ stale, uint32_t words,
                                                              const uint8_t* __restrict__ cur, uint8_t* nxt,
                                                              uint32_t m) {
  const int lane = threadIdx.x & 31;
  const uint64_t w0 = (blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x) >> 5;
  const uint64_t nw = (static_cast<uint64_t>(gridDim.x) * blockDim.x) >> 5;
  const uint32_t q = m / 16;
  for (uint64_t w = w0; w < words; w += nw) {
    uint32_t bits = __ldg(stale + w);
    while (bits) {
      const uint64_t v = w * 32 + (__ffs(bits) - 1);
      bits &= bits - 1u;
      const uint4* src = reinterpret_cast<const uint4*>(cur + v * m);
      uint4* dst = reinterpret_cast<uint4*>(nxt + v * m);
      for (uint32_t i = lane; i < q; i += 32) dst[i] = __ldg(src + i);
    }
  }
}

__global__ void __launch_bounds__(kHllThreads) k_hll_scatter(
    const uint32_t* __restrict__ active, uint32_t V, const uint64_t* __restrict__ out_off,
    const uint32_t* __restrict__ out_adj, const uint32_t* __restrict__ covered,
    const uint32_t* __restrict__ cur, uint32_t* nxt, uint32_t* changed, uint32_t m) {
  const int lane = threadIdx.x & 31;
  const uint64_t w0 = (blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x) >> 5;
  const uint64_t nw = (static_cast<uint64_t>(gridDim.x) * blockDim.x) >> 5;
  const uint32_t W = m / 4;                       // register words per row
  const uint32_t Wc = W < 32 ? W : 32;            // words per destination and step
  const uint32_t G = 32 / Wc;                     // destinations per step
  const uint32_t slot = lane / Wc, wi = lane % Wc;
  const bool lane_on = slot < G;
  const uint32_t passes = W / Wc;
  const uint64_t words = (static_cast<uint64_t>(V) + 31) / 32;
  for (uint64_t w = w0; w < words; w += nw) {
    uint32_t bits = bitmap_word(active, w, V);  // warp-uniform
    while (bits) {
      const uint32_t u = static_cast<uint32_t>(w * 32 + (__ffs(bits) - 1));
      bits &= bits - 1u;
      const uint64_t b = __ldg(out_off + u), e = __ldg(out_off + u + 1);
      for (uint32_t pass = 0; pass < passes; ++pass) {
        const uint32_t col = pass * Wc + wi;
        const uint32_t mine = lane_on ? __ldg(cur + static_cast<size_t>(u) * W + col) : 0u;
        for (uint64_t c = b + slot; c < e; c += G) {
          if (!lane_on) break;
          const uint32_t v = __ldg(out_adj + c);
          if (covered && !test_bit(covered, v)) continue;
          uint32_t* p = nxt + static_cast<size_t>(v) * W + col;
          uint32_t old = *p;
          for (;;) {  // ends: every failed swap saw a word that grew, and words only grow
            const uint32_t want = bmax(old, mine);
            if (want == old) break;
            const uint32_t prev = atomicCAS(p, old, want);
            if (prev == old) {
              atomicOr(changed + (v >> 5), 1u << (v & 31));
              break;
            }
            old = prev;
          }
        }
      }
    }
  }
}

__global__ void __launch_bounds__(kHllThreads) k_hll_finish(
    const uint32_t* __restrict__ changed, uint32_t words, const uint8_t* __restrict__ nxt, double* est,
    uint32_t P, uint32_t m, double alpha_mm, const uint32_t* __restrict__ fwd_outdeg,
    unsigned long long* counters) {
  const int lane = threadIdx.x & 31;
  const uint64_t w0 = (blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x) >> 5;
  const uint64_t nw = (static_cast<uint64_t>(gridDim.x) * blockDim.x) >> 5;
  const uint32_t q = m / 16;
  unsigned long long n = 0, deg = 0;
  for (uint64_t w = w0; w < words; w += nw) {
    uint32_t bits = __ldg(changed + w);
    while (bits) {
      const uint64_t v = w * 32 + (__ffs(bits) - 1);
      bits &= bits - 1u;
      const uint4* row = reinterpret_cast<const uint4*>(nxt + v * m);
      unsigned long long sfx = 0;
      uint32_t zeros = 0;
      for (uint32_t i = lane; i < q; i += 32) acc_regs(row[i], sfx, zeros);
      sfx = warp_sum(sfx);
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) zeros += __shfl_xor_sync(0xFFFFFFFFu, zeros, o);
      if (lane == 0) {
        est[v] = hll_estimate(P, alpha_mm, sfx, zeros);
        ++n;
        deg += __ldg(fwd_outdeg + v);
      }
    }
  }
  n = warp_sum(n);
  deg = warp_sum(deg);
  if (lane == 0 && n) {
    atomicAdd(counters, n);
    atomicAdd(counters + 1, deg);
  }
}

// Count and forward out-degree sum of a vertex set (the switch's weight).
__global__ void k_bits_weight(const uint32_t* __restrict__ bits, const uint32_t* __restrict__ fwd_outdeg,
                              uint32_t V, unsigned long long* counters) {
  unsigned long long n = 0, deg = 0;
  for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < V;
       i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
    const uint32_t v = static_cast<uint32_t>(i);
    if (test_bit(bits, v)) {
      ++n;
      deg += fwd_outdeg[v];
    }
  }
  n = warp_sum(n);
  deg = warp_sum(deg);
  if ((threadIdx.x & 31) == 0 && n) {
    atomicAdd(counters, n);
    atomicAdd(counters + 1, deg);
  }
}

// Rows with more than hub_deg sources, selected in ascending id order (on a
// graph relabelled by descending in-degree: heaviest first).
struct heavy_row {
  const uint64_t* off;
  uint32_t hub_deg;
  __device__ bool operator()(uint32_t v) const { return off[v + 1] - off[v] > hub_deg; }
};

// Deterministic sum of the estimates: fixed contiguous ranges per block, a
// fixed reduction tree, then one block over the partials.
__global__ void __launch_bounds__(kHllThreads) k_sum_partial(const double* __restrict__ x, uint32_t V,
                                                             double* partial) {
  __shared__ double scratch[32];
  const uint64_t per = (static_cast<uint64_t>(V) + gridDim.x - 1) / gridDim.x;
  const uint64_t lo = blockIdx.x * per, hi = lo + per < V ? lo + per : V;
  double s = 0.0;
  for (uint64_t i = lo + threadIdx.x; i < hi; i += blockDim.x) s += x[i];
  s = block_sum<kHllThreads>(s, scratch);
  if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

__global__ void __launch_bounds__(kHllThreads) k_sum_final(const double* __restrict__ partial, uint32_t n,
                                                           double* out) {
  __shared__ double scratch[32];
  double s = 0.0;
  for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) s += partial[i];
  s = block_sum<kHllThreads>(s, scratch);
  if (threadIdx.x == 0) *out = s;
}

// degree[ext(v)] = (uint32)estimate - 1 for every target (nstepdegrees.hpp:357-372).
__global__ void k_nstep_out(const double* __restrict__ est, const uint32_t* __restrict__ target,
                            const uint32_t* __restrict__ to_ext, uint32_t V, uint32_t* out) {
  for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < V;
       i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
    const uint32_t v = static_cast<uint32_t>(i);
    if (test_bit(target, v)) out[to_ext ? to_ext[v] : v] = static_cast<uint32_t>(est[v]) - 1u;
  }
}

// Register rows to caller order: dst row to_ext[v] = src row v.
__global__ void k_rows_to_ext(const uint8_t* __restrict__ src, uint8_t* dst,
                              const uint32_t* __restrict__ to_ext, uint32_t V, uint32_t m) {
  const uint32_t wpr = m / 16;
  const uint64_t n = static_cast<uint64_t>(V) * wpr;
  for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
    const uint32_t v = static_cast<uint32_t>(i / wpr), w = static_cast<uint32_t>(i % wpr);
    const uint32_t d = to_ext ? to_ext[v] : v;
    reinterpret_cast<uint4*>(dst + static_cast<size_t>(d) * m)[w] =
        reinterpret_cast<const uint4*>(src + static_cast<size_t>(v) * m)[w];
  }
}

}  // namespace

// ---------------------------------------------------------------------------

struct hll_direction {
  const uint64_t* off;
  const uint32_t* adj;
  const uint32_t* hubs;
  uint32_t n_hubs;
};

// Per-graph HLL state, kept between calls: register buffers (released after
// a call when they exceed kKeepBytes), estimates, bitmaps, counters and the
// hub-row lists of both directions.
class hll_engine {
 public:
  static constexpr size_t kKeepBytes = 8ull << 30;

  explicit hll_engine(plato_graph* g) : g_(g), st_(g->stream), V_(g->info.vertices) {}

  int init(uint32_t P) {
    P_ = P;
    m_ = 1u << P;
    alpha_ = hll_alpha_mm(P);
    const uint32_t slice = P >= 12 ? 4096u : m_;
    passes_ = m_ / slice;
    hub_deg_ = std::min(kHubMaxDeg, std::max(kHubMinDeg, kHubBytes / m_));
    const size_t rows = static_cast<size_t>(V_ ? V_ : 1) * m_;
    PLATO_TRY(A_.alloc(rows));
    PLATO_TRY(B_.alloc(rows));
    PLATO_TRY(est_.alloc(V_ ? V_ : 1));
    PLATO_TRY(partial_.alloc(kSumBlocks + 1));
    PLATO_TRY(ctr_.alloc(3));
    words_ = (V_ + 31) / 32;
    for (auto& b : bits_) PLATO_TRY(b.alloc(words_ ? words_ : 1));
    for (auto& d : deg_) PLATO_TRY(d.alloc(V_ ? V_ : 1));
    PLATO_TRY(h_ctr_.alloc(3));
    return PLATO_OK;
  }

  // Rows gather their in-neighbours (csr = false) or out-neighbours (csr =
  // true); the hub rows of each direction are listed once per width class.
  int direction(bool csr, hll_direction* d) {
    const int k = csr ? 1 : 0;
    if (hub_deg_of_[k] != hub_deg_) {
      PLATO_TRY(list_hubs(csr ? g_->out_off.p : g_->in_off.p, hub_list_[k], &hub_n_[k]));
      hub_deg_of_[k] = hub_deg_;
    }
    *d = hll_direction{csr ? g_->out_off.p : g_->in_off.p, csr ? g_->out_adj.p : g_->in_adj.p,
                       hub_list_[k].p, hub_n_[k]};
    return PLATO_OK;
  }

  // Large register buffers are not kept past the call.
  void trim() {
    if (A_.bytes() + B_.bytes() > kKeepBytes) {
      A_.release();
      B_.release();
    }
  }

  uint32_t* degrees(int i) { return deg_[i].p; }

 private:
  int list_hubs(const uint64_t* off, dbuf<uint32_t>& list, uint32_t* n) {
    PLATO_TRY(list.alloc(V_ ? V_ : 1));
    *n = 0;
    if (!V_) return PLATO_OK;
    uint32_t* cnt = reinterpret_cast<uint32_t*>(ctr_.p);
    const thrust::counting_iterator<uint32_t> ids(0);
    const heavy_row pred{off, hub_deg_};
    size_t bytes = 0;
    PLATO_CUDA_TRY(cub::DeviceSelect::If(nullptr, bytes, ids, list.p, cnt, V_, pred, st_));
    PLATO_TRY(select_tmp_.alloc(bytes ? bytes : 1));
    PLATO_CUDA_TRY(cub::DeviceSelect::If(select_tmp_.p, bytes, ids, list.p, cnt, V_, pred, st_));
    count_launch();
    PLATO_CUDA_TRY(cudaMemcpyAsync(n, cnt, sizeof(uint32_t), cudaMemcpyDeviceToHost, st_));
    PLATO_CUDA_TRY(cudaStreamSynchronize(st_));
    return PLATO_OK;
  }

 public:
  int clear_bits(uint32_t* b) {
    PLATO_CUDA_TRY(cudaMemsetAsync(b, 0, 4ull * (words_ ? words_ : 1), st_));
    return PLATO_OK;
  }
  int copy_bits(uint32_t* dst, const uint32_t* src) {
    PLATO_CUDA_TRY(cudaMemcpyAsync(dst, src, 4ull * (words_ ? words_ : 1), cudaMemcpyDeviceToDevice, st_));
    return PLATO_OK;
  }
  int zero_counters() {
    PLATO_CUDA_TRY(cudaMemsetAsync(ctr_.p, 0, 3 * sizeof(unsigned long long), st_));
    return PLATO_OK;
  }
  int read_counters(unsigned long long* n, unsigned long long* deg) {
    PLATO_CUDA_TRY(cudaMemcpyAsync(h_ctr_.p, ctr_.p, 2 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st_));
    PLATO_CUDA_TRY(cudaStreamSynchronize(st_));
    *n = h_ctr_.p[0];
    *deg = h_ctr_.p[1];
    return PLATO_OK;
  }

  // Count and forward out-degree sum of a vertex set.
  int weight(const uint32_t* bits, unsigned long long* n, unsigned long long* deg) {
    PLATO_TRY(zero_counters());
    k_bits_weight<<<grid_for(V_, kHllThreads), kHllThreads, 0, st_>>>(bits, g_->out_deg.p, V_, ctr_.p);
    PLATO_LAUNCHED("k_bits_weight");
    return read_counters(n, deg);
  }

  // Fresh registers: covered rows (all when null) hold their own id.
  int init_rows(const uint32_t* covered) {
    if (!V_) return PLATO_OK;
    const size_t rows = static_cast<size_t>(V_) * m_;
    PLATO_CUDA_TRY(cudaMemsetAsync(A_.p, 0, rows, st_));
    PLATO_CUDA_TRY(cudaMemsetAsync(B_.p, 0, rows, st_));
    const uint32_t* to_ext = g_->relabeled ? g_->to_ext.p : nullptr;
    k_hll_init<<<grid_for(V_, kHllThreads), kHllThreads, 0, st_>>>(A_.p, B_.p, est_.p, covered, to_ext,
                                                                   V_, P_, alpha_);
    PLATO_LAUNCHED("k_hll_init");
    cur_ = A_.p;
    nxt_ = B_.p;
    return PLATO_OK;
  }

  // One propagation epoch over `dir`: rows merge their filtered sources.
  // Counters hold the changed rows and their forward out-degrees afterwards.
  int epoch(const hll_direction& dir, const uint32_t* filter, const uint32_t* covered, const uint32_t* stale,
            uint32_t* changed, unsigned long long* n_changed, unsigned long long* deg_changed) {
    PLATO_TRY(clear_bits(changed));
    PLATO_TRY(zero_counters());
    if (V_) {
      gather_args a{};
      a.off = dir.off;
      a.adj = dir.adj;
      a.filter = filter;
      a.covered = covered;
      a.stale = stale;
      a.cur = cur_;
      a.nxt = nxt_;
      a.changed = changed;
      a.est = est_.p;
      a.fwd_outdeg = g_->out_deg.p;
      a.counters = ctr_.p;
      a.hubs = dir.hubs;
      a.n_hubs = dir.n_hubs;
      a.V = V_;
      a.P = P_;
      a.m = m_;
      a.passes = passes_;
      a.hub_deg = hub_deg_;
      a.alpha_mm = alpha_;
      PLATO_TRY(launch_gather(a));
    }
    std::swap(cur_, nxt_);
    return read_counters(n_changed, deg_changed);
  }

  // One push-mode propagation epoch: the rows of `active` (every vertex when
  // null) scatter over their forward out-edges.  Counters as for epoch().
  int epoch_push(const uint32_t* active, const uint32_t* covered, const uint32_t* stale, uint32_t* changed,
                 unsigned long long* n_changed, unsigned long long* deg_changed) {
    PLATO_TRY(clear_bits(changed));
    PLATO_TRY(zero_counters());
    if (V_) {
      const unsigned grid = grid_for(static_cast<uint64_t>(words_) * 32, kHllThreads, 148u * 16u);
      if (stale) {
        k_hll_sync_rows<<<grid, kHllThreads, 0, st_>>>(stale, words_, cur_, nxt_, m_);
        PLATO_LAUNCHED("k_hll_sync_rows");
      }
      {
        prof_scope ps("k_hll_scatter", st_);
        k_hll_scatter<<<grid, kHllThreads, 0, st_>>>(active, V_, g_->out_off.p, g_->out_adj.p, covered,
                                                     reinterpret_cast<const uint32_t*>(cur_),
                                                     reinterpret_cast<uint32_t*>(nxt_), changed, m_);
        PLATO_LAUNCHED("k_hll_scatter");
      }
      k_hll_finish<<<grid, kHllThreads, 0, st_>>>(changed, words_, nxt_, est_.p, P_, m_, alpha_,
                                                  g_->out_deg.p, ctr_.p);
      PLATO_LAUNCHED("k_hll_finish");
    }
    std::swap(cur_, nxt_);
    return read_counters(n_changed, deg_changed);
  }

  // One spread epoch over `dir` (rows = candidates, sources tested in `active`).
  int spread(const hll_direction& dir, const uint32_t* active, uint32_t* covered, uint32_t* next,
             unsigned long long* n, unsigned long long* deg) {
    PLATO_TRY(clear_bits(next));
    PLATO_TRY(zero_counters());
    if (V_) {
      prof_scope ps("k_hll_spread", st_);
      k_hll_spread<<<grid_for(static_cast<uint64_t>(V_) * 32, kHllThreads, 148u * 16u), kHllThreads, 0,
                     st_>>>(dir.off, dir.adj, active, covered, next, g_->out_deg.p, V_, ctr_.p);
      PLATO_LAUNCHED("k_hll_spread");
    }
    return read_counters(n, deg);
  }

  // One push-mode spread epoch: the actives scatter over their forward
  // out-edges, then covered |= next.
  int spread_push(const uint32_t* active, uint32_t* covered, uint32_t* next, unsigned long long* n,
                  unsigned long long* deg) {
    PLATO_TRY(clear_bits(next));
    PLATO_TRY(zero_counters());
    if (V_) {
      {
        prof_scope ps("k_hll_spread_push", st_);
        k_hll_spread_push<<<grid_for(static_cast<uint64_t>(words_) * 32, kHllThreads, 148u * 16u), kHllThreads,
                            0, st_>>>(g_->out_off.p, g_->out_adj.p, active, covered, next, g_->out_deg.p,
                                      words_, ctr_.p);
        PLATO_LAUNCHED("k_hll_spread_push");
      }
      k_bits_or<<<grid_for(words_, kHllThreads), kHllThreads, 0, st_>>>(covered, next, words_);
      PLATO_LAUNCHED("k_bits_or");
    }
    return read_counters(n, deg);
  }

  int sum_estimates(double* out) {
    if (!V_) {
      *out = 0.0;
      return PLATO_OK;
    }
    k_sum_partial<<<kSumBlocks, kHllThreads, 0, st_>>>(est_.p, V_, partial_.p);
    PLATO_LAUNCHED("k_sum_partial");
    k_sum_final<<<1, kHllThreads, 0, st_>>>(partial_.p, kSumBlocks, partial_.p + kSumBlocks);
    PLATO_LAUNCHED("k_sum_final");
    PLATO_CUDA_TRY(cudaMemcpyAsync(out, partial_.p + kSumBlocks, sizeof(double), cudaMemcpyDeviceToHost, st_));
    PLATO_CUDA_TRY(cudaStreamSynchronize(st_));
    return PLATO_OK;
  }

  // Latest registers (the buffer the last epoch wrote) to host, caller order.
  int registers_to_host(uint8_t* out) {
    if (!V_) return PLATO_OK;
    const size_t rows = static_cast<size_t>(V_) * m_;
    const uint8_t* latest = cur_;
    uint8_t* spare = nxt_;
    const uint32_t* to_ext = g_->relabeled ? g_->to_ext.p : nullptr;
    k_rows_to_ext<<<grid_for(rows / 16, kHllThreads), kHllThreads, 0, st_>>>(latest, spare, to_ext, V_, m_);
    PLATO_LAUNCHED("k_rows_to_ext");
    PLATO_CUDA_TRY(cudaMemcpyAsync(out, spare, rows, cudaMemcpyDeviceToHost, st_));
    PLATO_CUDA_TRY(cudaStreamSynchronize(st_));
    return PLATO_OK;
  }

  int degrees_out(const uint32_t* target, uint32_t* d_out) {
    const uint32_t* to_ext = g_->relabeled ? g_->to_ext.p : nullptr;
    k_nstep_out<<<grid_for(V_, kHllThreads), kHllThreads, 0, st_>>>(est_.p, target, to_ext, V_, d_out);
    PLATO_LAUNCHED("k_nstep_out");
    return PLATO_OK;
  }

  uint32_t* bits(int i) { return bits_[i].p; }
  uint32_t V() const { return V_; }
  cudaStream_t stream() const { return st_; }

 private:
  int launch_gather(const gather_args& a) {
    switch (P_) {
      case 4: return launch<1, 1>(a);
      case 5: return launch<2, 1>(a);
      case 6: return launch<4, 1>(a);
      case 7: return launch<8, 1>(a);
      case 8: return launch<16, 1>(a);
      case 9: return launch<32, 1>(a);
      case 10: return launch<32, 2>(a);
      case 11: return launch<32, 4>(a);
      default: return launch<32, 8>(a);
    }
  }

  template <int T, int VEC>
  int launch(const gather_args& a) {
    {
      prof_scope ps("k_hll_rows", st_);
      const unsigned grid = grid_for(static_cast<uint64_t>(V_) * T, kHllThreads, 148u * 8u);
      k_hll_rows<T, VEC><<<grid, kHllThreads, 0, st_>>>(a);
      PLATO_LAUNCHED("k_hll_rows");
    }
    if (a.n_hubs) {
      prof_scope ps("k_hll_hubs", st_);
      const unsigned grid = a.n_hubs < 148u * 8u ? a.n_hubs : 148u * 8u;
      k_hll_hubs<T, VEC><<<grid, kHllThreads, 0, st_>>>(a);
      PLATO_LAUNCHED("k_hll_hubs");
    }
    return PLATO_OK;
  }

  plato_graph* g_;
  cudaStream_t st_;
  uint32_t V_;
  uint32_t P_ = 0, m_ = 0, passes_ = 1, hub_deg_ = 0, words_ = 0;
  double alpha_ = 0.0;
  dbuf<uint8_t> A_, B_;
  uint8_t* cur_ = nullptr;
  uint8_t* nxt_ = nullptr;
  dbuf<double> est_, partial_;
  dbuf<unsigned long long> ctr_;
  dbuf<uint8_t> select_tmp_;
  dbuf<uint32_t> bits_[5];
  dbuf<uint32_t> deg_[2];
  dbuf<uint32_t> hub_list_[2];
  uint32_t hub_n_[2] = {0, 0};
  uint32_t hub_deg_of_[2] = {0, 0};
  struct pinned {
    unsigned long long* p = nullptr;
    int alloc(size_t n) {
      if (p) return PLATO_OK;
      if (cudaMallocHost(reinterpret_cast<void**>(&p), n * sizeof(unsigned long long)) != cudaSuccess) {
        p = nullptr;
        cudaGetLastError();
        return set_error(PLATO_ENOMEM, "cudaMallocHost of the HLL counters failed");
      }
      return PLATO_OK;
    }
    ~pinned() {
      if (p) cudaFreeHost(p);
    }
  } h_ctr_;
};

struct hll_workspace {
  explicit hll_workspace(plato_graph* g) : eng(g) {}
  hll_engine eng;
};

void destroy_hll_workspace(hll_workspace* w) { delete w; }

namespace {

hll_engine& engine_of(plato_graph* g) {
  if (!g->hll_ws) g->hll_ws = new hll_workspace(g);
  return g->hll_ws->eng;
}

void record_mode(plato_run_stats& s, bool push) {
  if (push) {
    if (s.iterations < 64) s.mode_trace |= 1ull << s.iterations;
    ++s.push_iterations;
  } else {
    ++s.pull_iterations;
  }
  ++s.iterations;
}

bool is_push(unsigned long long active_edges, uint64_t edges, double threshold) {
  // dualmode.hpp:262-279 (0/0 is NaN in the reference: never push)
  return edges > 0 && static_cast<double>(active_edges) / static_cast<double>(edges) < threshold;
}

int check_bits(uint32_t bits) {
  if (bits < 4 || bits > 16)
    return set_error(PLATO_EINVAL, "hyperloglog width must be in [4, 16], got " + std::to_string(bits));
  return PLATO_OK;
}

int hyperanf_impl(plato_graph* g, const plato_hyperanf_opts* o, const plato_dualmode_opts* eo,
                  double* avg_distance, double* anfs_out, uint32_t* n_anfs, uint8_t* registers,
                  plato_run_stats* stats) {
  const uint32_t P = o ? o->bits : 6u;
  const uint32_t iterations = o ? o->iteration : 20u;
  const double thr = eo ? eo->push_threshold : 0.05;
  PLATO_TRY(check_bits(P));
  hll_engine& h = engine_of(g);
  PLATO_TRY(h.init(P));
  hll_direction in_dir{};
  PLATO_TRY(h.direction(false, &in_dir));
  PLATO_TRY(h.init_rows(nullptr));
  std::vector<double> anfs;
  double anf = 0.0;
  PLATO_TRY(h.sum_estimates(&anf));
  anfs.push_back(anf);
  plato_run_stats st{};
  const uint64_t E = g->stored_edges;
  unsigned long long active_edges = E;  // every vertex active (hyperanf.hpp:108-109)
  uint32_t* act = h.bits(0);
  uint32_t* chg = h.bits(1);
  bool first = true;
  for (uint32_t it = 0; it < iterations; ++it) {
    const bool push = is_push(active_edges, E, thr);
    record_mode(st, push);
    unsigned long long n = 0, deg = 0;
    if (push)  // the changed rows scatter (the same registers as the gather, at the cost of the actives)
      PLATO_TRY(h.epoch_push(first ? nullptr : act, nullptr, first ? nullptr : act, chg, &n, &deg));
    else
      PLATO_TRY(h.epoch(in_dir, first ? nullptr : act, nullptr, first ? nullptr : act, chg, &n, &deg));
    PLATO_TRY(h.sum_estimates(&anf));
    if (anf - anfs.back() < DBL_EPSILON) break;  // hyperanf.hpp:185-187
    anfs.push_back(anf);
    std::swap(act, chg);
    active_edges = deg;
    first = false;
  }
  // GetAvgDistance (hyperanf.hpp:61-70)
  double avg = 0.0;
  for (size_t i = 1; i < anfs.size(); ++i) avg += static_cast<double>(i) * (anfs[i] - anfs[i - 1]);
  avg /= (anfs.back() - anfs.front());
  if (avg_distance) *avg_distance = avg;
  if (n_anfs) *n_anfs = static_cast<uint32_t>(anfs.size());
  if (anfs_out) std::copy(anfs.begin(), anfs.end(), anfs_out);
  if (registers) PLATO_TRY(h.registers_to_host(registers));
  h.trim();
  if (stats) *stats = st;
  return PLATO_OK;
}

int nstep_impl(plato_graph* g, const plato_nstep_opts* o, const plato_dualmode_opts* eo,
               const uint8_t* targets, uint32_t* in_degrees, uint32_t* out_degrees,
               plato_run_stats* stats) {
  const uint32_t P = o ? o->bits : 6u;
  const uint32_t steps = o ? o->step : 20u;
  const uint32_t type = o ? o->type : static_cast<uint32_t>(PLATO_NSTEP_BOTH);
  const bool opt_directed = o ? o->is_directed != 0 : false;
  const double thr = eo ? eo->push_threshold : 0.05;
  PLATO_TRY(check_bits(P));
  if (type < PLATO_NSTEP_IN || type > PLATO_NSTEP_BOTH)
    return set_error(PLATO_EINVAL, "nstep degrees: type must be 1 (in), 2 (out) or 3 (both)");
  hll_engine& h = engine_of(g);
  PLATO_TRY(h.init(P));
  const uint32_t V = h.V();
  const cudaStream_t s = h.stream();
  // targets (caller ids) -> internal bitmap
  uint32_t* target = h.bits(4);
  {
    std::vector<uint32_t> hb((V + 31) / 32 + 1, 0u);
    const std::vector<uint32_t>* to_int = nullptr;
    if (g->relabeled) PLATO_TRY(host_to_internal(g, &to_int, s));
    for (uint32_t x = 0; x < V; ++x) {
      if (targets && !targets[x]) continue;
      const uint32_t v = to_int ? (*to_int)[x] : x;
      hb[v >> 5] |= 1u << (v & 31);
    }
    PLATO_CUDA_TRY(cudaMemcpyAsync(target, hb.data(), 4ull * ((V + 31) / 32 ? (V + 31) / 32 : 1),
                                   cudaMemcpyHostToDevice, s));
  }
  hll_direction fwd{}, rev{};
  PLATO_TRY(h.direction(false, &fwd));  // rows gather their in-neighbours
  PLATO_TRY(h.direction(true, &rev));   // rows gather their out-neighbours
  uint32_t* d_in = h.degrees(0);
  uint32_t* d_out = h.degrees(1);
  PLATO_CUDA_TRY(cudaMemsetAsync(d_in, 0, 4ull * (V ? V : 1), s));
  PLATO_CUDA_TRY(cudaMemsetAsync(d_out, 0, 4ull * (V ? V : 1), s));
  const uint64_t E = g->stored_edges;
  plato_run_stats st{};
  uint32_t* covered = h.bits(0);

  // One phase: mark_target + spread(reversed) + propagate(!reversed)
  // (nstepdegrees.hpp:380-402).  counting_in: in-degrees (spread against the
  // edges, registers along them); otherwise out-degrees.
  auto phase = [&](bool counting_in, uint32_t* d_deg) -> int {
    uint32_t* act = h.bits(1);
    uint32_t* nxt = h.bits(2);
    PLATO_TRY(h.copy_bits(covered, target));
    PLATO_TRY(h.copy_bits(act, target));
    const bool spread_reversed = counting_in;
    unsigned long long actives = 1, ae = 0, n_targets = 0;
    PLATO_TRY(h.weight(act, &n_targets, &ae));
    for (uint32_t i = 0; i < steps && actives > 0; ++i) {
      const bool push = is_push(ae, E, thr);
      record_mode(st, push);
      if (push) {  // the actives scatter forward (also when the phase is reversed)
        PLATO_TRY(h.spread_push(act, covered, nxt, &actives, &ae));
      } else {     // a pull tests in-neighbours, or out-neighbours when reversed
        PLATO_TRY(h.spread(spread_reversed ? rev : fwd, act, covered, nxt, &actives, &ae));
      }
      std::swap(act, nxt);
    }
    const bool prop_reversed = !counting_in;
    PLATO_TRY(h.init_rows(covered));
    PLATO_TRY(h.copy_bits(act, covered));
    PLATO_TRY(h.weight(act, &actives, &ae));
    uint32_t* chg = h.bits(3);
    bool first = true;
    for (uint32_t i = 0; i < steps && actives > 0; ++i) {
      const bool push = is_push(ae, E, thr);
      record_mode(st, push);
      const uint32_t* stale = first ? nullptr : act;
      if (push) {
        // the actives scatter forward (also when the phase is reversed)
        PLATO_TRY(h.epoch_push(act, covered, stale, chg, &actives, &ae));
      } else if (!prop_reversed) {
        // forward pull from the actives (the registers of a pull from every in-neighbour)
        PLATO_TRY(h.epoch(fwd, act, covered, stale, chg, &actives, &ae));
      } else {
        // reversed pull: every out-neighbour (rows outside `covered` are empty)
        PLATO_TRY(h.epoch(rev, covered, covered, stale, chg, &actives, &ae));
      }
      std::swap(act, chg);
      first = false;
    }
    return h.degrees_out(target, d_deg);
  };

  const bool want_in = type == PLATO_NSTEP_IN || type == PLATO_NSTEP_BOTH;
  const bool want_out = type == PLATO_NSTEP_OUT || type == PLATO_NSTEP_BOTH;
  if (want_in) PLATO_TRY(phase(true, d_in));
  if (want_out) {
    if (type == PLATO_NSTEP_OUT || opt_directed) {
      PLATO_TRY(phase(false, d_out));
    } else {
      // out = in for every vertex (nstepdegrees.hpp:393-398)
      PLATO_CUDA_TRY(cudaMemcpyAsync(d_out, d_in, 4ull * (V ? V : 1), cudaMemcpyDeviceToDevice, s));
    }
  }
  if (in_degrees && V)
    PLATO_CUDA_TRY(cudaMemcpyAsync(in_degrees, d_in, 4ull * V, cudaMemcpyDeviceToHost, s));
  if (out_degrees && V)
    PLATO_CUDA_TRY(cudaMemcpyAsync(out_degrees, d_out, 4ull * V, cudaMemcpyDeviceToHost, s));
  PLATO_CUDA_TRY(cudaStreamSynchronize(s));
  h.trim();
  if (stats) *stats = st;
  return PLATO_OK;
}

}  // namespace
}  // namespace plato_b200

using namespace plato_b200;

extern "C" int plato_hyperanf(plato_graph* g, const plato_hyperanf_opts* opts,
                              const plato_dualmode_opts* engine_opts, double* avg_distance,
                              double* anfs, uint32_t* n_anfs, uint8_t* registers,
                              plato_run_stats* stats) {
  if (!g) return set_error(PLATO_EINVAL, "plato_hyperanf: null graph");
  std::lock_guard<std::mutex> lock(g->mu);
  PLATO_CUDA_TRY(cudaSetDevice(g->device));
  try {
    return hyperanf_impl(g, opts, engine_opts, avg_distance, anfs, n_anfs, registers, stats);
  } catch (const std::exception& e) {
    return set_error(PLATO_ECUDA, std::string("plato_hyperanf: ") + e.what());
  }
}

extern "C" int plato_nstep_degrees(plato_graph* g, const plato_nstep_opts* opts,
                                   const plato_dualmode_opts* engine_opts, const uint8_t* targets,
                                   plato_vid_t* in_degrees, plato_vid_t* out_degrees,
                                   plato_run_stats* stats) {
  if (!g) return set_error(PLATO_EINVAL, "plato_nstep_degrees: null graph");
  std::lock_guard<std::mutex> lock(g->mu);
  PLATO_CUDA_TRY(cudaSetDevice(g->device));
  try {
    return nstep_impl(g, opts, engine_opts, targets, in_degrees, out_degrees, stats);
  } catch (const std::exception& e) {
    return set_error(PLATO_ECUDA, std::string("plato_nstep_degrees: ") + e.what());
  }
}
