/*
 * rmat.c — seeded RMAT edge lists for the CPU side of the measurements.
 *
 * TEST INFRASTRUCTURE ONLY.  bench.py's reference arm builds its graph with
 * this generator so that its process never loads the product library, and the
 * CPU tests hold it equal to the product's generator and to the numpy
 * restatement in tests/rmat_spec.py.
 *
 * The stream (the same one the product documents in its generator):
 *   base = mix64(seed); word(i, w) = mix64(base + 32*i + w)
 *   level l of sample i uses 32 bits of word(i, l/2): the low half for even l,
 *   the high half for odd l; level 0 is the most significant id bit.
 *   r < a -> (0,0); r < a+b -> (0,1); r < a+b+c -> (1,0); else (1,1), with
 *   thresholds floor(p * 2^32) compared against the 32-bit r.
 * Self-loops and duplicates are dropped (symmetrised lists keep one (min, max)
 * entry per unordered pair), ids are compacted to [0, V) in ascending order
 * (the reference requires compact ids: plato/graph/structure/dcsc.hpp:48-49,
 * plato/graph/partition/sequence.hpp:67) and the list comes out sorted by
 * (src, dst).  mix64 is the SplitMix64 finaliser (Steele, Lea, Flood 2014).
 */
#include <omp.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define EXPORT __attribute__((visibility("default")))

static inline uint64_t mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

/* LSD radix sort of n keys below 2^bits, 16-bit digits, OpenMP.  Returns the
 * buffer (a or tmp) that holds the sorted keys. */
static uint64_t* radix_sort(uint64_t* a, uint64_t* tmp, uint64_t n, int bits) {
  enum { R = 16 };
  const uint64_t B = 1ull << R;
  const int T = omp_get_max_threads();
  uint64_t* hist = (uint64_t*)malloc((size_t)T * B * 8);
  if (!hist) return NULL;
  for (int shift = 0; shift < bits; shift += R) {
#pragma omp parallel num_threads(T)
    {
      const int t = omp_get_thread_num(), nt = omp_get_num_threads();
      const uint64_t lo = n * (uint64_t)t / (uint64_t)nt, hi = n * (uint64_t)(t + 1) / (uint64_t)nt;
      uint64_t* h = hist + (size_t)t * B;
      memset(h, 0, B * 8);
      for (uint64_t i = lo; i < hi; ++i) h[(a[i] >> shift) & (B - 1)]++;
#pragma omp barrier
#pragma omp single
      {
        uint64_t sum = 0;
        for (uint64_t d = 0; d < B; ++d)
          for (int u = 0; u < nt; ++u) {
            const uint64_t c = hist[(size_t)u * B + d];
            hist[(size_t)u * B + d] = sum;
            sum += c;
          }
      }
      for (uint64_t i = lo; i < hi; ++i) tmp[h[(a[i] >> shift) & (B - 1)]++] = a[i];
    }
    uint64_t* s = a;
    a = tmp;
    tmp = s;
  }
  free(hist);
  return a;
}

/* -> 0 ok, 1 bad arguments, 2 out of memory.  *src_out / *dst_out are
 * malloc'd [*n_out] arrays, released with ref_rmat_free. */
EXPORT int ref_rmat(uint32_t scale, uint32_t edgefactor, uint64_t seed, double a, double b,
                    double c, int symmetrize, uint32_t* v_out, uint64_t* n_out,
                    uint32_t** src_out, uint32_t** dst_out) {
  if (scale < 1 || scale > 31 || edgefactor == 0 || !(a >= 0 && b >= 0 && c >= 0 && a + b + c <= 1.0))
    return 1;
  const uint64_t M = (uint64_t)edgefactor << scale;
  const uint64_t ta = (uint64_t)(a * 4294967296.0);
  const uint64_t tb = (uint64_t)((a + b) * 4294967296.0);
  const uint64_t tc = (uint64_t)((a + b + c) * 4294967296.0);
  const uint64_t base = mix64(seed);
  const uint64_t nv = 1ull << scale;
  /* key = (u << scale) | v; u == v == 2^scale - 1 is a self-loop, so that
   * value marks a dropped sample and sorts last */
  const uint64_t dropped = (1ull << (2 * scale)) - 1;
  uint64_t* keys = (uint64_t*)malloc(M * 8);
  uint64_t* tmp = (uint64_t*)malloc(M * 8);
  uint8_t* present = (uint8_t*)calloc(nv, 1);
  uint32_t* newid = (uint32_t*)malloc(nv * 4);
  if (!keys || !tmp || !present || !newid) {
    free(keys); free(tmp); free(present); free(newid);
    return 2;
  }
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < (int64_t)M; ++i) {
    uint64_t u = 0, v = 0, h = 0;
    for (uint32_t l = 0; l < scale; ++l) {
      if ((l & 1u) == 0) h = mix64(base + 32ull * (uint64_t)i + (l >> 1));
      const uint64_t r = (l & 1u) ? (h >> 32) : (h & 0xFFFFFFFFull);
      const uint64_t bu = r >= tb, bv = (r >= ta && r < tb) || r >= tc;
      u = (u << 1) | bu;
      v = (v << 1) | bv;
    }
    if (u == v) {
      keys[i] = dropped;
      continue;
    }
    if (symmetrize && u > v) {
      const uint64_t t = u;
      u = v;
      v = t;
    }
    keys[i] = (u << scale) | v;
  }
  uint64_t* sorted = radix_sort(keys, tmp, M, (int)(2 * scale));
  if (!sorted) {
    free(keys); free(tmp); free(present); free(newid);
    return 2;
  }
  uint64_t* out = sorted == keys ? tmp : keys;
  uint64_t n = 0;
  for (uint64_t i = 0; i < M; ++i) {
    const uint64_t k = sorted[i];
    if (k == dropped) break;
    if (n > 0 && out[n - 1] == k) continue;
    out[n++] = k;
  }
  const uint64_t vmask = nv - 1;
  for (uint64_t i = 0; i < n; ++i) {
    present[out[i] >> scale] = 1;
    present[out[i] & vmask] = 1;
  }
  uint32_t V = 0;
  for (uint64_t x = 0; x < nv; ++x) {
    newid[x] = V;
    V += present[x];
  }
  uint32_t* src = (uint32_t*)malloc((n ? n : 1) * 4);
  uint32_t* dst = (uint32_t*)malloc((n ? n : 1) * 4);
  if (!src || !dst) {
    free(src); free(dst); free(keys); free(tmp); free(present); free(newid);
    return 2;
  }
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < (int64_t)n; ++i) {
    src[i] = newid[out[i] >> scale];
    dst[i] = newid[out[i] & vmask];
  }
  free(keys);
  free(tmp);
  free(present);
  free(newid);
  *v_out = V;
  *n_out = n;
  *src_out = src;
  *dst_out = dst;
  return 0;
}

EXPORT void ref_rmat_free(void* p) { free(p); }
