// Seeded RMAT edge-list generator (host, OpenMP).
//
// Produces the synthetic inputs the engine is measured on: RMAT samples
// (Chakrabarti, Zhan, Faloutsos 2004) with self-loops and duplicates removed
// and ids compacted to [0, V).  Compaction is required by the reference: its
// partitions end at the count of distinct ids (plato/graph/partition/sequence.hpp:67)
// and DCSC demands compact ids (plato/graph/structure/dcsc.hpp:48-49).
//
// Random stream (counter based, so every thread count gives the same graph):
//   base = mix64(seed); word(i, w) = mix64(base + 32*i + w)
//   level l of sample i uses 32 bits of word(i, l/2): low half for even l,
//   high half for odd l; level 0 is the most significant id bit.
//   r < a -> (0,0); r < a+b -> (0,1); r < a+b+c -> (1,0); else (1,1)
//   with thresholds floor(p * 2^32) compared against the 32-bit r.
// Symmetrised graphs keep one (min, max) entry per unordered pair.
// Permutation: compact id c gets the rank of (mix64(mix64(seed ^ P) + c), c).
#include <omp.h>
#include <parallel/algorithm>

#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "plato_b200.h"
#include "host_common.hpp"
#include "edge_list.hpp"

namespace {

inline uint64_t mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ULL;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}

constexpr uint64_t kPermSalt = 0xA5A5F00DC0FFEE11ULL;
constexpr uint64_t kDropped = ~0ULL;

}  // namespace

extern "C" int plato_rmat_generate(const plato_rmat_params* p, plato_edge_list** out) {
  using namespace plato_b200;
  if (!p || !out) return set_error(PLATO_EINVAL, "plato_rmat_generate: null argument");
  if (p->scale < 1 || p->scale > 31)
    return set_error(PLATO_EINVAL, "plato_rmat_generate: scale must be in [1, 31]");
  if (p->edgefactor == 0) return set_error(PLATO_EINVAL, "plato_rmat_generate: edgefactor 0");
  const double a = p->a, b = p->b, c = p->c;
  if (!(a >= 0 && b >= 0 && c >= 0 && a + b + c <= 1.0))
    return set_error(PLATO_EINVAL, "plato_rmat_generate: bad probabilities");
  *out = nullptr;
  try {
    const uint32_t scale = p->scale;
    const uint64_t M = static_cast<uint64_t>(p->edgefactor) << scale;
    const uint64_t ta = static_cast<uint64_t>(a * 4294967296.0);
    const uint64_t tb = static_cast<uint64_t>((a + b) * 4294967296.0);
    const uint64_t tc = static_cast<uint64_t>((a + b + c) * 4294967296.0);
    const uint64_t base = mix64(p->seed);
    const bool sym = p->symmetrize != 0;

    std::vector<uint64_t> keys(M);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < static_cast<int64_t>(M); ++i) {
      uint64_t u = 0, v = 0, h = 0;
      for (uint32_t l = 0; l < scale; ++l) {
        if ((l & 1u) == 0) h = mix64(base + 32ULL * static_cast<uint64_t>(i) + (l >> 1));
        const uint64_t r = (l & 1u) ? (h >> 32) : (h & 0xFFFFFFFFULL);
        uint64_t bu, bv;
        if (r < ta) { bu = 0; bv = 0; }
        else if (r < tb) { bu = 0; bv = 1; }
        else if (r < tc) { bu = 1; bv = 0; }
        else { bu = 1; bv = 1; }
        u = (u << 1) | bu;
        v = (v << 1) | bv;
      }
      if (u == v) { keys[i] = kDropped; continue; }
      if (sym && u > v) std::swap(u, v);
      keys[i] = (u << 32) | v;
    }
    __gnu_parallel::sort(keys.begin(), keys.end());
    // unique, dropping the self-loop markers (they sort last)
    uint64_t n = 0;
    for (uint64_t i = 0; i < M; ++i) {
      const uint64_t k = keys[i];
      if (k == kDropped) break;
      if (n == 0 || keys[n - 1] != k) keys[n++] = k;
    }
    keys.resize(n);
    keys.shrink_to_fit();

    // compaction: ids that appear, in increasing order
    const uint64_t idspace = 1ULL << scale;
    std::vector<uint32_t> newid(idspace, 0);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < static_cast<int64_t>(n); ++i) {
      newid[keys[i] >> 32] = 1;
      newid[keys[i] & 0xFFFFFFFFULL] = 1;
    }
    uint32_t V = 0;
    for (uint64_t x = 0; x < idspace; ++x) {
      const uint32_t present = newid[x];
      newid[x] = present ? V : 0xFFFFFFFFu;
      V += present;
    }
    if (p->permute && V > 1) {
      std::vector<std::pair<uint64_t, uint32_t>> order(V);
      const uint64_t pbase = mix64(p->seed ^ kPermSalt);
#pragma omp parallel for schedule(static)
      for (int64_t cidx = 0; cidx < static_cast<int64_t>(V); ++cidx)
        order[cidx] = {mix64(pbase + static_cast<uint64_t>(cidx)), static_cast<uint32_t>(cidx)};
      __gnu_parallel::sort(order.begin(), order.end());
      std::vector<uint32_t> label(V);
#pragma omp parallel for schedule(static)
      for (int64_t r = 0; r < static_cast<int64_t>(V); ++r) label[order[r].second] = static_cast<uint32_t>(r);
#pragma omp parallel for schedule(static)
      for (int64_t x = 0; x < static_cast<int64_t>(idspace); ++x)
        if (newid[x] != 0xFFFFFFFFu) newid[x] = label[newid[x]];
    }
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < static_cast<int64_t>(n); ++i) {
      uint64_t u = newid[keys[i] >> 32], v = newid[keys[i] & 0xFFFFFFFFULL];
      if (sym && u > v) std::swap(u, v);
      keys[i] = (u << 32) | v;
    }
    if (p->permute) __gnu_parallel::sort(keys.begin(), keys.end());

    auto* el = new plato_edge_list();
    el->vertices = V;
    el->src.resize(n);
    el->dst.resize(n);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < static_cast<int64_t>(n); ++i) {
      el->src[i] = static_cast<plato_vid_t>(keys[i] >> 32);
      el->dst[i] = static_cast<plato_vid_t>(keys[i] & 0xFFFFFFFFULL);
    }
    *out = el;
    return PLATO_OK;
  } catch (const std::bad_alloc&) {
    return set_error(PLATO_ENOMEM, "plato_rmat_generate: host allocation failed");
  }
}

extern "C" int plato_edge_list_info(const plato_edge_list* el, plato_vid_t* vertices,
                                    uint64_t* edges) {
  if (!el) return plato_b200::set_error(PLATO_EINVAL, "plato_edge_list_info: null list");
  if (vertices) *vertices = el->vertices;
  if (edges) *edges = el->src.size();
  return PLATO_OK;
}

extern "C" int plato_edge_list_data(const plato_edge_list* el, const plato_vid_t** src,
                                    const plato_vid_t** dst) {
  if (!el) return plato_b200::set_error(PLATO_EINVAL, "plato_edge_list_data: null list");
  if (src) *src = el->src.data();
  if (dst) *dst = el->dst.data();
  return PLATO_OK;
}

extern "C" int plato_edge_list_free(plato_edge_list* el) {
  delete el;
  return PLATO_OK;
}
