// Device graph construction: edge list (host) -> CSC + CSR resident in HBM.
//
// Layout follows the reference's two structures, minus the MPI partitioning:
//   CSC  in_off[V+1] (uint64) + in_adj[E] (uint32 sources)   ~ dcsc_t, dcsc.hpp:148-152
//   CSR  out_off[V+1] (uint64) + out_adj[E] (uint32 dests)   ~ bcsr_t, bcsr.hpp:167-174
// The reference's DCSC drops empty columns (index_/local_vertex_); a single
// partition over compact ids gains nothing from that, so empty columns keep a
// zero-length range.  Undirected input is stored in both directions
// (dcsc.hpp:365-385).  Out-degrees are counted from the in-edge structure, as
// generate_dense_out_degrees_fg does (structure.hpp:291-346).
//
// By default (unless PLATO_GRAPH_NO_RELABEL) the engine renumbers vertices by descending
// in-degree (ties by caller id): CSC columns then form contiguous degree
// bins for the pull kernels, and since in- and out-degree go together in
// power-law graphs the most-gathered rank values share cache lines at the
// front of the rank vector; to_int/to_ext map between the numberings.  Adjacency lists are sorted
// ascending, so the graph is a pure function of the edge multiset.
//
// Weighted graphs (create_dcsc_seqs_from_path<double>, structure.hpp, as
// example/pagerank_weighted.cc:71-74 loads them) carry each edge's double
// weight through the same stable sorts: the CSC keeps a float weight per
// edge (in_w), the CSR side yields each vertex's sum of out-edge weights
// (out_wsum, summed in double per row, in row order, then rounded), the
// v_weight_sum of weighted_pagerank.hpp:86-99.
#include <cub/cub.cuh>

#include <algorithm>
#include <new>

#include "graph.cuh"

namespace plato_b200 {
namespace {

__global__ void k_degrees(const uint32_t* __restrict__ src, const uint32_t* __restrict__ dst,
                          uint64_t n, uint32_t V, int undirected, uint32_t* out_deg,
                          uint32_t* in_deg, unsigned long long* bad) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t s = src[i], d = dst[i];
    if (s >= V || d >= V) {
      atomicAdd(bad, 1ull);
      continue;
    }
    atomicAdd(&out_deg[s], 1u);
    atomicAdd(&in_deg[d], 1u);
    if (undirected) {
      atomicAdd(&out_deg[d], 1u);
      atomicAdd(&in_deg[s], 1u);
    }
  }
}

__global__ void k_relabel_keys(const uint32_t* __restrict__ out_deg, uint32_t V, uint64_t* keys) {
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < V;
       v += (uint64_t)gridDim.x * blockDim.x)
    keys[v] = (static_cast<uint64_t>(0xFFFFFFFFu - out_deg[v]) << 32) | v;
}

__global__ void k_perm_from_keys(const uint64_t* __restrict__ keys, uint32_t V, uint32_t* to_ext,
                                 uint32_t* to_int) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < V;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t ext = static_cast<uint32_t>(keys[i] & 0xFFFFFFFFull);
    to_ext[i] = ext;
    to_int[ext] = static_cast<uint32_t>(i);
  }
}

// keys[i] = (major << shift) | minor, in internal ids; `transpose` selects
// (dst, src) for the CSC or (src, dst) for the CSR.  Undirected input also
// writes the reversed edge at i + n.
__global__ void k_edge_keys(const uint32_t* __restrict__ src, const uint32_t* __restrict__ dst,
                            uint64_t n, int undirected, const uint32_t* __restrict__ to_int,
                            int shift, int by_dst, uint64_t* keys) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t s = src[i], d = dst[i];
    if (to_int) {
      s = to_int[s];
      d = to_int[d];
    }
    const uint64_t major = by_dst ? d : s, minor = by_dst ? s : d;
    keys[i] = (major << shift) | minor;
    if (undirected) keys[n + i] = (minor << shift) | major;
  }
}

// Weights follow their edge keys: vals[i] = w[i], and vals[n + i] = w[i] for
// the reversed copy of an undirected edge.
__global__ void k_edge_vals(const double* __restrict__ w, uint64_t n, int undirected, double* vals) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    vals[i] = w[i];
    if (undirected) vals[n + i] = w[i];
  }
}

__global__ void k_to_float(const double* __restrict__ in, uint64_t n, float* out) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x)
    out[i] = static_cast<float>(in[i]);
}

__global__ void k_keys_to_adj(const uint64_t* __restrict__ keys, uint64_t n, uint64_t mask,
                              uint32_t* adj) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x)
    adj[i] = static_cast<uint32_t>(keys[i] & mask);
}

// deg_int[i] = deg_ext[to_ext[i]] widened to uint64 for the offset scan; off64[V] = 0.
__global__ void k_internal_degrees(const uint32_t* __restrict__ deg_ext,
                                   const uint32_t* __restrict__ to_ext, uint32_t V,
                                   uint32_t* deg_int, uint64_t* deg64) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i <= V;
       i += (uint64_t)gridDim.x * blockDim.x) {
    if (i == V) {
      deg64[V] = 0;
      continue;
    }
    const uint32_t d = deg_ext[to_ext ? to_ext[i] : i];
    if (deg_int) deg_int[i] = d;
    deg64[i] = d;
  }
}

// Merge-path coordinates of tile starts (Merrill & Garland, "Merge-based
// parallel sparse matrix-vector multiplication", SC'16): list A = row end
// offsets in_off[1..V], list B = edge indices 0..E-1.
__global__ void k_merge_tiles(const uint64_t* __restrict__ off, uint32_t V, uint64_t E,
                              uint32_t items, uint32_t T, uint32_t* trow, uint64_t* tedge) {
  for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t <= T;
       t += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t total = static_cast<uint64_t>(V) + E;
    const uint64_t diag = min(t * static_cast<uint64_t>(items), total);
    uint64_t lo = diag > E ? diag - E : 0;
    uint64_t hi = min(diag, static_cast<uint64_t>(V));
    while (lo < hi) {
      const uint64_t pivot = (lo + hi) >> 1;
      if (off[pivot + 1] <= diag - pivot - 1)
        lo = pivot + 1;
      else
        hi = pivot;
    }
    trow[t] = static_cast<uint32_t>(lo);
    tedge[t] = diag - lo;
  }
}

template <typename T>
__global__ void k_scatter_ext(const T* __restrict__ in_int, const uint32_t* __restrict__ to_ext,
                              uint32_t V, T* out_ext) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < V;
       i += (uint64_t)gridDim.x * blockDim.x)
    out_ext[to_ext[i]] = in_int[i];
}

int bits_for(uint64_t maxval) {
  int b = 1;
  while (b < 64 && (maxval >> b) != 0) ++b;
  return b;
}

// Sorts `n` keys (begin..end bit) from `a` into `b`; returns the sorted buffer.
int radix_sort(uint64_t* a, uint64_t* b, uint64_t n, int end_bit, dbuf<uint8_t>& tmp,
               cudaStream_t st, uint64_t** sorted) {
  cub::DoubleBuffer<uint64_t> db(a, b);
  size_t bytes = 0;
  PLATO_CUDA_TRY(cub::DeviceRadixSort::SortKeys(nullptr, bytes, db, static_cast<int64_t>(n), 0,
                                                end_bit, st));
  PLATO_TRY(tmp.alloc(bytes));
  PLATO_CUDA_TRY(cub::DeviceRadixSort::SortKeys(tmp.p, bytes, db, static_cast<int64_t>(n), 0,
                                                end_bit, st));
  count_launch();
  *sorted = db.Current();
  return PLATO_OK;
}

// Stable key sort carrying double values.
int radix_sort_pairs(uint64_t* ka, uint64_t* kb, double* va, double* vb, uint64_t n, int end_bit,
                     dbuf<uint8_t>& tmp, cudaStream_t st, uint64_t** sk, double** sv) {
  cub::DoubleBuffer<uint64_t> dk(ka, kb);
  cub::DoubleBuffer<double> dv(va, vb);
  size_t bytes = 0;
  PLATO_CUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, bytes, dk, dv, static_cast<int64_t>(n), 0,
                                                 end_bit, st));
  PLATO_TRY(tmp.alloc(bytes));
  PLATO_CUDA_TRY(cub::DeviceRadixSort::SortPairs(tmp.p, bytes, dk, dv, static_cast<int64_t>(n), 0,
                                                 end_bit, st));
  count_launch();
  *sk = dk.Current();
  *sv = dv.Current();
  return PLATO_OK;
}

int exclusive_scan_u64(const uint64_t* in, uint64_t* out, uint64_t n, dbuf<uint8_t>& tmp,
                       cudaStream_t st) {
  size_t bytes = 0;
  PLATO_CUDA_TRY(cub::DeviceScan::ExclusiveSum(nullptr, bytes, in, out, static_cast<int64_t>(n), st));
  PLATO_TRY(tmp.alloc(bytes));
  PLATO_CUDA_TRY(cub::DeviceScan::ExclusiveSum(tmp.p, bytes, in, out, static_cast<int64_t>(n), st));
  count_launch();
  return PLATO_OK;
}

// Edge weights of one side (weighted graphs): the sorted values are kept
// per edge (edge_w, the CSC) or summed per row (row_wsum, the CSR).
struct side_weights {
  const double* w = nullptr;  // input order, device
  dbuf<double>* va = nullptr;
  dbuf<double>* vb = nullptr;
  dbuf<float>* edge_w = nullptr;
  dbuf<float>* row_wsum = nullptr;
};

int build_side(plato_graph* g, const dbuf<uint32_t>& d_src, const dbuf<uint32_t>& d_dst,
               const dbuf<uint32_t>& deg_ext, bool by_dst, dbuf<uint64_t>& keys_a,
               dbuf<uint64_t>& keys_b, dbuf<uint8_t>& tmp, dbuf<uint64_t>& off,
               dbuf<uint32_t>& adj, dbuf<uint32_t>* deg_int, cudaStream_t st,
               const side_weights& sw = side_weights()) {
  const uint32_t V = g->info.vertices;
  const uint64_t n = g->info.edges;
  const uint64_t E = g->stored_edges;
  const int undirected = g->info.is_directed ? 0 : 1;
  const int shift = bits_for(V > 0 ? V - 1 : 0);
  k_edge_keys<<<grid_for(n, 256), 256, 0, st>>>(d_src.p, d_dst.p, n, undirected,
                                                 g->relabeled ? g->to_int.p : nullptr, shift,
                                                 by_dst ? 1 : 0, keys_a.p);
  PLATO_LAUNCHED("k_edge_keys");
  uint64_t* sorted = keys_a.p;
  double* sorted_w = nullptr;
  if (sw.w) {
    k_edge_vals<<<grid_for(n, 256), 256, 0, st>>>(sw.w, n, undirected, sw.va->p);
    PLATO_LAUNCHED("k_edge_vals");
    sorted_w = sw.va->p;
    if (E > 1)
      PLATO_TRY(radix_sort_pairs(keys_a.p, keys_b.p, sw.va->p, sw.vb->p, E, 2 * shift, tmp, st, &sorted,
                                 &sorted_w));
  } else if (E > 1) {
    PLATO_TRY(radix_sort(keys_a.p, keys_b.p, E, 2 * shift, tmp, st, &sorted));
  }
  PLATO_TRY(adj.alloc(E > 0 ? E : 1));
  k_keys_to_adj<<<grid_for(E, 256), 256, 0, st>>>(sorted, E, (1ull << shift) - 1, adj.p);
  PLATO_LAUNCHED("k_keys_to_adj");
  // degrees in internal order -> offsets
  dbuf<uint64_t> deg64;
  PLATO_TRY(deg64.alloc(static_cast<size_t>(V) + 1));
  if (deg_int) PLATO_TRY(deg_int->alloc(V > 0 ? V : 1));
  k_internal_degrees<<<grid_for(static_cast<uint64_t>(V) + 1, 256), 256, 0, st>>>(
      deg_ext.p, g->relabeled ? g->to_ext.p : nullptr, V, deg_int ? deg_int->p : nullptr,
      deg64.p);
  PLATO_LAUNCHED("k_internal_degrees");
  PLATO_TRY(off.alloc(static_cast<size_t>(V) + 1));
  PLATO_TRY(exclusive_scan_u64(deg64.p, off.p, static_cast<uint64_t>(V) + 1, tmp, st));
  if (sw.edge_w) {
    PLATO_TRY(sw.edge_w->alloc(E > 0 ? E : 1));
    if (E > 0) {
      k_to_float<<<grid_for(E, 256), 256, 0, st>>>(sorted_w, E, sw.edge_w->p);
      PLATO_LAUNCHED("k_to_float");
    }
  }
  if (sw.row_wsum) {
    // per-row sums in double (a fixed reduction per segment), then float
    dbuf<double> sums;
    PLATO_TRY(sums.alloc(V));
    size_t bytes = 0;
    PLATO_CUDA_TRY(cub::DeviceSegmentedReduce::Sum(nullptr, bytes, sorted_w, sums.p, static_cast<int64_t>(V),
                                                   off.p, off.p + 1, st));
    PLATO_TRY(tmp.alloc(bytes));
    PLATO_CUDA_TRY(cub::DeviceSegmentedReduce::Sum(tmp.p, bytes, sorted_w, sums.p, static_cast<int64_t>(V),
                                                   off.p, off.p + 1, st));
    count_launch();
    PLATO_TRY(sw.row_wsum->alloc(V));
    k_to_float<<<grid_for(V, 256), 256, 0, st>>>(sums.p, V, sw.row_wsum->p);
    PLATO_LAUNCHED("k_to_float");
    PLATO_CUDA_TRY(cudaStreamSynchronize(st));  // sums is freed on return
  }
  return PLATO_OK;
}

int create_impl(const plato_graph_info* info, const uint32_t* src, const uint32_t* dst,
                const double* weights, uint32_t flags, plato_graph* g) {
  g->info = *info;
  g->info.max_v_i = info->vertices > 0 ? info->vertices - 1 : 0;
  const uint32_t V = info->vertices;
  const uint64_t n = info->edges;
  g->stored_edges = info->is_directed ? n : 2 * n;
  const uint64_t E = g->stored_edges;
  PLATO_CUDA_TRY(cudaGetDevice(&g->device));
  PLATO_CUDA_TRY(cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking));
  cudaStream_t st = g->stream;

  dbuf<uint32_t> d_src, d_dst, deg_out_ext, deg_in_ext;
  dbuf<unsigned long long> bad;
  PLATO_TRY(d_src.alloc(n > 0 ? n : 1));
  PLATO_TRY(d_dst.alloc(n > 0 ? n : 1));
  PLATO_TRY(deg_out_ext.alloc(V));
  PLATO_TRY(deg_in_ext.alloc(V));
  PLATO_TRY(bad.alloc(1));
  if (n > 0) {
    PLATO_CUDA_TRY(cudaMemcpyAsync(d_src.p, src, n * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
    PLATO_CUDA_TRY(cudaMemcpyAsync(d_dst.p, dst, n * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
  }
  PLATO_CUDA_TRY(cudaMemsetAsync(deg_out_ext.p, 0, V * sizeof(uint32_t), st));
  PLATO_CUDA_TRY(cudaMemsetAsync(deg_in_ext.p, 0, V * sizeof(uint32_t), st));
  PLATO_CUDA_TRY(cudaMemsetAsync(bad.p, 0, sizeof(unsigned long long), st));
  if (n > 0) {
    k_degrees<<<grid_for(n, 256), 256, 0, st>>>(d_src.p, d_dst.p, n, V,
                                                info->is_directed ? 0 : 1, deg_out_ext.p,
                                                deg_in_ext.p, bad.p);
    PLATO_LAUNCHED("k_degrees");
  }
  unsigned long long h_bad = 0;
  PLATO_CUDA_TRY(cudaMemcpyAsync(&h_bad, bad.p, sizeof(h_bad), cudaMemcpyDeviceToHost, st));
  PLATO_CUDA_TRY(cudaStreamSynchronize(st));
  if (h_bad)
    return set_error(PLATO_EINVAL, "plato_graph_create: " + std::to_string(h_bad) +
                                       " edges have an endpoint >= vertices (ids must be compact)");

  dbuf<uint8_t> tmp;
  g->relabeled = (flags & PLATO_GRAPH_NO_RELABEL) == 0 && V > 1;
  if (g->relabeled) {
    dbuf<uint64_t> ka, kb;
    PLATO_TRY(ka.alloc(V));
    PLATO_TRY(kb.alloc(V));
    k_relabel_keys<<<grid_for(V, 256), 256, 0, st>>>(deg_in_ext.p, V, ka.p);
    PLATO_LAUNCHED("k_relabel_keys");
    uint64_t* sorted = nullptr;
    PLATO_TRY(radix_sort(ka.p, kb.p, V, 64, tmp, st, &sorted));
    PLATO_TRY(g->to_ext.alloc(V));
    PLATO_TRY(g->to_int.alloc(V));
    k_perm_from_keys<<<grid_for(V, 256), 256, 0, st>>>(sorted, V, g->to_ext.p, g->to_int.p);
    PLATO_LAUNCHED("k_perm_from_keys");
  }

  {
    dbuf<uint64_t> keys_a, keys_b;
    PLATO_TRY(keys_a.alloc(E > 0 ? E : 1));
    PLATO_TRY(keys_b.alloc(E > 0 ? E : 1));
    dbuf<double> d_w, va, vb;
    side_weights in_sw, out_sw;
    if (weights) {
      g->weighted = true;
      PLATO_TRY(d_w.alloc(n > 0 ? n : 1));
      PLATO_TRY(va.alloc(E > 0 ? E : 1));
      PLATO_TRY(vb.alloc(E > 0 ? E : 1));
      if (n > 0)
        PLATO_CUDA_TRY(cudaMemcpyAsync(d_w.p, weights, n * sizeof(double), cudaMemcpyHostToDevice, st));
      in_sw = side_weights{d_w.p, &va, &vb, &g->in_w, nullptr};
      out_sw = side_weights{d_w.p, &va, &vb, nullptr, &g->out_wsum};
    }
    PLATO_TRY(build_side(g, d_src, d_dst, deg_in_ext, true, keys_a, keys_b, tmp, g->in_off,
                         g->in_adj, &g->in_deg, st, in_sw));
    PLATO_TRY(build_side(g, d_src, d_dst, deg_out_ext, false, keys_a, keys_b, tmp, g->out_off,
                         g->out_adj, &g->out_deg, st, out_sw));
    PLATO_CUDA_TRY(cudaStreamSynchronize(st));
  }
  return PLATO_OK;
}

}  // namespace

int ensure_pull_tiles(plato_graph* g, uint32_t items, cudaStream_t st, const merge_tiles** out) {
  auto it = g->tiles.find(items);
  if (it != g->tiles.end()) {
    if (out) *out = &it->second;
    return PLATO_OK;
  }
  const uint64_t total = static_cast<uint64_t>(g->info.vertices) + g->stored_edges;
  const uint64_t T = (total + items - 1) / items;
  if (T >= 0xFFFFFFFFull) return set_error(PLATO_EINVAL, "graph too large for the tile size");
  merge_tiles mt;
  mt.items = items;
  mt.count = static_cast<uint32_t>(T);
  PLATO_TRY(mt.row.alloc(T + 1));
  PLATO_TRY(mt.edge.alloc(T + 1));
  k_merge_tiles<<<grid_for(T + 1, 256), 256, 0, st>>>(g->in_off.p, g->info.vertices,
                                                      g->stored_edges, items, mt.count, mt.row.p,
                                                      mt.edge.p);
  PLATO_LAUNCHED("k_merge_tiles");
  auto& slot = g->tiles[items];
  slot = std::move(mt);
  if (out) *out = &slot;
  return PLATO_OK;
}

int scatter_to_external_f32(const plato_graph* g, const float* in_int, float* out_ext,
                            cudaStream_t st) {
  const uint32_t V = g->info.vertices;
  if (!g->relabeled) {
    if (in_int != out_ext)
      PLATO_CUDA_TRY(cudaMemcpyAsync(out_ext, in_int, V * sizeof(float), cudaMemcpyDeviceToDevice, st));
    return PLATO_OK;
  }
  k_scatter_ext<float><<<grid_for(V, 256), 256, 0, st>>>(in_int, g->to_ext.p, V, out_ext);
  PLATO_LAUNCHED("k_scatter_ext<float>");
  return PLATO_OK;
}

int scatter_to_external_u32(const plato_graph* g, const uint32_t* in_int, uint32_t* out_ext,
                            cudaStream_t st) {
  const uint32_t V = g->info.vertices;
  if (!g->relabeled) {
    if (in_int != out_ext)
      PLATO_CUDA_TRY(cudaMemcpyAsync(out_ext, in_int, V * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st));
    return PLATO_OK;
  }
  k_scatter_ext<uint32_t><<<grid_for(V, 256), 256, 0, st>>>(in_int, g->to_ext.p, V, out_ext);
  PLATO_LAUNCHED("k_scatter_ext<uint32_t>");
  return PLATO_OK;
}

int lookup_internal(const plato_graph* g, uint32_t ext, uint32_t* internal, cudaStream_t st) {
  if (ext >= g->info.vertices) return set_error(PLATO_EINVAL, "vertex id out of range");
  if (!g->relabeled) {
    *internal = ext;
    return PLATO_OK;
  }
  PLATO_CUDA_TRY(cudaMemcpyAsync(internal, g->to_int.p + ext, sizeof(uint32_t),
                                 cudaMemcpyDeviceToHost, st));
  PLATO_CUDA_TRY(cudaStreamSynchronize(st));
  return PLATO_OK;
}

int host_to_internal(plato_graph* g, const std::vector<uint32_t>** map, cudaStream_t st) {
  *map = nullptr;
  if (!g->relabeled) return PLATO_OK;
  if (g->h_to_int.size() != g->info.vertices) {
    g->h_to_int.resize(g->info.vertices);
    PLATO_CUDA_TRY(cudaMemcpyAsync(g->h_to_int.data(), g->to_int.p,
                                   g->info.vertices * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    PLATO_CUDA_TRY(cudaStreamSynchronize(st));
  }
  *map = &g->h_to_int;
  return PLATO_OK;
}

}  // namespace plato_b200

plato_graph::~plato_graph() {
  plato_b200::destroy_batch_engine(batch_cache);
  plato_b200::destroy_rank_workspace(rank_ws);
  plato_b200::destroy_bfs_workspace(bfs_ws);
  plato_b200::destroy_hll_workspace(hll_ws);
  if (stream) cudaStreamDestroy(stream);
}

using namespace plato_b200;

namespace {

int create_checked(const plato_graph_info* info, const plato_vid_t* src, const plato_vid_t* dst,
                   const double* weights, uint32_t flags, plato_graph** out, const char* who) {
  if (!info || !out) return set_error(PLATO_EINVAL, std::string(who) + ": null argument");
  *out = nullptr;
  if (info->edges > 0 && (!src || !dst))
    return set_error(PLATO_EINVAL, std::string(who) + ": null edge arrays");
  if (info->vertices == 0) return set_error(PLATO_EINVAL, std::string(who) + ": zero vertices");
  if ((flags & PLATO_GRAPH_RELABEL) && (flags & PLATO_GRAPH_NO_RELABEL))
    return set_error(PLATO_EINVAL, std::string(who) + ": PLATO_GRAPH_RELABEL and PLATO_GRAPH_NO_RELABEL together");
  if (flags & ~(PLATO_GRAPH_RELABEL | PLATO_GRAPH_NO_RELABEL))
    return set_error(PLATO_EINVAL, std::string(who) + ": unknown flag bits");
  plato_graph* g = new (std::nothrow) plato_graph();
  if (!g) return set_error(PLATO_ENOMEM, std::string(who) + ": host allocation failed");
  const int s = create_impl(info, src, dst, weights, flags, g);
  if (s != PLATO_OK) {
    delete g;
    return s;
  }
  *out = g;
  return PLATO_OK;
}

}  // namespace

extern "C" int plato_graph_create(const plato_graph_info* info, const plato_vid_t* src,
                                  const plato_vid_t* dst, uint32_t flags, plato_graph** out) {
  return create_checked(info, src, dst, nullptr, flags, out, "plato_graph_create");
}

extern "C" int plato_graph_create_weighted(const plato_graph_info* info, const plato_vid_t* src,
                                           const plato_vid_t* dst, const double* weights, uint32_t flags,
                                           plato_graph** out) {
  if (info && info->edges > 0 && !weights)
    return set_error(PLATO_EINVAL, "plato_graph_create_weighted: null weights");
  static const double kNone = 0.0;
  return create_checked(info, src, dst, weights ? weights : &kNone, flags, out, "plato_graph_create_weighted");
}

extern "C" int plato_graph_destroy(plato_graph* g) {
  if (!g) return PLATO_OK;
  cudaSetDevice(g->device);
  if (g->stream) cudaStreamSynchronize(g->stream);
  delete g;
  return PLATO_OK;
}

extern "C" int plato_graph_get_info(const plato_graph* g, plato_graph_info* info) {
  if (!g || !info) return set_error(PLATO_EINVAL, "plato_graph_get_info: null argument");
  *info = g->info;
  return PLATO_OK;
}

extern "C" int plato_graph_get_device_view(const plato_graph* g, plato_graph_device_view* v) {
  if (!g || !v) return set_error(PLATO_EINVAL, "plato_graph_get_device_view: null argument");
  v->vertices = g->info.vertices;
  v->is_directed = g->info.is_directed;
  v->edges = g->info.edges;
  v->stored_edges = g->stored_edges;
  v->in_offsets = g->in_off.p;
  v->in_adj = g->in_adj.p;
  v->out_offsets = g->out_off.p;
  v->out_adj = g->out_adj.p;
  v->out_degree = g->out_deg.p;
  v->in_degree = g->in_deg.p;
  v->to_internal = g->relabeled ? g->to_int.p : nullptr;
  v->to_external = g->relabeled ? g->to_ext.p : nullptr;
  return PLATO_OK;
}

extern "C" int plato_graph_out_degrees(plato_graph* g, uint32_t* degrees_out) {
  if (!g || !degrees_out) return set_error(PLATO_EINVAL, "plato_graph_out_degrees: null argument");
  std::lock_guard<std::mutex> lock(g->mu);
  PLATO_CUDA_TRY(cudaSetDevice(g->device));
  dbuf<uint32_t> ext;
  PLATO_TRY(ext.alloc(g->info.vertices));
  PLATO_TRY(scatter_to_external_u32(g, g->out_deg.p, ext.p, g->stream));
  PLATO_CUDA_TRY(cudaMemcpyAsync(degrees_out, ext.p, g->info.vertices * sizeof(uint32_t),
                                 cudaMemcpyDeviceToHost, g->stream));
  PLATO_CUDA_TRY(cudaStreamSynchronize(g->stream));
  return PLATO_OK;
}

extern "C" int plato_graph_device_bytes(const plato_graph* g, uint64_t* bytes) {
  if (!g || !bytes) return set_error(PLATO_EINVAL, "plato_graph_device_bytes: null argument");
  *bytes = g->in_off.bytes() + g->out_off.bytes() + g->in_adj.bytes() + g->out_adj.bytes() +
           g->out_deg.bytes() + g->in_deg.bytes() + g->to_int.bytes() + g->to_ext.bytes() +
           g->in_w.bytes() + g->out_wsum.bytes();
  return PLATO_OK;
}
