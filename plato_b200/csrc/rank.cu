// PageRank and personalized PageRank drivers (pull-only and dual-mode).
//
//   plato_pagerank*               algo::pagerank               pagerank.hpp:60-149
//   plato_personalized_pagerank   algo::personalized_pagerank  personalized_pagerank.hpp:40-134
//                                 (PLATO_PPR_PULL) and :137-275 (PLATO_PPR_PUSHPULL)
//
// State between epochs is rank/outdeg, the last epoch stores the rank
// (pagerank.hpp:118-135); with eps > 0 and delta < eps the loop jumps to the
// final epoch (pagerank.hpp:137-139), so one more non-dividing epoch runs.
#include <algorithm>
#include <cmath>
#include <new>
#include <vector>

#include "graph.cuh"
#include "profile.cuh"
#include "pull_merge.cuh"
#include "pull_warp.cuh"
#include "push.cuh"

namespace plato_b200 {

struct rank_workspace {
  dbuf<float> x[2];
  dbuf<float> y;  // push-mode accumulator
  dbuf<float> carry, head;
  dbuf<double> partials;
  dbuf<double> delta;
  uint32_t sms = 0;           // CTAs of the persistent pull kernel
  uint32_t hub_cap = 0;       // ranks the pull kernel can stage in shared memory
  double* h_delta = nullptr;  // pinned
  push_frontier frontier;
  ~rank_workspace() {
    if (h_delta) cudaFreeHost(h_delta);
  }
};

void destroy_rank_workspace(rank_workspace* ws) { delete ws; }

namespace {

#ifndef PLATO_PULL_IPT
#define PLATO_PULL_IPT 7
#endif
constexpr int kIPT = PLATO_PULL_IPT;  // merge items per lane (odd: spreads lanes over banks)
using cfg = pull_warp_cfg<kIPT>;

// Opts the kernel into the largest dynamic shared memory the device allows
// next to its static shared memory; returns the hub capacity (floats) that fits.
template <class Tele>
int set_pull_smem_attr(int device, uint32_t* hub_cap) {
  static uint32_t cap = 0;
  if (cap == 0) {
    int optin = 0;
    PLATO_CUDA_TRY(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device));
    cudaFuncAttributes fa{};
    PLATO_CUDA_TRY(cudaFuncGetAttributes(&fa, k_pull_warp<kIPT, rank_update<Tele>>));
    const size_t dyn = static_cast<size_t>(optin) - fa.sharedSizeBytes;
    if (dyn <= cfg::kSlices + 64)
      return set_error(PLATO_ECUDA, "pull kernel: not enough shared memory on this device");
    PLATO_CUDA_TRY(cudaFuncSetAttribute(k_pull_warp<kIPT, rank_update<Tele>>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        static_cast<int>(dyn)));
    cap = static_cast<uint32_t>((dyn - cfg::kSlices - 16) / 4 / 32 * 32);
  }
  *hub_cap = cap;
  return PLATO_OK;
}

int ensure_ws(plato_graph* g, cudaStream_t st) {
  if (!g->rank_ws) {
    g->rank_ws = new (std::nothrow) rank_workspace();
    if (!g->rank_ws) return set_error(PLATO_ENOMEM, "rank workspace: host allocation failed");
  }
  rank_workspace* ws = g->rank_ws;
  const uint32_t V = g->info.vertices;
  PLATO_TRY(ensure_pull_tiles(g, cfg::kItems, st));
  if (ws->sms == 0) {
    int sms = 0;
    PLATO_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, g->device));
    ws->sms = static_cast<uint32_t>(sms);
  }
  const uint32_t W = ws->sms * cfg::kWarps;
  PLATO_TRY(ws->x[0].alloc(V));
  PLATO_TRY(ws->x[1].alloc(V));
  PLATO_TRY(ws->carry.alloc(W));
  PLATO_TRY(ws->head.alloc(W));
  // pull epochs: one partial per CTA + one per fixup block; dense epochs up to 148 * 8
  PLATO_TRY(ws->partials.alloc(std::max<size_t>(ws->sms + (W + 255) / 256 + 1, 148 * 8)));
  PLATO_TRY(ws->delta.alloc(1));
  if (!ws->h_delta) PLATO_CUDA_TRY(cudaMallocHost(reinterpret_cast<void**>(&ws->h_delta), sizeof(double)));
  uint32_t cap_a = 0, cap_b = 0;
  PLATO_TRY(set_pull_smem_attr<teleport_uniform>(g->device, &cap_a));
  PLATO_TRY(set_pull_smem_attr<teleport_single>(g->device, &cap_b));
  ws->hub_cap = std::min(cap_a, cap_b);
  return PLATO_OK;
}

// pagerank.hpp:90-98 (normalised): x = (1/V) / deg, or 1/V when deg == 0.
__global__ void k_init_pagerank(const uint32_t* __restrict__ deg, uint32_t V, float* x) {
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < V;
       v += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t dg = deg[v];
    x[v] = static_cast<float>(dg > 0 ? 1.0 / (static_cast<double>(V) * dg) : 1.0 / V);
  }
}

// personalized_pagerank.hpp:71-81: x = 0 except x[src] = 1/deg(src) (1 if deg == 0).
__global__ void k_init_single(const uint32_t* __restrict__ deg, uint32_t V, uint32_t src, float* x) {
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < V;
       v += (uint64_t)gridDim.x * blockDim.x) {
    float val = 0.f;
    if (v == src) {
      const uint32_t dg = deg[v];
      val = dg > 0 ? static_cast<float>(1.0 / dg) : 1.f;
    }
    x[v] = val;
  }
}

// One pull epoch: persistent warp-tile gather + cross-range fixup; partial
// deltas to ws->partials (one per CTA, then one per fixup block).
template <class Tele>
int pull_epoch(plato_graph* g, const float* x, float* xn, Tele tele, float d, bool final_epoch,
               cudaStream_t st) {
  rank_workspace* ws = g->rank_ws;
  const merge_tiles& mt = g->tiles.at(cfg::kItems);
  rank_update<Tele> upd{x, xn, g->out_deg.p, tele, d, final_epoch ? 1 : 0};
  const uint32_t H = std::min<uint32_t>(g->info.vertices, ws->hub_cap);
  pull_warp_args a{mt.row.p, mt.edge.p, mt.count, g->stored_edges, g->in_off.p, g->in_adj.p,
                   x, H, ws->carry.p, ws->head.p, ws->partials.p};
  {
    prof_scope ps("k_pull_warp", st);
    k_pull_warp<kIPT, rank_update<Tele>><<<ws->sms, 1024, cfg::smem_bytes(H), st>>>(a, upd);
    PLATO_LAUNCHED("k_pull_warp");
  }
  const uint32_t W = ws->sms * cfg::kWarps;
  a.partials = ws->partials.p + ws->sms;
  {
    prof_scope ps("k_pull_warp_fixup", st);
    k_pull_warp_fixup<rank_update<Tele>><<<(W + 255) / 256, 256, 0, st>>>(a, W, upd);
    PLATO_LAUNCHED("k_pull_warp_fixup");
  }
  return PLATO_OK;
}

int partial_count(const plato_graph* g) {
  const uint32_t W = g->rank_ws->sms * cfg::kWarps;
  return static_cast<int>(g->rank_ws->sms + (W + 255) / 256);
}

// Reads back the epoch's delta (sum of the partials).  Synchronises `st`.
int read_delta(plato_graph* g, uint32_t nparts, cudaStream_t st, double* out) {
  rank_workspace* ws = g->rank_ws;
  k_sum_partials<<<1, 1024, 0, st>>>(ws->partials.p, nparts, ws->delta.p);
  PLATO_LAUNCHED("k_sum_partials");
  PLATO_CUDA_TRY(cudaMemcpyAsync(ws->h_delta, ws->delta.p, sizeof(double), cudaMemcpyDeviceToHost, st));
  PLATO_CUDA_TRY(cudaStreamSynchronize(st));
  *out = *ws->h_delta;
  return PLATO_OK;
}

int check_rank_opts(uint32_t iteration, double damping) {
  if (iteration == 0) return set_error(PLATO_EINVAL, "iteration must be >= 1");
  if (!(damping >= 0.0 && damping <= 1.0)) return set_error(PLATO_EINVAL, "damping must be in [0, 1]");
  return PLATO_OK;
}

// PageRank into d_out (caller ids).  Internal buffers stay on the graph.
int pagerank_impl(plato_graph* g, const plato_pagerank_opts* o, float* d_out, cudaStream_t st,
                  plato_run_stats* stats) {
  PLATO_TRY(check_rank_opts(o->iteration, o->damping));
  PLATO_TRY(ensure_ws(g, st));
  rank_workspace* ws = g->rank_ws;
  const uint32_t V = g->info.vertices;
  const float d = static_cast<float>(o->damping);
  const teleport_uniform tele{static_cast<float>((1.0 - o->damping) / V)};
  k_init_pagerank<<<grid_for(V, 256), 256, 0, st>>>(g->out_deg.p, V, ws->x[0].p);
  PLATO_LAUNCHED("k_init_pagerank");
  int cur = 0;
  uint32_t epochs = 0;
  double delta = 0.0;
  for (uint32_t epoch = 0; epoch < o->iteration; ++epoch) {
    const bool final_epoch = (epoch == o->iteration - 1);
    PLATO_TRY(pull_epoch(g, ws->x[cur].p, ws->x[cur ^ 1].p, tele, d, final_epoch, st));
    ++epochs;
    if (!final_epoch && o->eps > 0.0) {
      PLATO_TRY(read_delta(g, partial_count(g), st, &delta));
      delta *= static_cast<double>(V);  // reference units (ranks summing to ~V)
      if (delta < o->eps) epoch = o->iteration - 2;
    }
    cur ^= 1;
  }
  PLATO_TRY(scatter_to_external_f32(g, ws->x[cur].p, d_out, st));
  if (stats) {
    *stats = plato_run_stats{};
    stats->iterations = epochs;
    stats->pull_iterations = epochs;
    stats->delta = delta;
  }
  return PLATO_OK;
}

// Dense update after a push epoch (personalized_pagerank.hpp:242-266).
template <class Tele>
__global__ void __launch_bounds__(256) k_dense_update(const float* __restrict__ y, uint32_t V,
                                                      rank_update<Tele> upd,
                                                      double* __restrict__ partials) {
  __shared__ double s_red[32];
  double dl = 0.0;
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < V;
       v += (uint64_t)gridDim.x * blockDim.x)
    dl += upd.apply(static_cast<uint32_t>(v), y[v]);
  dl = block_sum<256>(dl, s_red);
  if (threadIdx.x == 0) partials[blockIdx.x] = dl;
}

int ppr_impl(plato_graph* g, const plato_ppr_opts* o, int mode, float* d_out, cudaStream_t st,
             plato_run_stats* stats) {
  PLATO_TRY(check_rank_opts(o->iteration, o->damping));
  if (mode != PLATO_PPR_PULL && mode != PLATO_PPR_PUSHPULL)
    return set_error(PLATO_EINVAL, "personalized_pagerank: unknown mode");
  const uint32_t V = g->info.vertices;
  if (o->src >= V) return set_error(PLATO_EINVAL, "personalized_pagerank: src out of range");
  PLATO_TRY(ensure_ws(g, st));
  rank_workspace* ws = g->rank_ws;
  uint32_t src = 0;
  PLATO_TRY(lookup_internal(g, o->src, &src, st));
  const float d = static_cast<float>(o->damping);
  const teleport_single tele{src, static_cast<float>(1.0 - o->damping)};
  k_init_single<<<grid_for(V, 256), 256, 0, st>>>(g->out_deg.p, V, src, ws->x[0].p);
  PLATO_LAUNCHED("k_init_single");

  bool do_pull = (mode == PLATO_PPR_PULL);
  // personalized_pagerank.hpp:160-161: edges doubled for undirected graphs
  const uint64_t edges = g->stored_edges;
  if (!do_pull) {
    PLATO_TRY(ws->y.alloc(V));
    PLATO_TRY(frontier_alloc(ws->frontier, g));
    PLATO_TRY(frontier_reset(ws->frontier, V, st));
    PLATO_TRY(frontier_seed(ws->frontier, g, src, st));
  }
  const uint32_t dense_blocks = grid_for(V, 256, 148 * 8);
  int cur = 0;
  uint32_t epochs = 0, push_epochs = 0;
  uint64_t trace = 0;
  double delta = 0.0;
  for (uint32_t epoch = 0; epoch < o->iteration; ++epoch) {
    const bool final_epoch = (epoch == o->iteration - 1);
    uint32_t nparts;
    if (!do_pull) {
      // personalized_pagerank.hpp:184-205: sticky switch on active_edges > edges/20
      uint64_t active_edges = 0;
      PLATO_TRY(frontier_active_edges(ws->frontier, st, &active_edges));
      do_pull = active_edges > edges / 20;
    }
    if (do_pull) {
      PLATO_TRY(pull_epoch(g, ws->x[cur].p, ws->x[cur ^ 1].p, tele, d, final_epoch, st));
      nparts = partial_count(g);
    } else {
      PLATO_CUDA_TRY(cudaMemsetAsync(ws->y.p, 0, V * sizeof(float), st));
      PLATO_TRY(frontier_push_scatter(ws->frontier, g, ws->x[cur].p, ws->y.p, st));
      rank_update<teleport_single> upd{ws->x[cur].p, ws->x[cur ^ 1].p, g->out_deg.p, tele, d,
                                       final_epoch ? 1 : 0};
      k_dense_update<teleport_single><<<dense_blocks, 256, 0, st>>>(ws->y.p, V, upd,
                                                                    ws->partials.p);
      PLATO_LAUNCHED("k_dense_update");
      nparts = dense_blocks;
      if (epoch < 64) trace |= (1ull << epoch);
      ++push_epochs;
    }
    ++epochs;
    if (!final_epoch && o->eps > 0.0) {
      PLATO_TRY(read_delta(g, nparts, st, &delta));
      if (delta < o->eps) epoch = o->iteration - 2;
    }
    cur ^= 1;
  }
  PLATO_TRY(scatter_to_external_f32(g, ws->x[cur].p, d_out, st));
  if (stats) {
    *stats = plato_run_stats{};
    stats->iterations = epochs;
    stats->push_iterations = push_epochs;
    stats->pull_iterations = epochs - push_epochs;
    stats->delta = delta;
    stats->mode_trace = trace;
  }
  return PLATO_OK;
}

// Host-buffer wrapper: run into a device staging buffer, copy to `host`.
template <class F>
int with_host_output(plato_graph* g, float* host, F&& run) {
  cudaStream_t st = g->stream;
  dbuf<float> out;
  PLATO_TRY(out.alloc(g->info.vertices));
  PLATO_TRY(run(out.p, st));
  PLATO_CUDA_TRY(cudaMemcpyAsync(host, out.p, g->info.vertices * sizeof(float),
                                 cudaMemcpyDeviceToHost, st));
  PLATO_CUDA_TRY(cudaStreamSynchronize(st));
  return PLATO_OK;
}

}  // namespace
}  // namespace plato_b200

using namespace plato_b200;

extern "C" int plato_pagerank(plato_graph* g, const plato_pagerank_opts* opts, float* ranks,
                              plato_run_stats* stats) {
  if (!g || !opts || !ranks) return set_error(PLATO_EINVAL, "plato_pagerank: null argument");
  std::lock_guard<std::mutex> lock(g->mu);
  PLATO_CUDA_TRY(cudaSetDevice(g->device));
  return with_host_output(g, ranks, [&](float* d_out, cudaStream_t st) {
    return pagerank_impl(g, opts, d_out, st, stats);
  });
}

extern "C" int plato_pagerank_device(plato_graph* g, const plato_pagerank_opts* opts,
                                     float* d_ranks, void* stream, plato_run_stats* stats) {
  if (!g || !opts || !d_ranks) return set_error(PLATO_EINVAL, "plato_pagerank_device: null argument");
  std::lock_guard<std::mutex> lock(g->mu);
  PLATO_CUDA_TRY(cudaSetDevice(g->device));
  return pagerank_impl(g, opts, d_ranks, static_cast<cudaStream_t>(stream), stats);
}

extern "C" int plato_personalized_pagerank(plato_graph* g, const plato_ppr_opts* opts, int mode,
                                           float* ranks, plato_run_stats* stats) {
  if (!g || !opts || !ranks)
    return set_error(PLATO_EINVAL, "plato_personalized_pagerank: null argument");
  std::lock_guard<std::mutex> lock(g->mu);
  PLATO_CUDA_TRY(cudaSetDevice(g->device));
  return with_host_output(g, ranks, [&](float* d_out, cudaStream_t st) {
    return ppr_impl(g, opts, mode, d_out, st, stats);
  });
}
