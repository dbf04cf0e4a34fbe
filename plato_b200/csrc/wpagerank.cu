// Weighted PageRank: algo::weighted_pagerank
// (plato/algo/pagerank/weighted_pagerank.hpp:60-149) on a weighted graph.
//
//   v_weight_sum[u] = sum of the weights of u's out-edges (:86-99; built with
//                     the graph, graph.cu)
//   rank = 1 for every vertex (:104-109), then per epoch
//     y(v)     = sum over in-edges (u, v, w) of rank[u] * w / v_weight_sum[u]   (:112-118)
//     rank'(v) = 1 - d + d * y(v)                                               (:126-137)
//     delta    = sum over all vertices of |rank' - rank|, except in the last
//                epoch; eps > 0 and delta < eps jumps to the last epoch (:131-137)
// Ranks stay in the reference's units (not normalised).
//
// The epoch is the merge-path pull of pull_warp.cuh with per-edge weights
// (kWeighted): the gathered state is z = rank / v_weight_sum, so an edge costs
// its id, its weight and one gathered float, and the update writes rank' and
// z' in the same pass.  A vertex without out-edges is never gathered; one
// whose out-edge weights sum to 0 gives inf * 0 = NaN downstream, as the
// reference's 0 / 0 does.
#include <algorithm>
#include <exception>
#include <mutex>
#include <vector>

#include "graph.cuh"
#include "profile.cuh"
#include "pull_warp.cuh"

namespace plato_b200 {
namespace {

constexpr int kIPT = 7;  // merge items per lane (the tiles of the unweighted pull)
using cfg = pull_warp_cfg<kIPT>;

struct wrank_update {
  const float* __restrict__ r;     // current ranks
  float* __restrict__ rn;          // next ranks
  float* __restrict__ zn;          // next gathered state: rank' / v_weight_sum
  const float* __restrict__ wsum;  // v_weight_sum
  float base;                      // 1 - d
  float d;
  int final_epoch;

  __device__ __forceinline__ bool skip() const { return false; }

  __device__ __forceinline__ double apply(uint32_t v, float y) const {
    const float rv = fmaf(d, y, base);
    rn[v] = rv;
    if (final_epoch) return 0.0;
    zn[v] = rv / __ldg(wsum + v);
    return static_cast<double>(fabsf(rv - __ldg(r + v)));
  }
};

__global__ void k_wpr_init(const float* __restrict__ wsum, uint32_t V, float* r, float* z) {
  for (uint64_t v = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; v < V;
       v += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
    r[v] = 1.0f;
    z[v] = 1.0f / wsum[v];
  }
}

using wpull_kernel_t = void (*)(pull_warp_args, wrank_update);

}  // namespace

struct wpr_workspace {
  dbuf<float> r[2], z[2], out_stage;
  dbuf<float> carry, head;
  dbuf<double> partials;
  uint32_t sms = 0, hub_cap = 0;
};

void destroy_wpr_workspace(wpr_workspace* w) { delete w; }

namespace {

int prepare(plato_graph* g, cudaStream_t st, wpr_workspace** out) {
  if (!g->wpr_ws) g->wpr_ws = new wpr_workspace();
  wpr_workspace* ws = g->wpr_ws;
  const uint32_t V = g->info.vertices;
  if (ws->sms == 0) {
    int sms = 0, optin = 0;
    PLATO_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, g->device));
    PLATO_CUDA_TRY(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, g->device));
    const wpull_kernel_t kern = k_pull_warp<kIPT, wrank_update, true>;
    cudaFuncAttributes fa{};
    PLATO_CUDA_TRY(cudaFuncGetAttributes(&fa, kern));
    const size_t dyn = static_cast<size_t>(optin) - fa.sharedSizeBytes;
    if (dyn <= cfg::kSlices + 64)
      return set_error(PLATO_ECUDA, "weighted pull: not enough shared memory on this device");
    PLATO_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(dyn)));
    ws->hub_cap = static_cast<uint32_t>((dyn - cfg::kSlices - 16) / 4 / 32 * 32);
    ws->sms = static_cast<uint32_t>(sms);
  }
  for (auto& b : ws->r) PLATO_TRY(b.alloc(V));
  for (auto& b : ws->z) PLATO_TRY(b.alloc(V));
  PLATO_TRY(ws->out_stage.alloc(V));
  const uint32_t W = ws->sms * cfg::kWarps;
  PLATO_TRY(ws->carry.alloc(W));
  PLATO_TRY(ws->head.alloc(W));
  PLATO_TRY(ws->partials.alloc(ws->sms + (W + 255) / 256));
  PLATO_TRY(ensure_pull_tiles(g, cfg::kItems, st));
  *out = ws;
  return PLATO_OK;
}

int wpr_impl(plato_graph* g, const plato_pagerank_opts* o, float* ranks, plato_run_stats* stats) {
  if (!g->weighted)
    return set_error(PLATO_EINVAL, "plato_weighted_pagerank: the graph has no edge weights "
                                   "(create it with plato_graph_create_weighted)");
  const uint32_t iterations = o ? o->iteration : 100u;
  const double damping = o ? o->damping : 0.85;
  const double eps = o ? o->eps : 0.001;
  const cudaStream_t st = g->stream;
  const uint32_t V = g->info.vertices;
  wpr_workspace* ws = nullptr;
  PLATO_TRY(prepare(g, st, &ws));
  const merge_tiles& mt = g->tiles.at(cfg::kItems);
  const uint32_t H = std::min<uint32_t>(V, ws->hub_cap);
  const uint32_t W = ws->sms * cfg::kWarps;
  const uint32_t n_part = ws->sms + (W + 255) / 256;
  std::vector<double> h_part(n_part);

  int cur = 0;
  k_wpr_init<<<grid_for(V, 256), 256, 0, st>>>(g->out_wsum.p, V, ws->r[0].p, ws->z[0].p);
  PLATO_LAUNCHED("k_wpr_init");
  plato_run_stats s{};
  double delta = 0.0;  // read back only when eps > 0
  uint32_t epochs = 0;
  for (uint32_t epoch = 0; epoch < iterations; ++epoch) {
    const bool last = epoch + 1 == iterations;
    wrank_update upd{ws->r[cur].p, ws->r[cur ^ 1].p, ws->z[cur ^ 1].p, g->out_wsum.p,
                     static_cast<float>(1.0 - damping), static_cast<float>(damping), last ? 1 : 0};
    pull_warp_args a{mt.row.p, mt.edge.p, mt.count, g->stored_edges, g->in_off.p, g->in_adj.p,
                     ws->z[cur].p, H, ws->carry.p, ws->head.p, ws->partials.p, g->in_w.p};
    {
      prof_scope ps("k_pull_warp_weighted", st);
      k_pull_warp<kIPT, wrank_update, true><<<ws->sms, 1024, cfg::smem_bytes(H), st>>>(a, upd);
      PLATO_LAUNCHED("k_pull_warp_weighted");
    }
    a.partials = ws->partials.p + ws->sms;
    k_pull_warp_fixup<wrank_update><<<(W + 255) / 256, 256, 0, st>>>(a, W, upd);
    PLATO_LAUNCHED("k_pull_warp_fixup");
    ++epochs;
    cur ^= 1;
    if (last) break;
    if (eps > 0.0) {
      PLATO_CUDA_TRY(cudaMemcpyAsync(h_part.data(), ws->partials.p, n_part * sizeof(double),
                                     cudaMemcpyDeviceToHost, st));
      PLATO_CUDA_TRY(cudaStreamSynchronize(st));
      delta = 0.0;
      for (double p : h_part) delta += p;
      if (delta < eps) epoch = iterations - 2;  // next epoch is the last (:135-137)
    }
  }
  if (ranks) {
    PLATO_TRY(scatter_to_external_f32(g, ws->r[cur].p, ws->out_stage.p, st));
    PLATO_CUDA_TRY(cudaMemcpyAsync(ranks, ws->out_stage.p, V * sizeof(float), cudaMemcpyDeviceToHost, st));
  }
  PLATO_CUDA_TRY(cudaStreamSynchronize(st));
  if (stats) {
    s.iterations = epochs;
    s.pull_iterations = epochs;
    s.delta = delta;
    *stats = s;
  }
  return PLATO_OK;
}

}  // namespace
}  // namespace plato_b200

using namespace plato_b200;

extern "C" int plato_weighted_pagerank(plato_graph* g, const plato_pagerank_opts* opts, float* ranks,
                                       plato_run_stats* stats) {
  if (!g) return set_error(PLATO_EINVAL, "plato_weighted_pagerank: null graph");
  std::lock_guard<std::mutex> lock(g->mu);
  PLATO_CUDA_TRY(cudaSetDevice(g->device));
  try {
    return wpr_impl(g, opts, ranks, stats);
  } catch (const std::exception& e) {
    return set_error(PLATO_ECUDA, std::string("plato_weighted_pagerank: ") + e.what());
  }
}
