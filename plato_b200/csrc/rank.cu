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
#include <cstdlib>
#include <new>
#include <vector>

#include "graph.cuh"
#include "profile.cuh"
#include "pull_merge.cuh"
#include "pull_binned.cuh"
#include "pull_warp.cuh"
#include "push.cuh"

namespace plato_b200 {

// Degree-bin plan of a relabelled graph (see pull_binned.cuh).
struct pull_plan {
  bool valid = false;
  uint32_t n_long = 0, n_items = 0, n_hubs = 0;
  uint32_t rows_begin[4] = {0, 0, 0, 0};  // k_pull_rows<16>, <8>, <4> bins; [3] = first short row
  uint32_t blocks_long = 0, blocks_hubs = 0, blocks_rows[3] = {0, 0, 0}, blocks_short = 0;
  dbuf<uint2> items;
  dbuf<uint32_t> hub_rows, hub_item0, hub_pieces;
  dbuf<float> piece_sum;
  uint32_t partials() const {
    return blocks_long + blocks_hubs + blocks_rows[0] + blocks_rows[1] + blocks_rows[2] + blocks_short;
  }
};

struct rank_workspace {
  dbuf<float> x[2];
  dbuf<float> r[2];  // weighted PageRank: ranks (x holds rank / out-weight sum)
  dbuf<float> y;  // push-mode accumulator
  dbuf<float> carry, head;
  dbuf<double> partials;
  dbuf<double> delta;
  uint32_t sms = 0;           // CTAs of the persistent pull kernel
  uint32_t hub_cap = 0;       // ranks the pull kernel can stage in shared memory
  bool plan_built = false;
  pull_plan plan;
  dbuf<uint32_t> seed_bits, seed_list;  // seed-set PPR
  dbuf<float> out_stage;                // caller-id ranks before the copy to the host
  dbuf<int> ctrl;                       // device epoch control (k_epoch_control)
  double* h_delta = nullptr;  // pinned
  int* h_ctrl = nullptr;      // pinned [2]
  push_frontier frontier;
  ~rank_workspace() {
    if (h_delta) cudaFreeHost(h_delta);
    if (h_ctrl) cudaFreeHost(h_ctrl);
  }
};

void destroy_rank_workspace(rank_workspace* ws) { delete ws; }

namespace {

#ifndef PLATO_PULL_IPT
#define PLATO_PULL_IPT 7
#endif
constexpr int kIPT = PLATO_PULL_IPT;  // merge items per lane (odd: spreads lanes over banks)
using cfg = pull_warp_cfg<kIPT>;

// Update of weighted PageRank (weighted_pagerank.hpp:112-137): the pull
// gathers x = rank / v_weight_sum times each edge's weight;
// rank' = 1 - d + d * y, x' = rank' / v_weight_sum, delta += |rank' - rank|.
// A vertex whose out-weights sum to 0 gets x' = inf, so its edges give
// inf * 0 = NaN, as the reference's 0 / 0 does.
struct wrank_update {
  const float* __restrict__ r;     // current ranks
  float* __restrict__ rn;          // next ranks
  float* __restrict__ xn;          // next gathered state
  const float* __restrict__ wsum;  // v_weight_sum
  float base;                      // 1 - d
  float d;
  int final_epoch;

  __device__ __forceinline__ bool skip() const { return false; }

  struct operands {
    float ro;
    float ws;
  };
  __device__ __forceinline__ operands load(uint32_t v) const {
    if (final_epoch) return {0.f, 1.f};
    return {__ldcs(r + v), __ldcs(wsum + v)};
  }

  __device__ __forceinline__ double apply(uint32_t v, float y) const { return apply(v, y, load(v)); }

  __device__ __forceinline__ double apply(uint32_t v, float y, operands o) const {
    const float rv = fmaf(d, y, base);
    rn[v] = rv;
    if (final_epoch) return 0.0;
    xn[v] = rv / o.ws;
    return static_cast<double>(fabsf(rv - o.ro));
  }
};

// PageRank update of one partition whose next state is replicated on every
// partition's GPU: each new value is stored in the local replica and, over
// peer memory (NVLink), at the same place in the other replicas, so the pull
// epoch itself carries the exchange that an all-gather would do after it.
constexpr uint32_t kMaxPartitionPeers = 7;  // 8 partitions (one node) at most
struct bcast_rank_update {
  rank_update<teleport_uniform> u;  // local replica: u.xn
  float* peers[kMaxPartitionPeers];  // this partition's slice of the next state in the other replicas
  uint32_t npeers;
  using operands = rank_update<teleport_uniform>::operands;

  __device__ __forceinline__ bool skip() const { return u.skip(); }
  __device__ __forceinline__ operands load(uint32_t v) const { return u.load(v); }
  __device__ __forceinline__ double apply(uint32_t v, float y) const { return apply(v, y, load(v)); }
  __device__ __forceinline__ double apply(uint32_t v, float y, operands o) const {
    const float r = fmaf(u.d, y, u.tele(v));
    float xv = r;
    double dl = 0.0;
    if (!u.storing_rank()) {  // the update of rank_update::apply (pagerank.hpp:118-135)
      if (o.dg > 0) {
        const float fd = static_cast<float>(o.dg);
        xv = r / fd;
        dl = fabsf(xv - o.xo) * fd;
      } else {
        dl = fabsf(xv - o.xo);
      }
    }
    u.xn[v] = xv;
    for (uint32_t k = 0; k < npeers; ++k) peers[k][v] = xv;
    return dl;
  }
};

// Opts the kernel into the largest dynamic shared memory the device allows
// next to its static shared memory; returns the hub capacity (floats) that fits.
template <class Upd, bool kW = false>
int set_pull_smem_attr(int device, uint32_t* hub_cap) {
  static uint32_t cap = 0;
  if (cap == 0) {
    int optin = 0;
    PLATO_CUDA_TRY(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device));
    cudaFuncAttributes fa{};
    PLATO_CUDA_TRY(cudaFuncGetAttributes(&fa, k_pull_warp<kIPT, Upd, kW>));
    const size_t dyn = static_cast<size_t>(optin) - fa.sharedSizeBytes;
    if (dyn <= cfg::kSlices + 64)
      return set_error(PLATO_ECUDA, "pull kernel: not enough shared memory on this device");
    PLATO_CUDA_TRY(cudaFuncSetAttribute(k_pull_warp<kIPT, Upd, kW>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        static_cast<int>(dyn)));
    cap = static_cast<uint32_t>((dyn - cfg::kSlices - 16) / 4 / 32 * 32);
  }
  *hub_cap = cap;
  return PLATO_OK;
}

// Builds the degree-bin plan when the internal order sorts columns by
// descending in-degree (relabelled graphs); otherwise plan.valid stays false
// and the merge-path kernel handles the pull.
int build_plan(plato_graph* g, pull_plan& pl, cudaStream_t st) {
  const uint32_t V = g->info.vertices;
  if (!g->relabeled) return PLATO_OK;
  std::vector<uint32_t> deg(V);
  PLATO_CUDA_TRY(cudaMemcpyAsync(deg.data(), g->in_deg.p, V * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
  PLATO_CUDA_TRY(cudaStreamSynchronize(st));
  for (uint32_t v = 1; v < V; ++v)
    if (deg[v] > deg[v - 1]) return PLATO_OK;  // not sorted: keep the merge-path kernel
  uint32_t n_long = 0;
  while (n_long < V && deg[n_long] > kRowsMax[0]) ++n_long;
  uint32_t row = n_long;
  for (int b = 0; b < 3; ++b) {
    pl.rows_begin[b] = row;
    const uint32_t lower = b < 2 ? kRowsMax[b + 1] : kShortMax;
    while (row < V && deg[row] > lower) ++row;
  }
  pl.rows_begin[3] = row;
  // long-bin units: the pieces of every hub row, then groups of consecutive
  // rows (up to kGroupRows rows and kGroupEdges edges, at least one row)
  std::vector<uint2> items;
  std::vector<uint32_t> hr, hi0, hp;
  for (uint32_t r = 0; r < n_long; ++r) {
    const uint32_t pieces = (deg[r] + kLongPiece - 1) / kLongPiece;
    if (pieces <= 1) continue;
    hr.push_back(r);
    hi0.push_back(static_cast<uint32_t>(items.size()));
    hp.push_back(pieces);
    for (uint32_t k = 0; k < pieces; ++k) items.push_back(make_uint2(r, kPieceFlag | k));
  }
  for (uint32_t r = 0; r < n_long;) {
    if (deg[r] > kLongPiece) {
      ++r;
      continue;
    }
    uint32_t n = 0, edges = 0;
    while (r + n < n_long && n < kGroupRows && deg[r + n] <= kLongPiece &&
           (n == 0 || edges + deg[r + n] <= kGroupEdges))
      edges += deg[r + n++];
    items.push_back(make_uint2(r, n));
    r += n;
  }
  pl.n_long = n_long;
  pl.n_items = static_cast<uint32_t>(items.size());
  pl.n_hubs = static_cast<uint32_t>(hr.size());
  PLATO_TRY(pl.items.alloc(std::max<size_t>(items.size(), 1)));
  PLATO_TRY(pl.piece_sum.alloc(std::max<size_t>(items.size(), 1)));
  PLATO_TRY(pl.hub_rows.alloc(std::max<size_t>(hr.size(), 1)));
  PLATO_TRY(pl.hub_item0.alloc(std::max<size_t>(hr.size(), 1)));
  PLATO_TRY(pl.hub_pieces.alloc(std::max<size_t>(hr.size(), 1)));
  if (!items.empty())
    PLATO_CUDA_TRY(cudaMemcpyAsync(pl.items.p, items.data(), items.size() * sizeof(uint2), cudaMemcpyHostToDevice, st));
  if (!hr.empty()) {
    PLATO_CUDA_TRY(cudaMemcpyAsync(pl.hub_rows.p, hr.data(), hr.size() * 4, cudaMemcpyHostToDevice, st));
    PLATO_CUDA_TRY(cudaMemcpyAsync(pl.hub_item0.p, hi0.data(), hi0.size() * 4, cudaMemcpyHostToDevice, st));
    PLATO_CUDA_TRY(cudaMemcpyAsync(pl.hub_pieces.p, hp.data(), hp.size() * 4, cudaMemcpyHostToDevice, st));
  }
  PLATO_CUDA_TRY(cudaStreamSynchronize(st));
  const uint64_t n_short = static_cast<uint64_t>(V) - pl.rows_begin[3];
  // fixed grids of up to 8 CTAs (64 warps) per SM; the kernels stride over their work
  int sms = 0;
  PLATO_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, g->device));
  const uint64_t cap = static_cast<uint64_t>(sms) * 8;
  auto blocks = [cap](uint64_t threads) {
    return static_cast<uint32_t>(std::min<uint64_t>((threads + 255) / 256, cap));
  };
  pl.blocks_long = blocks(static_cast<uint64_t>(pl.n_items) * 32);
  pl.blocks_hubs = blocks(static_cast<uint64_t>(pl.n_hubs) * 32);
  for (int b = 0; b < 3; ++b)  // one warp per 32 rows
    pl.blocks_rows[b] = blocks(static_cast<uint64_t>(pl.rows_begin[b + 1] - pl.rows_begin[b] + 31) / 32 * 32);
  pl.blocks_short = blocks(n_short);
  pl.valid = true;
  return PLATO_OK;
}

int ensure_ws(plato_graph* g, cudaStream_t st) {
  if (!g->rank_ws) {
    g->rank_ws = new (std::nothrow) rank_workspace();
    if (!g->rank_ws) return set_error(PLATO_ENOMEM, "rank workspace: host allocation failed");
  }
  rank_workspace* ws = g->rank_ws;
  const uint32_t V = g->info.vertices;
  if (!ws->plan_built) {
    PLATO_TRY(build_plan(g, ws->plan, st));
    ws->plan_built = true;
  }
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
  // pull epochs: one partial per CTA + one per fixup block (merge path) or one
  // per block of each bin kernel; dense epochs up to 148 * 8
  PLATO_TRY(ws->partials.alloc(std::max<size_t>(
      {ws->sms + (W + 255) / 256 + 1, static_cast<size_t>(ws->plan.partials()) + 1, 148 * 8})));
  PLATO_TRY(ws->delta.alloc(1));
  PLATO_TRY(ws->ctrl.alloc(2));
  if (!ws->h_delta) PLATO_CUDA_TRY(cudaMallocHost(reinterpret_cast<void**>(&ws->h_delta), sizeof(double)));
  if (!ws->h_ctrl) PLATO_CUDA_TRY(cudaMallocHost(reinterpret_cast<void**>(&ws->h_ctrl), 2 * sizeof(int)));
  uint32_t cap_a = 0, cap_b = 0;
  PLATO_TRY(set_pull_smem_attr<rank_update<teleport_uniform>>(g->device, &cap_a));
  PLATO_TRY(set_pull_smem_attr<rank_update<teleport_single>>(g->device, &cap_b));
  uint32_t cap_c = 0, cap_d = 0;
  PLATO_TRY(set_pull_smem_attr<rank_update<teleport_seeds>>(g->device, &cap_c));
  PLATO_TRY((set_pull_smem_attr<wrank_update, true>(g->device, &cap_d)));
  uint32_t cap_e = 0;
  PLATO_TRY(set_pull_smem_attr<bcast_rank_update>(g->device, &cap_e));
  cap_d = std::min(cap_d, cap_e);
  cap_b = std::min(cap_b, std::min(cap_c, cap_d));
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

// One pull epoch gathering x (times the edge weights w when kW) with the
// fused update `upd`: the degree bins on a relabelled graph, else the
// persistent warp-tile merge path + cross-range fixup.  Partial deltas go to
// ws->partials (one per CTA of each kernel).
template <class Upd, bool kW>
int pull_epoch_with(plato_graph* g, const float* x, const Upd& upd, const float* w, cudaStream_t st) {
  rank_workspace* ws = g->rank_ws;
  const pull_plan& pl = ws->plan;
  if (pl.valid) {
    const pull_plan_view pv{pl.n_long, pl.rows_begin[3], g->info.vertices, pl.n_items, pl.items.p,
                            pl.n_hubs, pl.hub_rows.p, pl.hub_item0.p, pl.hub_pieces.p,
                            pl.piece_sum.p};
    double* part = ws->partials.p;
    if (pl.blocks_long) {
      prof_scope ps("k_pull_long", st);
      k_pull_long<Upd, kW><<<pl.blocks_long, 256, 0, st>>>(pv, g->in_off.p, g->in_adj.p, x, upd, part, w);
      PLATO_LAUNCHED("k_pull_long");
    }
    part += pl.blocks_long;
    if (pl.blocks_hubs) {
      prof_scope ps("k_pull_hubs", st);
      k_pull_hubs<Upd><<<pl.blocks_hubs, 256, 0, st>>>(pv, upd, part);
      PLATO_LAUNCHED("k_pull_hubs");
    }
    part += pl.blocks_hubs;
    if (pl.blocks_rows[0]) {
      prof_scope ps("k_pull_rows16", st);
      k_pull_rows<16, Upd, kW><<<pl.blocks_rows[0], 256, 0, st>>>(
          pl.rows_begin[0], pl.rows_begin[1], g->in_off.p, g->in_adj.p, x, upd, part, w);
      PLATO_LAUNCHED("k_pull_rows16");
    }
    part += pl.blocks_rows[0];
    if (pl.blocks_rows[1]) {
      prof_scope ps("k_pull_rows8", st);
      k_pull_rows<8, Upd, kW><<<pl.blocks_rows[1], 256, 0, st>>>(
          pl.rows_begin[1], pl.rows_begin[2], g->in_off.p, g->in_adj.p, x, upd, part, w);
      PLATO_LAUNCHED("k_pull_rows8");
    }
    part += pl.blocks_rows[1];
    if (pl.blocks_rows[2]) {
      prof_scope ps("k_pull_rows4", st);
      k_pull_rows<4, Upd, kW><<<pl.blocks_rows[2], 256, 0, st>>>(
          pl.rows_begin[2], pl.rows_begin[3], g->in_off.p, g->in_adj.p, x, upd, part, w);
      PLATO_LAUNCHED("k_pull_rows4");
    }
    part += pl.blocks_rows[2];
    if (pl.blocks_short) {
      prof_scope ps("k_pull_short", st);
      k_pull_short<Upd, kW><<<pl.blocks_short, 256, 0, st>>>(pv, g->in_off.p, g->in_adj.p, x, upd, part, w);
      PLATO_LAUNCHED("k_pull_short");
    }
    return PLATO_OK;
  }
  const merge_tiles& mt = g->tiles.at(cfg::kItems);
  const uint32_t H = std::min<uint32_t>(g->info.vertices, ws->hub_cap);
  pull_warp_args a{mt.row.p, mt.edge.p, mt.count, g->stored_edges, g->in_off.p, g->in_adj.p,
                   x, H, ws->carry.p, ws->head.p, ws->partials.p, w};
  {
    prof_scope ps("k_pull_warp", st);
    k_pull_warp<kIPT, Upd, kW><<<ws->sms, 1024, cfg::smem_bytes(H), st>>>(a, upd);
    PLATO_LAUNCHED("k_pull_warp");
  }
  const uint32_t W = ws->sms * cfg::kWarps;
  a.partials = ws->partials.p + ws->sms;
  {
    prof_scope ps("k_pull_warp_fixup", st);
    k_pull_warp_fixup<Upd><<<(W + 255) / 256, 256, 0, st>>>(a, W, upd);
    PLATO_LAUNCHED("k_pull_warp_fixup");
  }
  return PLATO_OK;
}

template <class Tele>
int pull_epoch(plato_graph* g, const float* x, float* xn, Tele tele, float d, bool final_epoch,
               cudaStream_t st, const int* mode = nullptr) {
  const rank_update<Tele> upd{x, xn, g->out_deg.p, tele, d, final_epoch ? 1 : 0, mode};
  return pull_epoch_with<rank_update<Tele>, false>(g, x, upd, nullptr, st);
}

int partial_count(const plato_graph* g) {
  if (g->rank_ws->plan.valid) return static_cast<int>(g->rank_ws->plan.partials());
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

// Pull-only epochs [start, iteration) from state x[*cur].  With eps == 0 the
// schedule is known and nothing is read back.  With eps > 0 each epoch is
// followed by k_epoch_control, which sums the delta on the device and sets
// the next epoch's kind (pagerank.hpp:137-139); the host enqueues epochs in
// batches and polls the control word between batches, so there is no host
// round trip per epoch.  `scale` converts the delta to the reference's units.
template <class Tele>
int run_pull_epochs(plato_graph* g, Tele tele, float d, uint32_t iteration, uint32_t start,
                    double eps, double scale, cudaStream_t st, int* cur, uint32_t* ran,
                    double* delta) {
  rank_workspace* ws = g->rank_ws;
  *ran = 0;
  if (start >= iteration) return PLATO_OK;
  if (eps <= 0.0) {
    for (uint32_t epoch = start; epoch < iteration; ++epoch) {
      PLATO_TRY(pull_epoch(g, ws->x[*cur].p, ws->x[*cur ^ 1].p, tele, d, epoch == iteration - 1, st));
      *cur ^= 1;
      ++*ran;
    }
    return PLATO_OK;
  }
  const int init[2] = {start == iteration - 1 ? 1 : 0, static_cast<int>(start)};
  PLATO_CUDA_TRY(cudaMemcpyAsync(ws->ctrl.p, init, sizeof(init), cudaMemcpyHostToDevice, st));
  const int cur0 = *cur;
  constexpr uint32_t kBatch = 8;
  uint32_t launched = 0;
  const uint32_t nparts = static_cast<uint32_t>(partial_count(g));
  while (start + launched < iteration) {
    const uint32_t n = std::min(kBatch, iteration - start - launched);
    for (uint32_t k = 0; k < n; ++k) {
      const int c = (cur0 + static_cast<int>(launched + k)) & 1;
      PLATO_TRY(pull_epoch(g, ws->x[c].p, ws->x[c ^ 1].p, tele, d, false, st, ws->ctrl.p));
      k_epoch_control<<<1, 1024, 0, st>>>(ws->partials.p, nparts, ws->ctrl.p, ws->delta.p, scale,
                                          eps, iteration);
      PLATO_LAUNCHED("k_epoch_control");
    }
    launched += n;
    PLATO_CUDA_TRY(cudaMemcpyAsync(ws->h_ctrl, ws->ctrl.p, 2 * sizeof(int), cudaMemcpyDeviceToHost, st));
    PLATO_CUDA_TRY(cudaMemcpyAsync(ws->h_delta, ws->delta.p, sizeof(double), cudaMemcpyDeviceToHost, st));
    PLATO_CUDA_TRY(cudaStreamSynchronize(st));
    if (ws->h_ctrl[0] == 2) break;
  }
  *ran = static_cast<uint32_t>(ws->h_ctrl[1]) - start;
  *cur = (cur0 + static_cast<int>(*ran)) & 1;
  *delta = *ws->h_delta;
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
  // reference units: the reference's ranks sum to ~V
  PLATO_TRY(run_pull_epochs(g, tele, d, o->iteration, 0, o->eps, static_cast<double>(V), st, &cur,
                            &epochs, &delta));
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
  uint32_t epoch = 0;
  // push phase (host-driven: the frontier decides), personalized_pagerank.hpp:184-239
  for (; epoch < o->iteration; ++epoch) {
    if (!do_pull) {
      // personalized_pagerank.hpp:184-205: sticky switch on active_edges > edges/20
      uint64_t active_edges = 0;
      PLATO_TRY(frontier_active_edges(ws->frontier, st, &active_edges));
      do_pull = active_edges > edges / 20;
    }
    if (do_pull) break;
    const bool final_epoch = (epoch == o->iteration - 1);
    PLATO_CUDA_TRY(cudaMemsetAsync(ws->y.p, 0, V * sizeof(float), st));
    PLATO_TRY(frontier_push_scatter(ws->frontier, g, ws->x[cur].p, ws->y.p, st));
    rank_update<teleport_single> upd{ws->x[cur].p, ws->x[cur ^ 1].p, g->out_deg.p, tele, d,
                                     final_epoch ? 1 : 0};
    k_dense_update<teleport_single><<<dense_blocks, 256, 0, st>>>(ws->y.p, V, upd, ws->partials.p);
    PLATO_LAUNCHED("k_dense_update");
    if (epoch < 64) trace |= (1ull << epoch);
    ++push_epochs;
    ++epochs;
    cur ^= 1;
    if (!final_epoch && o->eps > 0.0) {
      PLATO_TRY(read_delta(g, dense_blocks, st, &delta));
      if (delta < o->eps) epoch = o->iteration - 2;
    }
  }
  // pull phase (sticky): device-controlled epochs
  uint32_t pulled = 0;
  PLATO_TRY(run_pull_epochs(g, tele, d, o->iteration, epoch, o->eps, 1.0, st, &cur, &pulled, &delta));
  epochs += pulled;
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

// trustrank.hpp:197-206 with explicit seeds: x = (1/|S|)/deg on seeds (1/|S| if deg 0).
__global__ void k_init_seeds(const uint32_t* __restrict__ deg, uint32_t V,
                             const uint32_t* __restrict__ bits, float init, float* x) {
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < V;
       v += (uint64_t)gridDim.x * blockDim.x) {
    float val = 0.f;
    if ((bits[v >> 5] >> (v & 31)) & 1u) {
      const uint32_t dg = deg[v];
      val = dg > 0 ? init / static_cast<float>(dg) : init;
    }
    x[v] = val;
  }
}

__global__ void k_set_seed_bits(const uint32_t* __restrict__ seeds, uint32_t n, uint32_t* bits) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    atomicOr(bits + (seeds[i] >> 5), 1u << (seeds[i] & 31));
}

// Seed-set PPR, one query (algo::trustrank with the seeds given, pull-only).
int seedset_impl(plato_graph* g, const uint32_t* seeds_ext, uint32_t n, const plato_ppr_opts* o,
                 float* d_out, cudaStream_t st, plato_run_stats* stats) {
  PLATO_TRY(check_rank_opts(o->iteration, o->damping));
  const uint32_t V = g->info.vertices;
  if (n == 0) return set_error(PLATO_EINVAL, "seedset ppr: empty seed set");
  const std::vector<uint32_t>* to_int = nullptr;
  PLATO_TRY(host_to_internal(g, &to_int, st));
  std::vector<uint32_t> s;
  s.reserve(n);
  for (uint32_t i = 0; i < n; ++i) {
    if (seeds_ext[i] >= V) return set_error(PLATO_EINVAL, "seedset ppr: seed out of range");
    s.push_back(to_int ? (*to_int)[seeds_ext[i]] : seeds_ext[i]);
  }
  std::sort(s.begin(), s.end());
  s.erase(std::unique(s.begin(), s.end()), s.end());
  PLATO_TRY(ensure_ws(g, st));
  rank_workspace* ws = g->rank_ws;
  PLATO_TRY(ws->seed_bits.alloc((V + 31) / 32));
  PLATO_TRY(ws->seed_list.alloc(s.size()));
  PLATO_CUDA_TRY(cudaMemsetAsync(ws->seed_bits.p, 0, ((V + 31) / 32) * sizeof(uint32_t), st));
  PLATO_CUDA_TRY(cudaMemcpyAsync(ws->seed_list.p, s.data(), s.size() * sizeof(uint32_t),
                                 cudaMemcpyHostToDevice, st));
  k_set_seed_bits<<<grid_for(s.size(), 256), 256, 0, st>>>(ws->seed_list.p, static_cast<uint32_t>(s.size()),
                                                           ws->seed_bits.p);
  PLATO_LAUNCHED("k_set_seed_bits");
  const float init = static_cast<float>(1.0 / static_cast<double>(s.size()));
  k_init_seeds<<<grid_for(V, 256), 256, 0, st>>>(g->out_deg.p, V, ws->seed_bits.p, init, ws->x[0].p);
  PLATO_LAUNCHED("k_init_seeds");
  const float d = static_cast<float>(o->damping);
  const teleport_seeds tele{ws->seed_bits.p,
                            static_cast<float>((1.0 - o->damping) / static_cast<double>(s.size()))};
  int cur = 0;
  uint32_t epochs = 0;
  double delta = 0.0;
  PLATO_TRY(run_pull_epochs(g, tele, d, o->iteration, 0, o->eps, 1.0, st, &cur, &epochs, &delta));
  PLATO_TRY(scatter_to_external_f32(g, ws->x[cur].p, d_out, st));
  if (stats) {
    *stats = plato_run_stats{};
    stats->iterations = epochs;
    stats->pull_iterations = epochs;
    stats->delta = delta;
  }
  return PLATO_OK;
}

// weighted_pagerank.hpp:104-109: ranks 1, gathered state 1 / v_weight_sum.
__global__ void k_init_weighted(const float* __restrict__ wsum, uint32_t V, float* r, float* x) {
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < V;
       v += (uint64_t)gridDim.x * blockDim.x) {
    r[v] = 1.0f;
    x[v] = 1.0f / wsum[v];
  }
}

// algo::weighted_pagerank (weighted_pagerank.hpp:60-149) into d_out (caller
// ids, the reference's units).  Epochs are the pull epochs of PageRank with
// the edge weights multiplied into the gathers; with eps > 0 the delta is read
// back after each non-final epoch and a small one jumps to the last epoch
// (:131-137).
int wpagerank_impl(plato_graph* g, const plato_pagerank_opts* o, float* d_out, cudaStream_t st,
                   plato_run_stats* stats) {
  if (!g->weighted)
    return set_error(PLATO_EINVAL, "plato_weighted_pagerank: the graph has no edge weights "
                                   "(create it with plato_graph_create_weighted)");
  if (!(o->damping >= 0.0 && o->damping <= 1.0)) return set_error(PLATO_EINVAL, "damping must be in [0, 1]");
  rank_workspace* ws = g->rank_ws;
  const uint32_t V = g->info.vertices;
  PLATO_TRY(ws->r[0].alloc(V));
  PLATO_TRY(ws->r[1].alloc(V));
  k_init_weighted<<<grid_for(V, 256), 256, 0, st>>>(g->out_wsum.p, V, ws->r[0].p, ws->x[0].p);
  PLATO_LAUNCHED("k_init_weighted");
  const float base = static_cast<float>(1.0 - o->damping), d = static_cast<float>(o->damping);
  const uint32_t nparts = static_cast<uint32_t>(partial_count(g));
  int cur = 0;
  uint32_t epochs = 0;
  double delta = 0.0;
  for (uint32_t epoch = 0; epoch < o->iteration; ++epoch) {
    const bool last = epoch + 1 == o->iteration;
    const wrank_update upd{ws->r[cur].p, ws->r[cur ^ 1].p, ws->x[cur ^ 1].p, g->out_wsum.p, base, d,
                           last ? 1 : 0};
    PLATO_TRY((pull_epoch_with<wrank_update, true>(g, ws->x[cur].p, upd, g->in_w.p, st)));
    cur ^= 1;
    ++epochs;
    if (last) break;
    if (o->eps > 0.0) {
      PLATO_TRY(read_delta(g, nparts, st, &delta));
      if (delta < o->eps) epoch = o->iteration - 2;  // the next epoch is the last
    }
  }
  PLATO_TRY(scatter_to_external_f32(g, ws->r[cur].p, d_out, st));
  if (stats) {
    *stats = plato_run_stats{};
    stats->iterations = epochs;
    stats->pull_iterations = epochs;
    stats->delta = delta;
  }
  return PLATO_OK;
}

// Host-buffer wrapper: run into a device staging buffer, copy to `host`.
template <class F>
int with_host_output(plato_graph* g, float* host, F&& run) {
  cudaStream_t st = g->stream;
  PLATO_TRY(ensure_ws(g, st));
  dbuf<float>& out = g->rank_ws->out_stage;  // kept on the graph: no allocation per call
  PLATO_TRY(out.alloc(g->info.vertices));
  PLATO_TRY(run(out.p, st));
  PLATO_CUDA_TRY(cudaMemcpyAsync(host, out.p, g->info.vertices * sizeof(float),
                                 cudaMemcpyDeviceToHost, st));
  PLATO_CUDA_TRY(cudaStreamSynchronize(st));
  return PLATO_OK;
}

}  // namespace

// 1D partitions (partition.cu): the workspace of a partition's rows, and one
// PageRank pull epoch over them gathering the replicated state x_gather
// (global ids) and updating the partition's slice (x_old -> xn); the sum of
// the epoch's delta partials (normalised units) goes to *d_partial_sum.
int partition_prepare(plato_graph* g, cudaStream_t st) { return ensure_ws(g, st); }

int pull_epoch_partition(plato_graph* g, const float* x_gather, const float* x_old, float* xn, float tele,
                         float d, bool final_epoch, cudaStream_t st, double* d_partial_sum) {
  PLATO_TRY(ensure_ws(g, st));
  const rank_update<teleport_uniform> upd{x_old, xn, g->out_deg.p, teleport_uniform{tele}, d,
                                          final_epoch ? 1 : 0};
  PLATO_TRY((pull_epoch_with<rank_update<teleport_uniform>, false>(g, x_gather, upd, nullptr, st)));
  if (d_partial_sum) {
    k_sum_partials<<<1, 1024, 0, st>>>(g->rank_ws->partials.p, static_cast<uint32_t>(partial_count(g)),
                                       d_partial_sum);
    PLATO_LAUNCHED("k_sum_partials");
  }
  return PLATO_OK;
}

// The same epoch with the next state stored into every replica: xn is the
// local slice, peers[k] the slices of the other replicas (peer memory).
// `mode` (device, or null): the epoch kind decided on the device (0 normal,
// 1 final, 2 done, as k_epoch_control); d_partial_sum (or null) receives the
// epoch's delta partials summed (normalised units).
int pull_epoch_partition_bcast(plato_graph* g, const float* x_gather, const float* x_old, float* xn,
                               float* const* peers, uint32_t npeers, float tele, float d, bool final_epoch,
                               const int* mode, cudaStream_t st, double* d_partial_sum) {
  if (npeers > kMaxPartitionPeers) return set_error(PLATO_EINVAL, "partition: more than 8 partitions");
  PLATO_TRY(ensure_ws(g, st));
  bcast_rank_update upd{};
  upd.u = rank_update<teleport_uniform>{x_old, xn, g->out_deg.p, teleport_uniform{tele}, d, final_epoch ? 1 : 0,
                                        mode};
  for (uint32_t k = 0; k < npeers; ++k) upd.peers[k] = peers[k];
  upd.npeers = npeers;
  PLATO_TRY((pull_epoch_with<bcast_rank_update, false>(g, x_gather, upd, nullptr, st)));
  if (d_partial_sum) {
    k_sum_partials<<<1, 1024, 0, st>>>(g->rank_ws->partials.p, static_cast<uint32_t>(partial_count(g)),
                                       d_partial_sum);
    PLATO_LAUNCHED("k_sum_partials");
  }
  return PLATO_OK;
}

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

extern "C" int plato_seedset_ppr(plato_graph* g, const plato_vid_t* seeds, uint32_t n,
                                 const plato_ppr_opts* opts, float* ranks, plato_run_stats* stats) {
  if (!g || !seeds || !opts || !ranks) return set_error(PLATO_EINVAL, "plato_seedset_ppr: null argument");
  std::lock_guard<std::mutex> lock(g->mu);
  PLATO_CUDA_TRY(cudaSetDevice(g->device));
  return with_host_output(g, ranks, [&](float* d_out, cudaStream_t st) {
    return seedset_impl(g, seeds, n, opts, d_out, st, stats);
  });
}

extern "C" int plato_weighted_pagerank(plato_graph* g, const plato_pagerank_opts* opts, float* ranks,
                                       plato_run_stats* stats) {
  if (!g || !opts || !ranks) return set_error(PLATO_EINVAL, "plato_weighted_pagerank: null argument");
  std::lock_guard<std::mutex> lock(g->mu);
  PLATO_CUDA_TRY(cudaSetDevice(g->device));
  return with_host_output(g, ranks, [&](float* d_out, cudaStream_t st) {
    return wpagerank_impl(g, opts, d_out, st, stats);
  });
}
