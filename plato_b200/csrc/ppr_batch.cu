// Batched multi-source PPR: host driver (batch_engine) and plato_ppr_batch.
#include <algorithm>
#include <new>
#include <set>

#include <cub/device/device_scan.cuh>

#include "batch.cuh"
#include "batch_engine.hpp"
#include "profile.cuh"
#include "topk.cuh"

namespace plato_b200 {
namespace {

constexpr int kKernelsPerIteration = 4;
constexpr uint32_t kBatchItersPerPoll = 8;

bool kt_supported(uint32_t kt) { return kt == 8 || kt == 16 || kt == 32 || kt == 64 || kt == 128; }
// Every lane gathers a float4 (4 columns, 16 bytes) per edge; kt/4 lanes
// share one edge's kt-float row, so a warp gathers 128/kt edges per load.
int group_lanes(uint32_t kt) { return static_cast<int>(kt / 4); }

template <int GL, int VEC>
int launch_pass(const batch_pass& p, uint32_t T, uint32_t fix_blocks, uint32_t ntiles,
                cudaStream_t st) {
  k_batch_pull<GL, VEC><<<dim3(T, ntiles), 256, 0, st>>>(p);
  PLATO_LAUNCHED("k_batch_pull");
  k_batch_fixup<GL, VEC><<<dim3(fix_blocks, ntiles), 256, 0, st>>>(p);
  PLATO_LAUNCHED("k_batch_fixup");
  return PLATO_OK;
}

// X[tile(q)][v][q % kt] = 0 for the listed columns.  Neighbouring threads
// take neighbouring listed columns of one row, so a run of consecutive
// columns (a whole batch) is written with coalesced stores.
__global__ void k_zero_columns(float* X, uint32_t V, uint32_t kt, const uint32_t* cols,
                               uint32_t ncols) {
  const uint64_t total = static_cast<uint64_t>(V) * ncols;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t q = cols[i % ncols];
    const uint32_t v = static_cast<uint32_t>(i / ncols);
    X[(static_cast<size_t>(q / kt) * V + v) * kt + q % kt] = 0.f;
  }
}

// Seed initial values (trustrank.hpp:197-206): (1/|S|) / deg, or 1/|S| when deg == 0.
__global__ void k_seed_init(float* X, uint32_t V, uint32_t kt, const uint32_t* sv,
                            const uint32_t* sq, const float* init, uint32_t n,
                            const uint32_t* __restrict__ deg) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint32_t v = sv[i], q = sq[i];
    const uint32_t dg = deg[v];
    X[(static_cast<size_t>(q / kt) * V + v) * kt + q % kt] = dg > 0 ? init[i] / static_cast<float>(dg) : init[i];
  }
}

__global__ void k_set_states(uint8_t* state, uint32_t* iters, const uint32_t* cols, uint32_t n,
                             uint8_t value) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    state[cols[i]] = value;
    iters[cols[i]] = 0;
  }
}

// out[i][caller id] = rank of column cols[i] (from the buffer holding its result).
__global__ void k_gather_columns(const float* X0, const float* X1, const uint8_t* parity,
                                 uint32_t V, uint32_t kt, const uint32_t* cols, uint32_t ncols,
                                 const uint32_t* to_ext, float* out) {
  const uint64_t total = static_cast<uint64_t>(V) * ncols;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t ci = static_cast<uint32_t>(i / V), v = static_cast<uint32_t>(i % V);
    const uint32_t q = cols[ci];
    const float* X = parity[q] ? X1 : X0;
    const float val = X[(static_cast<size_t>(q / kt) * V + v) * kt + q % kt];
    out[static_cast<size_t>(ci) * V + (to_ext ? to_ext[v] : v)] = val;
  }
}

template <typename T>
int upload(dbuf<T>& d, const std::vector<T>& h, cudaStream_t st) {
  PLATO_TRY(d.alloc(std::max<size_t>(h.size(), 1)));
  if (!h.empty())
    PLATO_CUDA_TRY(cudaMemcpyAsync(d.p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, st));
  return PLATO_OK;
}

// Seed index on the device: cnt[v] = number of (v, column) seed entries.
__global__ void k_seed_count(const uint32_t* __restrict__ ev, uint32_t n, uint32_t* cnt) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    atomicAdd(&cnt[ev[i]], 1u);
}

// Entry i goes to slot off[v] + rank (entries arrive sorted by (v, column),
// rank = position among the entries of v), so the layout is deterministic.
__global__ void k_seed_scatter(const uint32_t* __restrict__ ev, const uint32_t* __restrict__ eq,
                               const uint32_t* __restrict__ er, const float* __restrict__ et,
                               uint32_t n, const uint32_t* __restrict__ off, uint32_t* col,
                               float* tele) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint32_t slot = off[ev[i]] + er[i];
    col[slot] = eq[i];
    tele[slot] = et[i];
  }
}

}  // namespace

batch_engine::~batch_engine() {
  for (auto& e : exec_)
    if (e) cudaGraphExecDestroy(e);
  if (h_counters_) cudaFreeHost(h_counters_);
}

void destroy_batch_engine(batch_engine* e) { delete e; }

int batch_engine::init(uint32_t K, uint32_t kt, uint32_t max_iterations, double damping,
                       double eps, cudaStream_t st) {
  if (K == 0) return set_error(PLATO_EINVAL, "batched ppr: no queries");
  if (!kt_supported(kt)) return set_error(PLATO_EINVAL, "batched ppr: k_tile must be 8/16/32/64/128");
  if (max_iterations == 0) return set_error(PLATO_EINVAL, "batched ppr: max_iterations must be >= 1");
  if (!(damping >= 0.0 && damping <= 1.0)) return set_error(PLATO_EINVAL, "damping must be in [0, 1]");
  // the two iteration graphs bake in the buffers and the scalar options: a
  // repeat of the previous configuration with no buffer moved reuses them
  const bool same_opts = exec_[0] && exec_[1] && st == st_ && K == K_ && kt == kt_ &&
                         max_iterations == max_iterations_ && damping == damping_ && eps == eps_;
  const auto buffers = [this]() {
    return std::vector<const void*>{X_[0].p, X_[1].p, state_.p, parity_.p, iters_.p, delta_.p,
                                    tcarry_.p, thead_.p, partials_.p, seed_off_.p, seed_col_.p,
                                    seed_tele_.p, counters_.p, retired_.p, h_counters_};
  };
  const std::vector<const void*> before = buffers();
  st_ = st;
  K_ = K;
  kt_ = kt;
  Kp_ = (K + kt - 1) / kt * kt;
  ntiles_ = Kp_ / kt;
  max_iterations_ = max_iterations;
  damping_ = damping;
  eps_ = eps;
  const uint32_t V = g_->info.vertices;
  if (hot_l2_bytes_ == 0) {
    int l2 = 0;
    PLATO_CUDA_TRY(cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, g_->device));
    hot_l2_bytes_ = static_cast<uint64_t>(l2) / 2;
  }
  const merge_tiles* mt = nullptr;
  PLATO_TRY(ensure_pull_tiles(g_, batch_tile_items(static_cast<int>(kt)), st_, &mt));
  const uint32_t T = mt->count;
  const uint32_t NG = 256 / group_lanes(kt);
  rows_ = T + (T + NG - 1) / NG;
  const size_t cells = static_cast<size_t>(Kp_) * V;
  PLATO_TRY(X_[0].alloc(cells));
  PLATO_TRY(X_[1].alloc(cells));
  PLATO_TRY(state_.alloc(Kp_));
  PLATO_TRY(parity_.alloc(Kp_));
  PLATO_TRY(iters_.alloc(Kp_));
  PLATO_TRY(delta_.alloc(Kp_));
  PLATO_TRY(tcarry_.alloc(static_cast<size_t>(ntiles_) * T * kt));
  PLATO_TRY(thead_.alloc(static_cast<size_t>(ntiles_) * T * kt));
  PLATO_TRY(partials_.alloc(static_cast<size_t>(ntiles_) * rows_ * kt));
  PLATO_TRY(seed_off_.alloc(static_cast<size_t>(V) + 1));
  PLATO_TRY(seed_cnt_.alloc(static_cast<size_t>(V)));
  if (scan_bytes_ == 0) {
    PLATO_CUDA_TRY(cub::DeviceScan::InclusiveSum(nullptr, scan_bytes_, seed_cnt_.p, seed_off_.p + 1,
                                                 static_cast<int>(V), st_));
    PLATO_TRY(scan_tmp_.alloc(std::max<size_t>(scan_bytes_, 1)));
  }
  PLATO_TRY(seed_col_.alloc(static_cast<size_t>(Kp_) * 64));
  PLATO_TRY(seed_tele_.alloc(static_cast<size_t>(Kp_) * 64));
  PLATO_TRY(counters_.alloc(2));
  PLATO_TRY(retired_.alloc(Kp_));
  PLATO_CUDA_TRY(cudaMemsetAsync(state_.p, COL_FREE, Kp_, st_));
  PLATO_CUDA_TRY(cudaMemsetAsync(parity_.p, 0, Kp_, st_));
  PLATO_CUDA_TRY(cudaMemsetAsync(iters_.p, 0, Kp_ * sizeof(uint32_t), st_));
  PLATO_CUDA_TRY(cudaMemsetAsync(seed_off_.p, 0, (static_cast<size_t>(V) + 1) * sizeof(uint32_t), st_));
  if (!h_counters_ || h_counters_cap_ < 2 + Kp_) {
    if (h_counters_) cudaFreeHost(h_counters_);
    h_counters_ = nullptr;
    PLATO_CUDA_TRY(cudaMallocHost(reinterpret_cast<void**>(&h_counters_), (2 + Kp_) * sizeof(uint32_t)));
    h_counters_cap_ = 2 + Kp_;
  }
  col_seeds_.assign(Kp_, {});
  cur_ = 0;
  if (same_opts && buffers() == before) return PLATO_OK;
  return capture();
}

int batch_engine::launch_iteration(int parity) {
  const uint32_t V = g_->info.vertices;
  const merge_tiles& mt = g_->tiles.at(batch_tile_items(static_cast<int>(kt_)));
  batch_pass p{};
  p.trow = mt.row.p;
  p.tedge = mt.edge.p;
  p.T = mt.count;
  p.V = V;
  p.rows = rows_;
  p.off = g_->in_off.p;
  p.adj = g_->in_adj.p;
  p.deg = g_->out_deg.p;
  p.X = X_[parity].p;
  p.Xn = X_[parity ^ 1].p;
  p.state = state_.p;
  p.seeds = seed_index_view{seed_off_.p, seed_col_.p, seed_tele_.p};
  p.col_base = 0;
  p.d = static_cast<float>(damping_);
  p.tcarry = tcarry_.p;
  p.thead = thead_.p;
  p.partials = partials_.p;
  const uint32_t T = mt.count;
  // the live count restarts every iteration (k_batch_delta clears it); the
  // retired list accumulates over the iterations of one step() and is reset
  // and read there
  const uint32_t fix_blocks = rows_ - T;
  // rows whose gathers keep normal L2 priority: half of L2 for one column tile
  // (a launch's CTAs run tile by tile, blockIdx.x fastest)
  p.hot_rows = static_cast<uint32_t>(std::min<uint64_t>(V, hot_l2_bytes_ / (4ull * kt_)));
  switch (kt_) {
    case 8: PLATO_TRY((launch_pass<2, 4>(p, T, fix_blocks, ntiles_, st_))); break;
    case 16: PLATO_TRY((launch_pass<4, 4>(p, T, fix_blocks, ntiles_, st_))); break;
    case 32: PLATO_TRY((launch_pass<8, 4>(p, T, fix_blocks, ntiles_, st_))); break;
    case 64: PLATO_TRY((launch_pass<16, 4>(p, T, fix_blocks, ntiles_, st_))); break;
    default: PLATO_TRY((launch_pass<32, 4>(p, T, fix_blocks, ntiles_, st_))); break;
  }
  k_batch_delta<<<dim3(kt_, ntiles_), 256, 0, st_>>>(partials_.p, rows_, kt_, state_.p, delta_.p,
                                                     counters_.p);
  PLATO_LAUNCHED("k_batch_delta");
  k_batch_states<<<grid_for(Kp_, 256, 64), 256, 0, st_>>>(
      Kp_, state_.p, iters_.p, parity_.p, delta_.p, max_iterations_, eps_, parity ^ 1,
      counters_.p, retired_.p, counters_.p + 1);
  PLATO_LAUNCHED("k_batch_states");
  return PLATO_OK;
}

int batch_engine::capture() {
  for (int parity = 0; parity < 2; ++parity) {
    if (exec_[parity]) {
      cudaGraphExecDestroy(exec_[parity]);
      exec_[parity] = nullptr;
    }
    cudaGraph_t graph = nullptr;
    PLATO_CUDA_TRY(cudaStreamBeginCapture(st_, cudaStreamCaptureModeThreadLocal));
    const int s = launch_iteration(parity);
    const cudaError_t e = cudaStreamEndCapture(st_, &graph);
    if (s != PLATO_OK) {
      if (graph) cudaGraphDestroy(graph);
      return s;
    }
    PLATO_CUDA_TRY(e);
    const cudaError_t ie = cudaGraphInstantiate(&exec_[parity], graph, 0);
    cudaGraphDestroy(graph);
    PLATO_CUDA_TRY(ie);
  }
  return PLATO_OK;
}

// Seed index (teleport entries by vertex) of every live column.  The host
// lists the entries (a few per column), sorted by (vertex, column); the
// device counts them per vertex, scans the counts into offsets and scatters
// the entries, so no V-sized array crosses PCIe or is touched on the host.
int batch_engine::rebuild_seed_index() {
  const uint32_t V = g_->info.vertices;
  struct ent {
    uint32_t v, q;
    float tele;
  };
  std::vector<ent> ents;
  for (uint32_t q = 0; q < Kp_; ++q) {
    const auto& s = col_seeds_[q];
    if (s.empty()) continue;
    const float tele = static_cast<float>((1.0 - damping_) / static_cast<double>(s.size()));
    for (uint32_t v : s) ents.push_back({v, q, tele});
  }
  std::sort(ents.begin(), ents.end(), [](const ent& a, const ent& b) {
    return a.v != b.v ? a.v < b.v : a.q < b.q;
  });
  const size_t n = ents.size();
  std::vector<uint32_t> hv(n), hq(n), hr(n);
  std::vector<float> ht(n);
  for (size_t i = 0; i < n; ++i) {
    hv[i] = ents[i].v;
    hq[i] = ents[i].q;
    ht[i] = ents[i].tele;
    hr[i] = (i > 0 && ents[i - 1].v == ents[i].v) ? hr[i - 1] + 1 : 0;
  }
  bool recapture = false;
  if (n > seed_col_.n) {
    PLATO_TRY(seed_col_.alloc(n * 2));
    PLATO_TRY(seed_tele_.alloc(n * 2));
    recapture = true;
  }
  PLATO_TRY(upload(ent_v_, hv, st_));
  PLATO_TRY(upload(ent_q_, hq, st_));
  PLATO_TRY(upload(ent_r_, hr, st_));
  PLATO_TRY(upload(ent_t_, ht, st_));
  PLATO_CUDA_TRY(cudaMemsetAsync(seed_cnt_.p, 0, static_cast<size_t>(V) * sizeof(uint32_t), st_));
  PLATO_CUDA_TRY(cudaMemsetAsync(seed_off_.p, 0, sizeof(uint32_t), st_));
  const uint32_t n32 = static_cast<uint32_t>(n);
  if (n32) {
    k_seed_count<<<grid_for(n32, 256), 256, 0, st_>>>(ent_v_.p, n32, seed_cnt_.p);
    PLATO_LAUNCHED("k_seed_count");
  }
  size_t tmp = scan_bytes_;
  PLATO_CUDA_TRY(cub::DeviceScan::InclusiveSum(scan_tmp_.p, tmp, seed_cnt_.p, seed_off_.p + 1,
                                               static_cast<int>(V), st_));
  count_launch();
  if (n32) {
    k_seed_scatter<<<grid_for(n32, 256), 256, 0, st_>>>(ent_v_.p, ent_q_.p, ent_r_.p, ent_t_.p, n32,
                                                        seed_off_.p, seed_col_.p, seed_tele_.p);
    PLATO_LAUNCHED("k_seed_scatter");
  }
  PLATO_CUDA_TRY(cudaStreamSynchronize(st_));  // host vectors go out of scope
  if (recapture) PLATO_TRY(capture());
  return PLATO_OK;
}

int batch_engine::admit(const std::vector<uint32_t>& cols,
                        const std::vector<std::vector<uint32_t>>& seeds) {
  const uint32_t V = g_->info.vertices;
  if (cols.size() != seeds.size()) return set_error(PLATO_EINVAL, "admit: size mismatch");
  if (cols.empty()) return PLATO_OK;
  const std::vector<uint32_t>* to_int = nullptr;
  PLATO_TRY(host_to_internal(g_, &to_int, st_));
  std::vector<uint32_t> sv, sq;
  std::vector<float> init;
  for (size_t i = 0; i < cols.size(); ++i) {
    const uint32_t q = cols[i];
    if (q >= K_) return set_error(PLATO_EINVAL, "admit: column out of range");
    std::set<uint32_t> uniq;
    for (uint32_t v : seeds[i]) {
      if (v >= V) return set_error(PLATO_EINVAL, "ppr: seed vertex out of range");
      uniq.insert(to_int ? (*to_int)[v] : v);
    }
    if (uniq.empty()) return set_error(PLATO_EINVAL, "ppr: empty seed set");
    col_seeds_[q].assign(uniq.begin(), uniq.end());
    const float iv = static_cast<float>(1.0 / static_cast<double>(uniq.size()));
    for (uint32_t v : uniq) {
      sv.push_back(v);
      sq.push_back(q);
      init.push_back(iv);
    }
  }
  PLATO_TRY(upload(adm_cols_, cols, st_));
  PLATO_TRY(upload(adm_sv_, sv, st_));
  PLATO_TRY(upload(adm_sq_, sq, st_));
  PLATO_TRY(upload(adm_init_, init, st_));
  const uint32_t n = static_cast<uint32_t>(cols.size());
  k_zero_columns<<<grid_for(static_cast<uint64_t>(V) * n, 256), 256, 0, st_>>>(X_[cur_].p, V, kt_,
                                                                               adm_cols_.p, n);
  PLATO_LAUNCHED("k_zero_columns");
  k_seed_init<<<grid_for(sv.size(), 256), 256, 0, st_>>>(X_[cur_].p, V, kt_, adm_sv_.p, adm_sq_.p,
                                                         adm_init_.p, static_cast<uint32_t>(sv.size()),
                                                         g_->out_deg.p);
  PLATO_LAUNCHED("k_seed_init");
  k_set_states<<<grid_for(n, 256), 256, 0, st_>>>(state_.p, iters_.p, adm_cols_.p, n,
                                                  max_iterations_ == 1 ? COL_FINAL : COL_LIVE);
  PLATO_LAUNCHED("k_set_states");
  return rebuild_seed_index();  // synchronises before the temporaries go
}

int batch_engine::step(uint32_t* live, std::vector<uint32_t>* retired, uint32_t n) {
  PLATO_CUDA_TRY(cudaMemsetAsync(counters_.p + 1, 0, sizeof(uint32_t), st_));
  for (uint32_t i = 0; i < std::max(n, 1u); ++i) {
    {
      prof_scope ps("batch_iteration", st_);
      PLATO_CUDA_TRY(cudaGraphLaunch(exec_[cur_], st_));
    }
    count_launch(kKernelsPerIteration);
    cur_ ^= 1;
  }
  // one read of the counters and the retired list per poll
  PLATO_CUDA_TRY(cudaMemcpyAsync(h_counters_, counters_.p, 2 * sizeof(uint32_t), cudaMemcpyDeviceToHost, st_));
  PLATO_CUDA_TRY(cudaMemcpyAsync(h_counters_ + 2, retired_.p, Kp_ * sizeof(uint32_t), cudaMemcpyDeviceToHost, st_));
  PLATO_CUDA_TRY(cudaStreamSynchronize(st_));
  *live = h_counters_[0];
  const uint32_t nret = std::min(h_counters_[1], Kp_);
  if (retired) {
    retired->assign(h_counters_ + 2, h_counters_ + 2 + nret);
    std::sort(retired->begin(), retired->end());
  }
  for (uint32_t i = 0; i < nret; ++i) col_seeds_[h_counters_[2 + i]].clear();
  return PLATO_OK;
}

int batch_engine::release(const std::vector<uint32_t>& cols) {
  if (cols.empty()) return PLATO_OK;
  PLATO_TRY(upload(adm_cols_, cols, st_));
  const uint32_t n = static_cast<uint32_t>(cols.size());
  k_set_states<<<grid_for(n, 256), 256, 0, st_>>>(state_.p, iters_.p, adm_cols_.p, n, COL_FREE);
  PLATO_LAUNCHED("k_set_states");
  for (uint32_t q : cols) col_seeds_[q].clear();
  PLATO_CUDA_TRY(cudaStreamSynchronize(st_));
  return PLATO_OK;
}

int batch_engine::iterations(std::vector<uint32_t>* out) {
  out->resize(Kp_);
  PLATO_CUDA_TRY(cudaMemcpyAsync(out->data(), iters_.p, Kp_ * sizeof(uint32_t),
                                 cudaMemcpyDeviceToHost, st_));
  PLATO_CUDA_TRY(cudaStreamSynchronize(st_));
  return PLATO_OK;
}

int batch_engine::ranks(const std::vector<uint32_t>& cols, float* out) {
  const uint32_t V = g_->info.vertices;
  const uint32_t chunk = std::max<uint32_t>(1, std::min<uint32_t>(64, static_cast<uint32_t>(cols.size())));
  dbuf<float> d_out;
  dbuf<uint32_t> d_cols;
  PLATO_TRY(d_out.alloc(static_cast<size_t>(chunk) * V));
  for (size_t c0 = 0; c0 < cols.size(); c0 += chunk) {
    const uint32_t n = static_cast<uint32_t>(std::min<size_t>(chunk, cols.size() - c0));
    std::vector<uint32_t> part(cols.begin() + c0, cols.begin() + c0 + n);
    PLATO_TRY(upload(d_cols, part, st_));
    k_gather_columns<<<grid_for(static_cast<uint64_t>(V) * n, 256), 256, 0, st_>>>(
        X_[0].p, X_[1].p, parity_.p, V, kt_, d_cols.p, n, g_->relabeled ? g_->to_ext.p : nullptr,
        d_out.p);
    PLATO_LAUNCHED("k_gather_columns");
    PLATO_CUDA_TRY(cudaMemcpyAsync(out + c0 * V, d_out.p, static_cast<size_t>(n) * V * sizeof(float),
                                   cudaMemcpyDeviceToHost, st_));
    PLATO_CUDA_TRY(cudaStreamSynchronize(st_));
  }
  return PLATO_OK;
}

int batch_engine::topk(const std::vector<uint32_t>& cols, uint32_t k, uint32_t* ids, float* vals) {
  if (cols.empty() || k == 0) return PLATO_OK;
  if (k > kTopkMax) return set_error(PLATO_EINVAL, "topk must be <= 1024");
  const uint32_t n = static_cast<uint32_t>(cols.size());
  dbuf<uint32_t>& d_cols = tk_cols_;
  dbuf<uint32_t>& hist = tk_hist_;
  dbuf<uint32_t>& d_ids = tk_ids_;
  dbuf<uint32_t>& undone = tk_undone_;
  dbuf<unsigned long long>& cand = tk_cand_;
  dbuf<float>& d_vals = tk_vals_;
  PLATO_TRY(upload(d_cols, cols, st_));
  PLATO_TRY(tk_state_.alloc(static_cast<size_t>(n) * sizeof(topk_col)));
  PLATO_TRY(hist.alloc(static_cast<size_t>(n) * 256));
  PLATO_TRY(cand.alloc(static_cast<size_t>(n) * kCandCap));
  PLATO_TRY(d_ids.alloc(static_cast<size_t>(n) * k));
  PLATO_TRY(d_vals.alloc(static_cast<size_t>(n) * k));
  PLATO_TRY(undone.alloc(1));
  PLATO_CUDA_TRY(cudaMemsetAsync(hist.p, 0, static_cast<size_t>(n) * 256 * sizeof(uint32_t), st_));
  topk_job j{};
  j.buf[0] = X_[0].p;
  j.buf[1] = X_[1].p;
  j.parity = parity_.p;
  j.cols = d_cols.p;
  j.n = n;
  j.V = g_->info.vertices;
  j.kt = kt_;
  j.to_ext = g_->relabeled ? g_->to_ext.p : nullptr;
  j.st = reinterpret_cast<topk_col*>(tk_state_.p);
  j.hist = hist.p;
  j.cand = cand.p;
  k_topk_init<<<grid_for(n, 256), 256, 0, st_>>>(j, k);
  PLATO_LAUNCHED("k_topk_init");
  const unsigned blocks = 148 * 4;
  // a column is usually bounded after two or three digits: the first two
  // passes are enqueued without a host check (a finished column's lanes skip
  // the next pass), later ones stop as soon as every column is bounded
  constexpr int kUncheckedPasses = 2;
  for (int pass = 0; pass < 8; ++pass) {
    for (uint32_t c0 = 0; c0 < n; c0 += 32) {
      k_topk_hist<<<blocks, 256, 0, st_>>>(j, c0);
      PLATO_LAUNCHED("k_topk_hist");
    }
    PLATO_CUDA_TRY(cudaMemsetAsync(undone.p, 0, sizeof(uint32_t), st_));
    k_topk_pick<<<grid_for(n, 256), 256, 0, st_>>>(j, k, undone.p);
    PLATO_LAUNCHED("k_topk_pick");
    if (pass + 1 < kUncheckedPasses) continue;
    uint32_t h_undone = 0;
    PLATO_CUDA_TRY(cudaMemcpyAsync(&h_undone, undone.p, sizeof(uint32_t), cudaMemcpyDeviceToHost, st_));
    PLATO_CUDA_TRY(cudaStreamSynchronize(st_));
    if (h_undone == 0) break;
  }
  for (uint32_t c0 = 0; c0 < n; c0 += 32) {
    k_topk_collect<<<blocks, 256, 0, st_>>>(j, c0);
    PLATO_LAUNCHED("k_topk_collect");
  }
  k_topk_sort<<<n, 1024, 0, st_>>>(j, k, d_ids.p, d_vals.p);
  PLATO_LAUNCHED("k_topk_sort");
  PLATO_CUDA_TRY(cudaMemcpyAsync(ids, d_ids.p, static_cast<size_t>(n) * k * sizeof(uint32_t),
                                 cudaMemcpyDeviceToHost, st_));
  PLATO_CUDA_TRY(cudaMemcpyAsync(vals, d_vals.p, static_cast<size_t>(n) * k * sizeof(float),
                                 cudaMemcpyDeviceToHost, st_));
  PLATO_CUDA_TRY(cudaStreamSynchronize(st_));
  return PLATO_OK;
}

// Picks the column-tile width for a batch of K columns: every candidate runs
// full iterations over a probe of min(K rounded up, 512) live columns (all
// its tiles in one launch, as in the real batch), best of two trials of three
// iterations; the cost is scaled to K columns.  Cached per graph and per
// power-of-two bucket of K.
int batch_autotune(plato_graph* g, uint32_t K, cudaStream_t st, uint32_t* kt_out) {
  uint32_t bucket = 8;
  while (bucket < K && bucket < 1024) bucket <<= 1;
  auto it = g->batch_tuned.find(bucket);
  if (it != g->batch_tuned.end()) {
    *kt_out = it->second;
    return PLATO_OK;
  }
  const uint32_t cands[] = {8, 16, 32, 64, 128};
  const uint32_t V = g->info.vertices;
  double best = 1e300;
  uint32_t best_kt = 32;
  cudaEvent_t e0, e1;
  PLATO_CUDA_TRY(cudaEventCreate(&e0));
  PLATO_CUDA_TRY(cudaEventCreate(&e1));
  int rc = PLATO_OK;
  for (uint32_t kt : cands) {
    if (kt > bucket) break;
    // probe columns: up to 512, at most 8 GiB of state (two V x probe matrices)
    const uint64_t fit = (8ull << 30) / (8ull * std::max(V, 1u));
    const uint32_t cap = static_cast<uint32_t>(std::min<uint64_t>(512, std::max<uint64_t>(fit, kt)));
    const uint32_t probe = std::max(kt, std::min((bucket + kt - 1) / kt * kt, cap / kt * kt));
    batch_engine eng(g);
    rc = eng.init(probe, kt, 1u << 30, 0.85, 0.0, st);
    if (rc != PLATO_OK) break;
    std::vector<uint32_t> cols(probe);
    std::vector<std::vector<uint32_t>> seeds(probe);
    for (uint32_t q = 0; q < probe; ++q) {
      cols[q] = q;
      seeds[q].push_back(static_cast<uint32_t>((static_cast<uint64_t>(q) * 2654435761u) % V));
    }
    rc = eng.admit(cols, seeds);
    if (rc != PLATO_OK) break;
    uint32_t live = 0;
    rc = eng.step(&live, nullptr);
    if (rc != PLATO_OK) break;
    float best_ms = 1e30f;
    for (int trial = 0; trial < 2 && rc == PLATO_OK; ++trial) {
      const int reps = 3;
      if (cudaEventRecord(e0, st) != cudaSuccess) rc = set_error(PLATO_ECUDA, "autotune: event record failed");
      for (int r = 0; r < reps && rc == PLATO_OK; ++r) rc = eng.step(&live, nullptr);
      if (rc != PLATO_OK) break;
      float ms = 0.f;
      if (cudaEventRecord(e1, st) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
          cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess)
        rc = set_error(PLATO_ECUDA, "autotune: event timing failed");
      best_ms = std::min(best_ms, ms / reps);
    }
    if (rc != PLATO_OK) break;
    const double cost = best_ms * (static_cast<double>(K) / probe);  // per K-column iteration
    if (cost < best) {
      best = cost;
      best_kt = kt;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc != PLATO_OK) return rc;
  g->batch_tuned[bucket] = best_kt;
  *kt_out = best_kt;
  return PLATO_OK;
}

}  // namespace plato_b200

using namespace plato_b200;

extern "C" int plato_ppr_batch_k_tile(plato_graph* g, uint32_t K, uint32_t* k_tile) {
  if (!g || !k_tile) return set_error(PLATO_EINVAL, "plato_ppr_batch_k_tile: null argument");
  if (K == 0) return set_error(PLATO_EINVAL, "plato_ppr_batch_k_tile: K must be >= 1");
  std::lock_guard<std::mutex> lock(g->mu);
  PLATO_CUDA_TRY(cudaSetDevice(g->device));
  return batch_autotune(g, K, g->stream, k_tile);
}

extern "C" int plato_ppr_batch(plato_graph* g, uint32_t K, const uint64_t* seed_offsets,
                               const plato_vid_t* seeds, const plato_ppr_batch_opts* opts,
                               float* ranks, plato_vid_t* topk_ids, float* topk_vals,
                               uint32_t* iterations) {
  if (!g || !seed_offsets || !seeds || !opts)
    return set_error(PLATO_EINVAL, "plato_ppr_batch: null argument");
  if (K == 0) return set_error(PLATO_EINVAL, "plato_ppr_batch: K must be >= 1");
  if (opts->topk > kTopkMax) return set_error(PLATO_EINVAL, "plato_ppr_batch: topk must be <= 1024");
  if (opts->topk && (!topk_ids || !topk_vals))
    return set_error(PLATO_EINVAL, "plato_ppr_batch: topk output buffers missing");
  std::vector<std::vector<uint32_t>> sets(K);
  std::vector<uint32_t> cols(K);
  for (uint32_t q = 0; q < K; ++q) {
    if (seed_offsets[q + 1] < seed_offsets[q])
      return set_error(PLATO_EINVAL, "plato_ppr_batch: seed_offsets must be non-decreasing");
    sets[q].assign(seeds + seed_offsets[q], seeds + seed_offsets[q + 1]);
    cols[q] = q;
  }
  std::lock_guard<std::mutex> lock(g->mu);
  PLATO_CUDA_TRY(cudaSetDevice(g->device));
  cudaStream_t st = g->stream;
  uint32_t kt = opts->k_tile;
  if (kt == 0) PLATO_TRY(batch_autotune(g, K, st, &kt));
  // the engine (and its V x K buffers) stays on the graph between calls, so a
  // stream of batches pays for allocation and graph capture once
  if (!g->batch_cache) {
    g->batch_cache = new (std::nothrow) batch_engine(g);
    if (!g->batch_cache) return set_error(PLATO_ENOMEM, "plato_ppr_batch: host allocation failed");
  }
  batch_engine& eng = *g->batch_cache;
  PLATO_TRY(eng.init(K, kt, opts->max_iterations, opts->damping, opts->eps, st));
  PLATO_TRY(eng.admit(cols, sets));
  uint32_t live = K;
  // several iterations per host poll: the device state machine idles the
  // finished columns, and a busy host cannot stall the device between polls
  while (live > 0) PLATO_TRY(eng.step(&live, nullptr, kBatchItersPerPoll));
  if (iterations) {
    std::vector<uint32_t> it;
    PLATO_TRY(eng.iterations(&it));
    std::copy(it.begin(), it.begin() + K, iterations);
  }
  if (opts->topk) PLATO_TRY(eng.topk(cols, opts->topk, topk_ids, topk_vals));
  if (ranks) PLATO_TRY(eng.ranks(cols, ranks));
  return PLATO_OK;
}
