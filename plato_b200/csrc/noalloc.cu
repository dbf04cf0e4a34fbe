// PageRank over a caller-owned device CSC that allocates no memory.
//
// Some callers cannot let a library call cudaMalloc: a host application that
// hands all of HBM to its own pooling allocator and forbids foreign
// allocations, a plugin that runs under a strict per-process memory budget,
// or a latency-critical loop that cannot afford the implicit device-wide
// synchronisation an allocation may cause.  For them this entry point keeps
// every temporary of the PageRank pull (the second rank buffer, the merge-path
// tile table, per-warp carries and the delta partials) in one fixed-size
// array that lives in the library's own device image, so the caller only
// passes its graph and its output buffer.
//
// The array (kNoAllocScratchBytes) is held by every GPU that loads the
// library until the process exits.  All calls share it and it keeps the
// previous call's contents; everything a call reads from it is written by
// the same call first (the epoch-control words by a launch at the start of
// the call), so no clearing is needed.  Calls whose work overlaps on the GPU
// (two streams, two host threads) race on it: serialise them.
//
// With eps > 0 the early exit of pagerank.hpp:137-139 is decided on the
// device (k_epoch_control after each epoch, as the main path does): every
// epoch is enqueued, those after the last one return at once, and a last
// launch moves the result into d_ranks when it ended in the scratch buffer.
#include <cstdint>
#include <mutex>

#include "common.cuh"
#include "pull_binned.cuh"
#include "pull_merge.cuh"
#include "pull_warp.cuh"

namespace plato_b200 {
namespace {

constexpr size_t kNoAllocScratchBytes = PLATO_NOALLOC_SCRATCH_BYTES;
constexpr int kNoAllocIPT = 7;
using na_cfg = pull_warp_cfg<kNoAllocIPT>;
using na_update = rank_update<teleport_uniform>;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mu;
void* g_scratch_addr[kMaxDevices] = {};
uint32_t g_sms[kMaxDevices] = {};
uint32_t g_hub_cap[kMaxDevices] = {};

// Once per device, with that device current: the scratch array's device
// address (the host-side symbol is only a stand-in), the SM count and the
// shared-memory opt-in of the pull kernel.
int setup_device(int dev) {
  std::lock_guard<std::mutex> lock(g_setup_mu);
  if (g_scratch_addr[dev]) return PLATO_OK;
  void* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess || p == nullptr)
    return set_error(PLATO_ECUDA, std::string("no-alloc scratch: cudaGetSymbolAddress failed: ") +
                                      cudaGetErrorString(e));
  int sms = 0, optin = 0;
  PLATO_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  PLATO_CUDA_TRY(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  cudaFuncAttributes fa{};
  PLATO_CUDA_TRY(cudaFuncGetAttributes(&fa, k_pull_warp<kNoAllocIPT, na_update>));
  const size_t dyn = static_cast<size_t>(optin) - fa.sharedSizeBytes;
  if (dyn <= na_cfg::kSlices + 64) return set_error(PLATO_ECUDA, "no-alloc pagerank: shared memory too small");
  PLATO_CUDA_TRY(cudaFuncSetAttribute(k_pull_warp<kNoAllocIPT, na_update>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      static_cast<int>(dyn)));
  g_sms[dev] = static_cast<uint32_t>(sms);
  g_hub_cap[dev] = static_cast<uint32_t>((dyn - na_cfg::kSlices - 16) / 4 / 32 * 32);
  g_scratch_addr[dev] = p;
  return PLATO_OK;
}

__global__ void k_na_merge_tiles(const uint64_t* __restrict__ off, uint32_t V, uint64_t E,
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

__global__ void k_na_init(const uint32_t* __restrict__ deg, uint32_t V, float* x) {
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < V;
       v += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t dg = deg[v];
    x[v] = static_cast<float>(dg > 0 ? 1.0 / (static_cast<double>(V) * dg) : 1.0 / V);
  }
}

// ctrl = {epoch kind (0 normal, 1 final, 2 done), epochs run}; see k_epoch_control.
__global__ void k_na_ctrl_init(int* ctrl, uint32_t iteration, double* delta) {
  ctrl[0] = iteration == 1 ? 1 : 0;
  ctrl[1] = 0;
  delta[0] = 0.0;
}

// After the epochs of an eps > 0 call: the state ended in buf[ran & 1]; copy
// it to d_ranks (buf[0]) when it is the scratch buffer.
__global__ void k_na_finish(const int* __restrict__ ctrl, const float* __restrict__ x2,
                            float* __restrict__ out, uint32_t V) {
  if ((ctrl[1] & 1) == 0) return;
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < V;
       v += (uint64_t)gridDim.x * blockDim.x)
    out[v] = x2[v];
}

size_t align256(size_t n) { return (n + 255) / 256 * 256; }

bool aligned(const void* p, uintptr_t a) { return (reinterpret_cast<uintptr_t>(p) & (a - 1)) == 0; }

}  // namespace
}  // namespace plato_b200

using namespace plato_b200;

extern "C" int plato_pagerank_csc_noalloc(uint32_t vertices, uint64_t edges,
                                          const uint64_t* d_in_offsets, const uint32_t* d_in_adj,
                                          const uint32_t* d_out_degree,
                                          const plato_pagerank_opts* opts, float* d_ranks,
                                          void* stream, plato_run_stats* stats) {
  if (!d_in_offsets || !d_out_degree || !opts || !d_ranks || (edges > 0 && !d_in_adj))
    return set_error(PLATO_EINVAL, "plato_pagerank_csc_noalloc: null argument");
  if (vertices == 0) return set_error(PLATO_EINVAL, "plato_pagerank_csc_noalloc: zero vertices");
  if (opts->iteration == 0) return set_error(PLATO_EINVAL, "iteration must be >= 1");
  if (!(opts->damping >= 0.0 && opts->damping <= 1.0))
    return set_error(PLATO_EINVAL, "damping must be in [0, 1]");
  // d_ranks doubles as the first state buffer, which the pull kernel reads
  // with 16-byte vector loads; the other arrays need their natural alignment.
  if (!aligned(d_ranks, 16) || !aligned(d_in_offsets, 8) || !aligned(d_out_degree, 4) ||
      (d_in_adj && !aligned(d_in_adj, 4)))
    return set_error(PLATO_EINVAL,
                     "plato_pagerank_csc_noalloc: d_ranks must be 16-byte aligned, d_in_offsets "
                     "8-byte aligned, d_in_adj and d_out_degree 4-byte aligned");
  int dev = 0;
  PLATO_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) return set_error(PLATO_EINVAL, "device index out of range");
  PLATO_TRY(setup_device(dev));
  const uint32_t sms = g_sms[dev];
  const uint32_t Wr = sms * na_cfg::kWarps;
  const uint64_t W = Wr;
  const uint32_t fix_blocks = (Wr + 255) / 256;
  const uint32_t nparts = sms + fix_blocks;
  // scratch layout: x2 [V] | trow [T+1] | tedge [T+1] | carry [W] | head [W] |
  //                 partials [nparts] + delta | ctrl [2]
  const uint64_t items = na_cfg::kItems;
  const uint64_t T = (static_cast<uint64_t>(vertices) + edges + items - 1) / items;
  const size_t need = align256(4ull * vertices) + align256(4ull * (T + 1)) + align256(8ull * (T + 1)) +
                      2 * align256(4ull * W) + align256(8ull * (nparts + 1)) + align256(2 * sizeof(int));
  if (need > kNoAllocScratchBytes || T >= 0xFFFFFFFFull)
    return set_error(PLATO_EINVAL,
                     "plato_pagerank_csc_noalloc: graph needs " + std::to_string(need) +
                         " bytes of scratch, more than the fixed " +
                         std::to_string(kNoAllocScratchBytes) + " (PLATO_NOALLOC_SCRATCH_BYTES)");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  unsigned char* base = static_cast<unsigned char*>(g_scratch_addr[dev]);
  size_t o = 0;
  float* x2 = reinterpret_cast<float*>(base + o);
  o += align256(4ull * vertices);
  uint32_t* trow = reinterpret_cast<uint32_t*>(base + o);
  o += align256(4ull * (T + 1));
  uint64_t* tedge = reinterpret_cast<uint64_t*>(base + o);
  o += align256(8ull * (T + 1));
  float* carry = reinterpret_cast<float*>(base + o);
  o += align256(4ull * W);
  float* head = reinterpret_cast<float*>(base + o);
  o += align256(4ull * W);
  double* partials = reinterpret_cast<double*>(base + o);
  double* delta_dev = partials + nparts;
  o += align256(8ull * (nparts + 1));
  int* ctrl = reinterpret_cast<int*>(base + o);

  k_na_merge_tiles<<<grid_for(T + 1, 256), 256, 0, st>>>(d_in_offsets, vertices, edges,
                                                         static_cast<uint32_t>(items),
                                                         static_cast<uint32_t>(T), trow, tedge);
  PLATO_LAUNCHED("k_na_merge_tiles");
  float* buf[2] = {d_ranks, x2};
  k_na_init<<<grid_for(vertices, 256), 256, 0, st>>>(d_out_degree, vertices, buf[0]);
  PLATO_LAUNCHED("k_na_init");
  const float d = static_cast<float>(opts->damping);
  const teleport_uniform tele{static_cast<float>((1.0 - opts->damping) / vertices)};
  const uint32_t H = std::min<uint32_t>(vertices, g_hub_cap[dev]);
  const bool device_exit = opts->eps > 0.0;
  if (device_exit) {
    k_na_ctrl_init<<<1, 1, 0, st>>>(ctrl, opts->iteration, delta_dev);
    PLATO_LAUNCHED("k_na_ctrl_init");
  }
  int cur = 0;
  for (uint32_t epoch = 0; epoch < opts->iteration; ++epoch) {
    const bool final_epoch = !device_exit && (epoch == opts->iteration - 1);
    na_update upd{buf[cur], buf[cur ^ 1], d_out_degree, tele, d, final_epoch ? 1 : 0,
                  device_exit ? ctrl : nullptr};
    pull_warp_args a{trow, tedge, static_cast<uint32_t>(T), edges, d_in_offsets, d_in_adj,
                     buf[cur], H, carry, head, partials};
    k_pull_warp<kNoAllocIPT, na_update><<<sms, 1024, na_cfg::smem_bytes(H), st>>>(a, upd);
    PLATO_LAUNCHED("k_pull_warp (no-alloc)");
    a.partials = partials + sms;
    k_pull_warp_fixup<na_update><<<fix_blocks, 256, 0, st>>>(a, Wr, upd);
    PLATO_LAUNCHED("k_pull_warp_fixup (no-alloc)");
    if (device_exit) {
      // delta in the reference's units (its ranks sum to ~V)
      k_epoch_control<<<1, 1024, 0, st>>>(partials, nparts, ctrl, delta_dev,
                                          static_cast<double>(vertices), opts->eps, opts->iteration);
      PLATO_LAUNCHED("k_epoch_control (no-alloc)");
    }
    cur ^= 1;
  }
  if (device_exit) {
    k_na_finish<<<grid_for(vertices, 256), 256, 0, st>>>(ctrl, x2, d_ranks, vertices);
    PLATO_LAUNCHED("k_na_finish");
  } else if (buf[cur] != d_ranks) {
    PLATO_CUDA_TRY(cudaMemcpyAsync(d_ranks, buf[cur], 4ull * vertices, cudaMemcpyDeviceToDevice, st));
  }
  if (stats) {
    *stats = plato_run_stats{};
    uint32_t epochs = opts->iteration;
    double delta = 0.0;
    if (device_exit) {  // the epoch count and last delta are on the device: wait for them
      int h_ctrl[2] = {0, 0};
      PLATO_CUDA_TRY(cudaMemcpyAsync(h_ctrl, ctrl, sizeof(h_ctrl), cudaMemcpyDeviceToHost, st));
      PLATO_CUDA_TRY(cudaMemcpyAsync(&delta, delta_dev, sizeof(double), cudaMemcpyDeviceToHost, st));
      PLATO_CUDA_TRY(cudaStreamSynchronize(st));
      epochs = static_cast<uint32_t>(h_ctrl[1]);
    }
    stats->iterations = epochs;
    stats->pull_iterations = epochs;
    stats->delta = delta;
  }
  return PLATO_OK;
}
