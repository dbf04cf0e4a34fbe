// Pull-gather ceiling: what the memory system gives this graph's gather
// stream when nothing else is in the way.
//
// The long-bin pull kernel (k_pull_long) reads the CSC source ids of rows
// with in-degree > 64 as a coalesced stream and gathers one 4-byte rank per
// id at a random place in the rank vector.  These diagnostic kernels run the
// same id stream (the first row past in-degree 64 bounds it) with the
// row bookkeeping, the update and the delta taken out, so their times bound
// what any kernel with this access pattern can reach on this GPU:
//   0 ids      the id stream alone (16-byte coalesced loads): the DRAM part
//   1 gather4  ids + gathers, 4 ranks in flight per lane (k_pull_long's depth)
//   2 gather8  8 in flight per lane
//   3 gather16 16 in flight per lane
//   4 hot      as gather8 with every id folded into the first 64K ranks
//              (256 KB, L1-resident; fewer on graphs below 64K vertices):
//              the L1 rate for divergent gathers
//   5 coalesced as gather8 with the gather at the edge's own position mod V:
//              the same instruction mix with coalesced gathers
// Each launch runs a fixed grid (8 CTAs x 256 threads per SM; the 16-deep
// variant fits 4 CTAs at a time at its register count) over 32*M-edge
// chunks; a checksum per CTA keeps the loads live.  No counterpart in the
// reference; it serves the roofline analysis only.
#include <algorithm>
#include <string>
#include <vector>

#include "batch_engine.hpp"
#include "graph.cuh"

namespace plato_b200 {
namespace {

// Two timing events, destroyed on every way out.
struct event_pair {
  cudaEvent_t a = nullptr, b = nullptr;
  event_pair() = default;
  event_pair(const event_pair&) = delete;
  event_pair& operator=(const event_pair&) = delete;
  ~event_pair() {
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
  }
};

__global__ void __launch_bounds__(256, 8) k_ceil_ids(const uint32_t* __restrict__ adj, uint64_t n,
                                                     uint32_t* __restrict__ sink) {
  const uint64_t n4 = n / 4;
  const uint4* a4 = reinterpret_cast<const uint4*>(adj);
  uint32_t acc = 0;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n4; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint4 v = __ldcs(a4 + i);
    acc ^= v.x ^ v.y ^ v.z ^ v.w;
  }
  acc = __reduce_xor_sync(0xffffffffu, acc);
  if ((threadIdx.x & 31) == 0) atomicXor(sink + blockIdx.x, acc);
}

// kMode: 0 random gathers, 1 ids folded into the first 64K ranks, 2 gather at
// the edge position mod V.
template <int M, int kMode>
__global__ void __launch_bounds__(256, (M <= 8 ? 8 : 4)) k_ceil_gather(const uint32_t* __restrict__ adj, uint64_t n,
                                                        const float* __restrict__ x, uint32_t V,
                                                        uint32_t hot_mask, float* __restrict__ sink) {
  const unsigned lane = threadIdx.x & 31;
  const uint64_t nwarps = (uint64_t)gridDim.x * (blockDim.x >> 5);
  const uint64_t chunk = 32ull * M;
  float s = 0.f;
  for (uint64_t c = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5; c * chunk < n; c += nwarps) {
    const uint64_t b = c * chunk + lane;
    uint32_t id[M];
#pragma unroll
    for (int k = 0; k < M; ++k) {
      const uint64_t e = b + 32ull * k;
      uint32_t v = e < n ? __ldcs(adj + e) : 0u;
      if (kMode == 1) v &= hot_mask;  // hot_mask + 1 <= V
      if (kMode == 2) v = static_cast<uint32_t>(e % V);
      id[k] = v;
    }
#pragma unroll
    for (int k = 0; k < M; ++k) s += (b + 32ull * k < n) ? __ldg(x + id[k]) : 0.f;
  }
  s = warp_sum(s);
  if (lane == 0) atomicAdd(sink + blockIdx.x, s);
}

// Batched-pull row gathers: a group of GL lanes takes 4 consecutive edges of
// the whole CSC id stream at a time and gathers the source's kt-float row
// (kt = 4 GL, a float4 per lane, 4 rows in flight per lane, every row
// through one L2 range policy: rows below keep_rows at normal priority, the
// rest evict-first, as k_batch_pull).
// kMode: 0 the edge's own source row, 1 row = edge position mod V (sequential
// rows: the streaming rate of the same instruction mix), 2 source folded into
// the first hot_rows rows (an L2-resident block).
template <int GL, int kMode>
__global__ void __launch_bounds__(256, 5) k_ceil_rows(const uint32_t* __restrict__ adj, uint64_t n,
                                                      const float* __restrict__ X, uint32_t V,
                                                      uint32_t hot_rows, uint32_t keep_rows,
                                                      float* __restrict__ sink) {
  constexpr int KT = GL * 4;
  uint64_t pol;
  {
    const uint64_t bytes = static_cast<uint64_t>(V) * KT * 4;
    const uint32_t total = static_cast<uint32_t>(bytes < 0xFFFFFF00ull ? bytes : 0xFFFFFF00ull);
    const uint64_t keep = static_cast<uint64_t>(keep_rows) * KT * 4;
    const uint32_t primary = static_cast<uint32_t>(keep < total ? keep : total);
    asm("createpolicy.range.global.L2::evict_normal.L2::evict_first.b64 %0, [%1], %2, %3;"
        : "=l"(pol)
        : "l"(X), "r"(primary), "r"(total));
  }
  const unsigned lane_g = threadIdx.x % GL;
  const uint64_t groups = (uint64_t)gridDim.x * (blockDim.x / GL);
  float s = 0.f;
  for (uint64_t grp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) / GL; grp * 4 < n; grp += groups) {
    const uint64_t e0 = grp * 4;
    uint32_t row[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const uint64_t e = e0 + u;
      uint32_t v = e < n ? __ldg(adj + e) : 0u;
      if (kMode == 1) v = static_cast<uint32_t>(e % V);
      if (kMode == 2) v %= hot_rows;
      row[u] = v;
    }
    float4 a[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      a[u] = make_float4(0.f, 0.f, 0.f, 0.f);
      if (e0 + u < n)
        asm("ld.global.nc.L2::cache_hint.v4.f32 {%0,%1,%2,%3}, [%4], %5;"
            : "=f"(a[u].x), "=f"(a[u].y), "=f"(a[u].z), "=f"(a[u].w)
            : "l"(X + static_cast<size_t>(row[u]) * KT + 4 * lane_g), "l"(pol));
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) s += (a[u].x + a[u].y) + (a[u].z + a[u].w);
  }
  s = warp_sum(s);
  if ((threadIdx.x & 31) == 0) atomicAdd(sink + blockIdx.x, s);
}

__global__ void k_ceil_fill(float* X, uint64_t n, float v) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    X[i] = v;
}

template <int GL>
void launch_ceil_rows(uint32_t mode, unsigned grid, cudaStream_t st, const uint32_t* adj, uint64_t n,
                      const float* X, uint32_t V, uint32_t hot_rows, uint32_t keep_rows, float* sink) {
  switch (mode) {
    case 0: k_ceil_rows<GL, 0><<<grid, 256, 0, st>>>(adj, n, X, V, hot_rows, keep_rows, sink); break;
    case 1: k_ceil_rows<GL, 1><<<grid, 256, 0, st>>>(adj, n, X, V, hot_rows, keep_rows, sink); break;
    default: k_ceil_rows<GL, 2><<<grid, 256, 0, st>>>(adj, n, X, V, hot_rows, keep_rows, sink); break;
  }
}

}  // namespace
}  // namespace plato_b200

using namespace plato_b200;

extern "C" int plato_diag_pull_ceiling(plato_graph* g, uint32_t mode, uint32_t reps, double* ms_per_launch,
                                       uint64_t* edges, double* checksum) {
  if (!g || !ms_per_launch || mode > 5 || reps == 0)
    return set_error(PLATO_EINVAL, "plato_diag_pull_ceiling: bad argument");
  if (!g->relabeled) return set_error(PLATO_EINVAL, "plato_diag_pull_ceiling: the graph must be relabelled");
  std::lock_guard<std::mutex> lock(g->mu);
  try {
    PLATO_CUDA_TRY(cudaSetDevice(g->device));
    const uint32_t V = g->info.vertices;
    cudaStream_t st = g->stream;
    // rows are numbered by descending in-degree: the long bin is [0, n_long)
    std::vector<uint32_t> deg(V);
    PLATO_CUDA_TRY(cudaMemcpy(deg.data(), g->in_deg.p, 4ull * V, cudaMemcpyDeviceToHost));
    // first row with in-degree <= 64 (the array is non-increasing)
    const uint32_t n_long = static_cast<uint32_t>(
        std::partition_point(deg.begin(), deg.end(), [](uint32_t e) { return e > 64u; }) - deg.begin());
    uint64_t n = 0;
    PLATO_CUDA_TRY(cudaMemcpy(&n, g->in_off.p + n_long, 8, cudaMemcpyDeviceToHost));
    if (edges) *edges = n;
    int sms = 0;
    PLATO_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, g->device));
    const unsigned grid = 8u * static_cast<unsigned>(sms);
    uint32_t hot_mask = 1u << 16;  // a power of two <= min(V, 64K), minus one
    while (hot_mask > V) hot_mask >>= 1;
    hot_mask -= 1;
    dbuf<float> x;
    dbuf<float> sink;
    PLATO_TRY(x.alloc(V));
    PLATO_TRY(sink.alloc(grid));
    std::vector<float> h_x(V, 1.0f / V);
    PLATO_CUDA_TRY(cudaMemcpy(x.p, h_x.data(), 4ull * V, cudaMemcpyHostToDevice));
    PLATO_CUDA_TRY(cudaMemset(sink.p, 0, 4ull * grid));
    auto launch = [&]() {
      switch (mode) {
        case 0: k_ceil_ids<<<grid, 256, 0, st>>>(g->in_adj.p, n, reinterpret_cast<uint32_t*>(sink.p)); break;
        case 1: k_ceil_gather<4, 0><<<grid, 256, 0, st>>>(g->in_adj.p, n, x.p, V, hot_mask, sink.p); break;
        case 2: k_ceil_gather<8, 0><<<grid, 256, 0, st>>>(g->in_adj.p, n, x.p, V, hot_mask, sink.p); break;
        case 3: k_ceil_gather<16, 0><<<grid, 256, 0, st>>>(g->in_adj.p, n, x.p, V, hot_mask, sink.p); break;
        case 4: k_ceil_gather<8, 1><<<grid, 256, 0, st>>>(g->in_adj.p, n, x.p, V, hot_mask, sink.p); break;
        default: k_ceil_gather<8, 2><<<grid, 256, 0, st>>>(g->in_adj.p, n, x.p, V, hot_mask, sink.p); break;
      }
      count_launch();
    };
    for (int w = 0; w < 3; ++w) launch();
    event_pair ev;
    PLATO_CUDA_TRY(cudaEventCreate(&ev.a));
    PLATO_CUDA_TRY(cudaEventCreate(&ev.b));
    cudaEvent_t e0 = ev.a, e1 = ev.b;
    PLATO_CUDA_TRY(cudaEventRecord(e0, st));
    for (uint32_t r = 0; r < reps; ++r) launch();
    PLATO_CUDA_TRY(cudaEventRecord(e1, st));
    PLATO_CUDA_TRY(cudaEventSynchronize(e1));
    float ms = 0.f;
    PLATO_CUDA_TRY(cudaEventElapsedTime(&ms, e0, e1));
    PLATO_CUDA_TRY(cudaGetLastError());
    *ms_per_launch = static_cast<double>(ms) / reps;
    if (checksum) {
      std::vector<float> h(grid);
      PLATO_CUDA_TRY(cudaMemcpy(h.data(), sink.p, 4ull * grid, cudaMemcpyDeviceToHost));
      double cs = 0.0;
      for (float v : h) cs += v;
      *checksum = cs;
    }
  } catch (const std::exception& ex) {
    return set_error(PLATO_ECUDA, std::string("plato_diag_pull_ceiling: ") + ex.what());
  }
  return PLATO_OK;
}

// Batched-pull ceiling: the batched pull's row-gather stream on this graph
// with everything but the loads taken out (modes 0-2 of k_ceil_rows), and
// the real batched iteration (mode 3: k_batch_pull + fixup + delta + column
// states over kt live columns that never converge), at the same tile width.
extern "C" int plato_diag_batch_ceiling(plato_graph* g, uint32_t kt, uint32_t mode, uint32_t reps,
                                        double* ms_per_launch, uint64_t* edges, double* checksum) {
  if (!g || !ms_per_launch || mode > 3 || reps == 0 || !(kt == 16 || kt == 32 || kt == 64 || kt == 128))
    return set_error(PLATO_EINVAL, "plato_diag_batch_ceiling: bad argument");
  std::lock_guard<std::mutex> lock(g->mu);
  try {
    PLATO_CUDA_TRY(cudaSetDevice(g->device));
    const uint32_t V = g->info.vertices;
    const uint64_t n = g->stored_edges;
    cudaStream_t st = g->stream;
    if (edges) *edges = n;
    event_pair ev;
    PLATO_CUDA_TRY(cudaEventCreate(&ev.a));
    PLATO_CUDA_TRY(cudaEventCreate(&ev.b));
    cudaEvent_t e0 = ev.a, e1 = ev.b;
    float ms = 0.f;
    double cs = 0.0;
    if (mode == 3) {
      batch_engine eng(g);
      PLATO_TRY(eng.init(kt, kt, 1u << 30, 0.85, 0.0, st));
      std::vector<uint32_t> cols(kt);
      std::vector<std::vector<uint32_t>> seeds(kt);
      for (uint32_t q = 0; q < kt; ++q) {
        cols[q] = q;
        seeds[q].push_back(static_cast<uint32_t>((static_cast<uint64_t>(q) * 2654435761u) % V));
      }
      PLATO_TRY(eng.admit(cols, seeds));
      uint32_t live = 0;
      PLATO_TRY(eng.step(&live, nullptr, 3));
      PLATO_CUDA_TRY(cudaEventRecord(e0, st));
      PLATO_TRY(eng.step(&live, nullptr, reps));  // reps iterations back to back, then one poll
      PLATO_CUDA_TRY(cudaEventRecord(e1, st));
      PLATO_CUDA_TRY(cudaEventSynchronize(e1));
      PLATO_CUDA_TRY(cudaEventElapsedTime(&ms, e0, e1));
      cs = live;
    } else {
      int sms = 0;
      PLATO_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, g->device));
      const unsigned grid = 5u * static_cast<unsigned>(sms);
      // an L2-resident block of rows for mode 2: 16 MB
      const uint32_t hot_rows = std::max(1u, std::min(V, static_cast<uint32_t>((16u << 20) / (4u * kt))));
      // the batched pull's L2 split: rows within half of L2 keep normal priority
      int l2 = 0;
      PLATO_CUDA_TRY(cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, g->device));
      const uint32_t keep_rows = static_cast<uint32_t>(
          std::min<uint64_t>(V, static_cast<uint64_t>(l2) / 2 / (4ull * kt)));
      dbuf<float> X, sink;
      PLATO_TRY(X.alloc(static_cast<size_t>(V) * kt));
      PLATO_TRY(sink.alloc(grid));
      // every row sums to 1, so a launch's checksum is its edge count
      k_ceil_fill<<<grid_for(static_cast<uint64_t>(V) * kt, 256), 256, 0, st>>>(X.p, static_cast<uint64_t>(V) * kt,
                                                                            1.0f / static_cast<float>(kt));
      count_launch();
      PLATO_CUDA_TRY(cudaMemsetAsync(sink.p, 0, 4ull * grid, st));
      auto launch = [&]() {
        switch (kt) {
          case 16: launch_ceil_rows<4>(mode, grid, st, g->in_adj.p, n, X.p, V, hot_rows, keep_rows, sink.p); break;
          case 32: launch_ceil_rows<8>(mode, grid, st, g->in_adj.p, n, X.p, V, hot_rows, keep_rows, sink.p); break;
          case 64: launch_ceil_rows<16>(mode, grid, st, g->in_adj.p, n, X.p, V, hot_rows, keep_rows, sink.p); break;
          default: launch_ceil_rows<32>(mode, grid, st, g->in_adj.p, n, X.p, V, hot_rows, keep_rows, sink.p); break;
        }
        count_launch();
      };
      for (int w = 0; w < 3; ++w) launch();
      PLATO_CUDA_TRY(cudaEventRecord(e0, st));
      for (uint32_t r = 0; r < reps; ++r) launch();
      PLATO_CUDA_TRY(cudaEventRecord(e1, st));
      PLATO_CUDA_TRY(cudaEventSynchronize(e1));
      PLATO_CUDA_TRY(cudaEventElapsedTime(&ms, e0, e1));
      std::vector<float> h(grid);
      PLATO_CUDA_TRY(cudaMemcpy(h.data(), sink.p, 4ull * grid, cudaMemcpyDeviceToHost));
      for (float v : h) cs += v;
    }
    PLATO_CUDA_TRY(cudaGetLastError());
    *ms_per_launch = static_cast<double>(ms) / reps;
    if (checksum) *checksum = cs;
  } catch (const std::exception& ex) {
    return set_error(PLATO_ECUDA, std::string("plato_diag_batch_ceiling: ") + ex.what());
  }
  return PLATO_OK;
}
