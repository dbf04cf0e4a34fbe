// 1D partitioned PageRank: the graph split by destination over several GPUs.
//
// Follows the reference's multi-partition layout for the pull engine
// (create_dcsc_seqs_from_path, plato/graph/structure.hpp:471-555, with
// sequence_balanced_by_destination_t, plato/graph/partition/sequence.hpp:43-75):
// every partition owns a set of destination vertices with all of their
// in-edges, and the rank state the pull gathers is replicated, refreshed
// after every epoch by one exchange (the reference sends each pull message to
// the owner through MPI, message_passing.hpp:88-144; here each partition
// writes its own slice of the state and an all-gather over NCCL assembles the
// next state on every GPU).
//
// Layout, B200 first: vertices are ranked by descending in-degree (ties by
// caller id), the engine's own order, and position i goes to partition
// i % P at local row i / P.  Every partition then holds the same number of
// rows (n = ceil(V / P), the last rows of some partitions are padding), its
// rows are still sorted by in-degree (so each runs the degree-binned pull
// kernels unchanged), the edges are spread evenly (every partition takes one
// of each P consecutive degree ranks), and the replicated state is one
// P x n array in which partition r's rows sit at [r n, (r + 1) n): the
// all-gather is in place with equal counts.  Global internal id of a vertex
// = r n + local row; the CSC of a partition keeps its sources as global ids.
//
// Padding rows have no edges; their state is held at the value an edgeless
// vertex keeps, (1 - d) / V, so they add nothing to any delta and nothing
// gathers them.
//
// Fused exchange (plato_partition_p2p_*), the B200 form of the same epoch:
// every partition keeps two replicas of the whole state (ping-pong) and one
// flag word per partition in its own HBM, and maps the other partitions'
// replicas and flags (CUDA IPC between processes, plain pointers within
// one).  The pull kernels store each new row value into all replicas at
// once (peer stores over NVLink), so the exchange travels with the epoch's
// own stores instead of following it; a one-thread kernel then publishes
// the epoch (system-scope fence, release store of the epoch number into
// this partition's flag on every GPU), and the next epoch starts with a
// one-thread kernel that waits (acquire loads, bounded by a timeout) until
// every partition has published.  Two replicas and a full barrier per epoch
// mean no partition overwrites a replica another is still reading.  No
// collective and no host round trip per epoch.
#include <omp.h>
#include <parallel/algorithm>

#include <algorithm>
#include <new>
#include <vector>

#include "graph.cuh"
#include "pull_merge.cuh"

struct plato_partition {
  plato_graph* g = nullptr;  // this partition's rows (internal; never handed out)
  uint32_t rank = 0, world = 0, n = 0, real = 0, V = 0;
  std::vector<uint32_t> gid;  // caller id -> global internal id
  // fused exchange: local replicas and flags, the peers' mapped ones
  float* s[2] = {nullptr, nullptr};
  // one synchronisation block per partition: [world] u32 epoch flags at byte
  // 0, [2][world] double deltas at byte 64 (peers write both)
  unsigned char* sync = nullptr;
  uint32_t* flags = nullptr;
  double* deltas = nullptr;
  int* ctrl = nullptr;        // [4]: wait status (1 = gave up), epoch mode, epochs run, eps mode
  double* d_part = nullptr;   // this partition's delta of the last epoch
  float* peer_s[2][8] = {};
  uint32_t* peer_flags[8] = {};
  double* peer_deltas[8] = {};
  double eps = 0.0;
  uint32_t iterations = 0;
  void* ipc_base[8][3] = {};  // mappings opened from IPC handles (closed on destroy)
  bool p2p_ready = false;
  uint64_t timeout_ns = 5000000000ull;
  ~plato_partition() {
    for (auto& peer : ipc_base)
      for (void* b : peer)
        if (b) cudaIpcCloseMemHandle(b);
    for (float* b : s)
      if (b) cudaFree(b);
    if (sync) cudaFree(sync);
    if (ctrl) cudaFree(ctrl);
    if (d_part) cudaFree(d_part);
    delete g;
  }
};

namespace plato_b200 {

// defined in rank.cu
int partition_prepare(plato_graph* g, cudaStream_t st);
int pull_epoch_partition(plato_graph* g, const float* x_gather, const float* x_old, float* xn, float tele,
                         float d, bool final_epoch, cudaStream_t st, double* d_partial_sum);
int pull_epoch_partition_bcast(plato_graph* g, const float* x_gather, const float* x_old, float* xn,
                               float* const* peers, uint32_t npeers, float tele, float d, bool final_epoch,
                               const int* mode, cudaStream_t st, double* d_partial_sum);

namespace {

struct layout {
  uint32_t V = 0, world = 0, n = 0;
  std::vector<uint32_t> gid;  // caller id -> global internal id
  std::vector<uint32_t> indeg, outdeg;  // by caller id (undirected: both = degree)
};

int make_layout(const plato_graph_info* info, const uint32_t* src, const uint32_t* dst, uint32_t world,
                layout* L) {
  const uint32_t V = info->vertices;
  const uint64_t m = info->edges;
  L->V = V;
  L->world = world;
  L->n = static_cast<uint32_t>((static_cast<uint64_t>(V) + world - 1) / world);
  L->indeg.assign(V, 0);
  L->outdeg.assign(V, 0);
  for (uint64_t i = 0; i < m; ++i) {
    if (src[i] >= V || dst[i] >= V) return set_error(PLATO_EINVAL, "partition: vertex id >= vertices");
    ++L->indeg[dst[i]];
    ++L->outdeg[src[i]];
    if (!info->is_directed) {
      ++L->indeg[src[i]];
      ++L->outdeg[dst[i]];
    }
  }
  std::vector<uint32_t> order(V);
  for (uint32_t v = 0; v < V; ++v) order[v] = v;
  const std::vector<uint32_t>& deg = L->indeg;
  __gnu_parallel::sort(order.begin(), order.end(),
                       [&deg](uint32_t a, uint32_t b) { return deg[a] != deg[b] ? deg[a] > deg[b] : a < b; });
  L->gid.assign(V, 0);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < static_cast<int64_t>(V); ++i)
    L->gid[order[i]] = static_cast<uint32_t>((i % world) * L->n + i / world);
  return PLATO_OK;
}

__global__ void k_part_init(const uint32_t* __restrict__ deg, uint32_t rows, uint32_t real, uint32_t V,
                            float ghost, float* x) {
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < rows;
       v += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t dg = deg[v];
    x[v] = v >= real ? ghost : static_cast<float>(dg > 0 ? 1.0 / (static_cast<double>(V) * dg) : 1.0 / V);
  }
}

// Peer pointers by value (kernel parameters): at most 8 partitions.
struct peer_list {
  float* p[8];
};
struct flag_list {
  uint32_t* p[8];
};

// x0 of this partition's rows (as k_part_init) into every replica.
__global__ void k_part_init_bcast(const uint32_t* __restrict__ deg, uint32_t rows, uint32_t real, uint32_t V,
                                  float ghost, float* x, peer_list peers, uint32_t npeers) {
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < rows;
       v += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t dg = deg[v];
    const float xv = v >= real ? ghost : static_cast<float>(dg > 0 ? 1.0 / (static_cast<double>(V) * dg) : 1.0 / V);
    x[v] = xv;
    for (uint32_t k = 0; k < npeers; ++k) peers.p[k][v] = xv;
  }
}

struct delta_list {
  double* p[8];
};

// Publishes `value` as this partition's epoch count on every GPU: with
// deltas, first this partition's delta of the epoch (*d_part) into slot
// [slot][rank] of every GPU's deltas; then the earlier kernels' stores (local
// and peer) are made visible at system scope, then each flag gets a release
// store.
__global__ void k_p2p_signal(flag_list flags, delta_list deltas, uint32_t world, uint32_t rank, uint32_t value,
                             const double* d_part, uint32_t slot) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  if (d_part) {
    const double dv = *d_part;
    for (uint32_t q = 0; q < world; ++q) deltas.p[q][slot * world + rank] = dv;
  }
  __threadfence_system();
  for (uint32_t q = 0; q < world; ++q)
    asm volatile("st.release.sys.global.u32 [%0], %1;" ::"l"(flags.p[q] + rank), "r"(value) : "memory");
}

// The eps exit of pagerank.hpp:137-139 for the fused exchange, run by every
// partition at the start of epoch `epoch` >= 1 once all have published epoch
// - 1: the same rule as k_epoch_control on the delta summed over the
// partitions in rank order (so every partition takes the same decision).
// ctrl[1] = mode of this epoch (0 normal, 1 final, 2 done), ctrl[2] = epochs
// run before it.
__global__ void k_p2p_control(const double* deltas, uint32_t world, uint32_t epoch, int* ctrl, double scale,
                              double eps, uint32_t iteration) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const int mode = ctrl[1];
  if (mode == 2) return;
  const int ran = ctrl[2] + 1;
  ctrl[2] = ran;
  if (mode == 1) {
    ctrl[1] = 2;
    return;
  }
  const double* dv = deltas + ((epoch - 1) & 1u) * world;
  double sum = 0.0;
  for (uint32_t q = 0; q < world; ++q) {
    double v;
    asm volatile("ld.relaxed.sys.global.f64 %0, [%1];" : "=d"(v) : "l"(dv + q) : "memory");
    sum += v;
  }
  const double dlt = sum * scale;
  if ((eps > 0.0 && dlt < eps) || static_cast<uint32_t>(ran) >= iteration - 1) ctrl[1] = 1;
}

// Waits until every partition has published at least `target` in the local
// flags, for at most timeout_ns (the device's global timer); on a timeout it
// sets *status and returns, and every later wait returns at once.
__global__ void k_p2p_wait(const uint32_t* flags, uint32_t world, uint32_t target, int* status,
                           uint64_t timeout_ns) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  if (*(volatile int*)status) return;
  uint64_t t0;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0));
  for (uint32_t q = 0; q < world; ++q) {
    for (uint32_t spin = 0;; ++spin) {
      uint32_t v;
      asm volatile("ld.acquire.sys.global.u32 %0, [%1];" : "=r"(v) : "l"(flags + q) : "memory");
      if (v >= target) break;
      uint64_t t;
      asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
      if (t - t0 > timeout_ns || spin > (1u << 30)) {
        *status = 1;
        __threadfence_system();
        return;
      }
      __nanosleep(256);
    }
  }
}

}  // namespace
}  // namespace plato_b200


using namespace plato_b200;

extern "C" int plato_partition_layout(const plato_graph_info* info, const plato_vid_t* src,
                                      const plato_vid_t* dst, uint32_t world, plato_vid_t* global_ids,
                                      uint32_t* rows_per_partition) {
  if (!info || !global_ids || !rows_per_partition || (info->edges > 0 && (!src || !dst)))
    return set_error(PLATO_EINVAL, "plato_partition_layout: null argument");
  if (info->vertices == 0 || world == 0) return set_error(PLATO_EINVAL, "plato_partition_layout: empty");
  try {
    layout L;
    PLATO_TRY(make_layout(info, src, dst, world, &L));
    std::copy(L.gid.begin(), L.gid.end(), global_ids);
    *rows_per_partition = L.n;
  } catch (const std::bad_alloc&) {
    return set_error(PLATO_ENOMEM, "plato_partition_layout: host allocation failed");
  }
  return PLATO_OK;
}

namespace plato_b200 {
namespace {

int build_partition(const plato_graph_info* info, const plato_vid_t* src, const plato_vid_t* dst, uint32_t rank,
                    uint32_t world, plato_partition* p) {
  layout L;
  PLATO_TRY(make_layout(info, src, dst, world, &L));
  const uint32_t n = L.n;
  p->rank = rank;
  p->world = world;
  p->n = n;
  p->V = L.V;
  p->real = static_cast<uint32_t>((static_cast<uint64_t>(L.V) + world - 1 - rank) / world);
  // local CSC: rows = this partition's vertices, sources as global ids
  std::vector<uint64_t> off(static_cast<size_t>(n) + 1, 0);
  std::vector<uint32_t> odeg(n, 0), ideg(n, 0);
  const uint32_t lo = rank * n;
  for (uint32_t v = 0; v < L.V; ++v) {
    const uint32_t gv = L.gid[v];
    if (gv >= lo && gv < lo + n) {
      odeg[gv - lo] = L.outdeg[v];
      ideg[gv - lo] = L.indeg[v];
    }
  }
  for (uint32_t r = 0; r < n; ++r) off[r + 1] = off[r] + ideg[r];
  std::vector<uint32_t> adj(off[n]);
  std::vector<uint64_t> pos(off.begin(), off.end() - 1);
  const uint64_t m = info->edges;
  for (uint64_t i = 0; i < m; ++i) {
    const uint32_t gs = L.gid[src[i]], gd = L.gid[dst[i]];
    if (gd >= lo && gd < lo + n) adj[pos[gd - lo]++] = gs;
    if (!info->is_directed && gs >= lo && gs < lo + n) adj[pos[gs - lo]++] = gd;
  }
#pragma omp parallel for schedule(dynamic, 1024)
  for (int64_t r = 0; r < static_cast<int64_t>(n); ++r) std::sort(adj.begin() + off[r], adj.begin() + off[r + 1]);
  plato_graph* g = new plato_graph();
  p->g = g;
  PLATO_CUDA_TRY(cudaGetDevice(&g->device));
  g->info.is_directed = 1;
  g->info.vertices = n;
  g->info.edges = off[n];
  g->info.max_v_i = n - 1;
  g->stored_edges = off[n];
  g->relabeled = true;  // rows sorted by descending in-degree: the binned pull plan applies
  PLATO_TRY(g->in_off.alloc(static_cast<size_t>(n) + 1));
  PLATO_TRY(g->in_adj.alloc(std::max<size_t>(adj.size(), 1)));
  PLATO_TRY(g->out_deg.alloc(n));
  PLATO_TRY(g->in_deg.alloc(n));
  PLATO_CUDA_TRY(cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking));
  PLATO_CUDA_TRY(cudaMemcpy(g->in_off.p, off.data(), off.size() * 8, cudaMemcpyHostToDevice));
  if (!adj.empty()) PLATO_CUDA_TRY(cudaMemcpy(g->in_adj.p, adj.data(), adj.size() * 4, cudaMemcpyHostToDevice));
  PLATO_CUDA_TRY(cudaMemcpy(g->out_deg.p, odeg.data(), odeg.size() * 4, cudaMemcpyHostToDevice));
  PLATO_CUDA_TRY(cudaMemcpy(g->in_deg.p, ideg.data(), ideg.size() * 4, cudaMemcpyHostToDevice));
  p->gid = std::move(L.gid);
  PLATO_TRY(partition_prepare(g, g->stream));
  PLATO_CUDA_TRY(cudaStreamSynchronize(g->stream));
  return PLATO_OK;
}

}  // namespace
}  // namespace plato_b200

extern "C" int plato_partition_create(const plato_graph_info* info, const plato_vid_t* src,
                                      const plato_vid_t* dst, uint32_t rank, uint32_t world,
                                      plato_partition** out) {
  if (!info || !out || (info->edges > 0 && (!src || !dst)))
    return set_error(PLATO_EINVAL, "plato_partition_create: null argument");
  *out = nullptr;
  if (info->vertices == 0 || world == 0 || rank >= world)
    return set_error(PLATO_EINVAL, "plato_partition_create: need vertices > 0 and rank < world");
  plato_partition* p = new (std::nothrow) plato_partition();
  if (!p) return set_error(PLATO_ENOMEM, "plato_partition_create: host allocation failed");
  int rc = PLATO_OK;
  try {
    rc = build_partition(info, src, dst, rank, world, p);
  } catch (const std::bad_alloc&) {
    rc = set_error(PLATO_ENOMEM, "plato_partition_create: host allocation failed");
  }
  if (rc != PLATO_OK) {
    delete p;
    return rc;
  }
  *out = p;
  return PLATO_OK;
}

extern "C" int plato_partition_destroy(plato_partition* p) {
  delete p;
  return PLATO_OK;
}

extern "C" int plato_partition_info(const plato_partition* p, uint32_t* vertices, uint32_t* rows,
                                    uint32_t* real_rows, uint64_t* edges) {
  if (!p) return set_error(PLATO_EINVAL, "plato_partition_info: null partition");
  if (vertices) *vertices = p->V;
  if (rows) *rows = p->n;
  if (real_rows) *real_rows = p->real;
  if (edges) *edges = p->g->stored_edges;
  return PLATO_OK;
}

extern "C" int plato_partition_pagerank_init(plato_partition* p, float* d_state, double damping, void* stream) {
  if (!p || !d_state) return set_error(PLATO_EINVAL, "plato_partition_pagerank_init: null argument");
  if (!(damping >= 0.0 && damping <= 1.0)) return set_error(PLATO_EINVAL, "damping must be in [0, 1]");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const float ghost = static_cast<float>((1.0 - damping) / p->V);
  k_part_init<<<grid_for(p->n, 256), 256, 0, st>>>(p->g->out_deg.p, p->n, p->real, p->V, ghost,
                                                   d_state + static_cast<size_t>(p->rank) * p->n);
  PLATO_LAUNCHED("k_part_init");
  return PLATO_OK;
}

extern "C" int plato_partition_pagerank_epoch(plato_partition* p, const float* d_state, float* d_next,
                                              double damping, int final_epoch, double* d_delta, void* stream) {
  if (!p || !d_state || !d_next) return set_error(PLATO_EINVAL, "plato_partition_pagerank_epoch: null argument");
  if (!(damping >= 0.0 && damping <= 1.0)) return set_error(PLATO_EINVAL, "damping must be in [0, 1]");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const size_t base = static_cast<size_t>(p->rank) * p->n;
  return pull_epoch_partition(p->g, d_state, d_state + base, d_next + base,
                              static_cast<float>((1.0 - damping) / p->V), static_cast<float>(damping),
                              final_epoch != 0, st, d_delta);
}

extern "C" int plato_partition_ranks(const plato_partition* p, const float* h_state, float* ranks) {
  if (!p || !h_state || !ranks) return set_error(PLATO_EINVAL, "plato_partition_ranks: null argument");
  const std::vector<uint32_t>& gid = p->gid;
#pragma omp parallel for schedule(static)
  for (int64_t v = 0; v < static_cast<int64_t>(p->V); ++v) ranks[v] = h_state[gid[v]];
  return PLATO_OK;
}

// ---- fused exchange over peer memory -----------------------------------------

namespace {

constexpr size_t kSyncDeltas = 64;  // byte offset of the deltas in the sync block

int p2p_alloc_local(plato_partition* p) {
  if (p->world > 8) return set_error(PLATO_EINVAL, "partition p2p: at most 8 partitions");
  PLATO_CUDA_TRY(cudaSetDevice(p->g->device));
  if (p->s[0]) return PLATO_OK;
  const size_t cells = static_cast<size_t>(p->world) * p->n;
  for (float*& b : p->s) PLATO_CUDA_TRY(cudaMalloc(reinterpret_cast<void**>(&b), cells * sizeof(float)));
  const size_t sync_bytes = kSyncDeltas + 2ull * p->world * sizeof(double);
  PLATO_CUDA_TRY(cudaMalloc(reinterpret_cast<void**>(&p->sync), sync_bytes));
  PLATO_CUDA_TRY(cudaMalloc(reinterpret_cast<void**>(&p->ctrl), 4 * sizeof(int)));
  PLATO_CUDA_TRY(cudaMalloc(reinterpret_cast<void**>(&p->d_part), sizeof(double)));
  PLATO_CUDA_TRY(cudaMemset(p->sync, 0, sync_bytes));
  PLATO_CUDA_TRY(cudaMemset(p->ctrl, 0, 4 * sizeof(int)));
  PLATO_CUDA_TRY(cudaMemset(p->d_part, 0, sizeof(double)));
  p->flags = reinterpret_cast<uint32_t*>(p->sync);
  p->deltas = reinterpret_cast<double*>(p->sync + kSyncDeltas);
  for (int par = 0; par < 2; ++par) p->peer_s[par][p->rank] = p->s[par];
  p->peer_flags[p->rank] = p->flags;
  p->peer_deltas[p->rank] = p->deltas;
  return PLATO_OK;
}

// The other partitions' slices of replica `par` at this partition's rows.
plato_b200::peer_list p2p_peers(const plato_partition* p, int par) {
  plato_b200::peer_list l{};
  uint32_t k = 0;
  const size_t base = static_cast<size_t>(p->rank) * p->n;
  for (uint32_t q = 0; q < p->world; ++q)
    if (q != p->rank) l.p[k++] = p->peer_s[par][q] + base;
  return l;
}

plato_b200::flag_list p2p_flags(const plato_partition* p) {
  plato_b200::flag_list l{};
  for (uint32_t q = 0; q < p->world; ++q) l.p[q] = p->peer_flags[q];
  return l;
}

plato_b200::delta_list p2p_deltas(const plato_partition* p) {
  plato_b200::delta_list l{};
  for (uint32_t q = 0; q < p->world; ++q) l.p[q] = p->peer_deltas[q];
  return l;
}

}  // namespace

extern "C" int plato_partition_p2p_alloc(plato_partition* p, void* handles) {
  if (!p || !handles) return set_error(PLATO_EINVAL, "plato_partition_p2p_alloc: null argument");
  PLATO_TRY(p2p_alloc_local(p));
  auto* h = static_cast<cudaIpcMemHandle_t*>(handles);
  PLATO_CUDA_TRY(cudaIpcGetMemHandle(h + 0, p->s[0]));
  PLATO_CUDA_TRY(cudaIpcGetMemHandle(h + 1, p->s[1]));
  PLATO_CUDA_TRY(cudaIpcGetMemHandle(h + 2, p->sync));
  return PLATO_OK;
}

extern "C" int plato_partition_p2p_connect(plato_partition* p, const void* all_handles, uint32_t timeout_ms) {
  if (!p || !all_handles) return set_error(PLATO_EINVAL, "plato_partition_p2p_connect: null argument");
  if (!p->s[0]) return set_error(PLATO_EINVAL, "plato_partition_p2p_connect: call plato_partition_p2p_alloc first");
  PLATO_CUDA_TRY(cudaSetDevice(p->g->device));
  const auto* h = static_cast<const cudaIpcMemHandle_t*>(all_handles);
  for (uint32_t q = 0; q < p->world; ++q) {
    if (q == p->rank || p->ipc_base[q][0]) continue;
    for (int i = 0; i < 3; ++i)
      PLATO_CUDA_TRY(cudaIpcOpenMemHandle(&p->ipc_base[q][i], h[3 * q + i], cudaIpcMemLazyEnablePeerAccess));
    p->peer_s[0][q] = static_cast<float*>(p->ipc_base[q][0]);
    p->peer_s[1][q] = static_cast<float*>(p->ipc_base[q][1]);
    p->peer_flags[q] = static_cast<uint32_t*>(p->ipc_base[q][2]);
    p->peer_deltas[q] = reinterpret_cast<double*>(static_cast<unsigned char*>(p->ipc_base[q][2]) + kSyncDeltas);
  }
  p->timeout_ns = static_cast<uint64_t>(timeout_ms ? timeout_ms : 5000) * 1000000ull;
  p->p2p_ready = true;
  return PLATO_OK;
}

extern "C" int plato_partition_p2p_connect_local(plato_partition* const* parts, uint32_t world, uint32_t timeout_ms) {
  if (!parts || world == 0 || world > 8) return set_error(PLATO_EINVAL, "plato_partition_p2p_connect_local: bad argument");
  for (uint32_t r = 0; r < world; ++r) {
    if (!parts[r] || parts[r]->world != world || parts[r]->rank != r)
      return set_error(PLATO_EINVAL, "plato_partition_p2p_connect_local: parts[r] must be partition r of world");
    PLATO_TRY(p2p_alloc_local(parts[r]));
  }
  for (uint32_t r = 0; r < world; ++r) {
    plato_partition* p = parts[r];
    for (uint32_t q = 0; q < world; ++q) {
      const plato_partition* o = parts[q];
      if (o->g->device != p->g->device) {  // partitions on several GPUs of one process
        int ok = 0;
        PLATO_CUDA_TRY(cudaDeviceCanAccessPeer(&ok, p->g->device, o->g->device));
        if (!ok) return set_error(PLATO_EINVAL, "plato_partition_p2p_connect_local: no peer access between the GPUs");
        PLATO_CUDA_TRY(cudaSetDevice(p->g->device));
        const cudaError_t e = cudaDeviceEnablePeerAccess(o->g->device, 0);
        if (e != cudaSuccess && e != cudaErrorPeerAccessAlreadyEnabled) PLATO_CUDA_TRY(e);
        cudaGetLastError();
      }
      p->peer_s[0][q] = o->s[0];
      p->peer_s[1][q] = o->s[1];
      p->peer_flags[q] = o->flags;
      p->peer_deltas[q] = o->deltas;
    }
    p->timeout_ns = static_cast<uint64_t>(timeout_ms ? timeout_ms : 5000) * 1000000ull;
    p->p2p_ready = true;
  }
  return PLATO_OK;
}

extern "C" int plato_partition_p2p_reset(plato_partition* p) {
  if (!p || !p->s[0]) return set_error(PLATO_EINVAL, "plato_partition_p2p_reset: not allocated");
  PLATO_CUDA_TRY(cudaSetDevice(p->g->device));
  PLATO_CUDA_TRY(cudaMemset(p->sync, 0, kSyncDeltas + 2ull * p->world * sizeof(double)));
  PLATO_CUDA_TRY(cudaMemset(p->ctrl, 0, 4 * sizeof(int)));
  return PLATO_OK;
}

extern "C" int plato_partition_p2p_init(plato_partition* p, uint32_t iterations, double damping, double eps,
                                        void* stream) {
  if (!p || !p->p2p_ready) return set_error(PLATO_EINVAL, "plato_partition_p2p_init: not connected");
  if (!(damping >= 0.0 && damping <= 1.0)) return set_error(PLATO_EINVAL, "damping must be in [0, 1]");
  if (iterations == 0 || iterations > 0x7FFFFFF0u) return set_error(PLATO_EINVAL, "iteration must be >= 1");
  PLATO_CUDA_TRY(cudaSetDevice(p->g->device));
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  p->iterations = iterations;
  p->eps = eps > 0.0 ? eps : 0.0;
  // the device epoch control: mode of epoch 0, nothing run yet, eps mode
  const int c[3] = {iterations == 1 ? 1 : 0, 0, p->eps > 0.0 ? 1 : 0};
  PLATO_CUDA_TRY(cudaMemcpyAsync(p->ctrl + 1, c, sizeof(c), cudaMemcpyHostToDevice, st));
  const float ghost = static_cast<float>((1.0 - damping) / p->V);
  k_part_init_bcast<<<grid_for(p->n, 256), 256, 0, st>>>(p->g->out_deg.p, p->n, p->real, p->V, ghost,
                                                         p->s[0] + static_cast<size_t>(p->rank) * p->n,
                                                         p2p_peers(p, 0), p->world - 1);
  PLATO_LAUNCHED("k_part_init_bcast");
  k_p2p_signal<<<1, 32, 0, st>>>(p2p_flags(p), p2p_deltas(p), p->world, p->rank, 1u, nullptr, 0u);
  PLATO_LAUNCHED("k_p2p_signal");
  return PLATO_OK;
}

extern "C" int plato_partition_p2p_epoch(plato_partition* p, uint32_t epoch, double damping, void* stream) {
  if (!p || !p->p2p_ready || p->iterations == 0)
    return set_error(PLATO_EINVAL, "plato_partition_p2p_epoch: not initialised");
  if (epoch >= p->iterations) return set_error(PLATO_EINVAL, "plato_partition_p2p_epoch: epoch >= iterations");
  if (!(damping >= 0.0 && damping <= 1.0)) return set_error(PLATO_EINVAL, "damping must be in [0, 1]");
  PLATO_CUDA_TRY(cudaSetDevice(p->g->device));
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int par = static_cast<int>(epoch & 1u);
  const bool eps_mode = p->eps > 0.0;
  // every partition has published epoch - 1 (init counts as 0): state[par],
  // and with eps their deltas of epoch - 1, are complete here
  k_p2p_wait<<<1, 32, 0, st>>>(p->flags, p->world, epoch + 1, p->ctrl, p->timeout_ns);
  PLATO_LAUNCHED("k_p2p_wait");
  if (eps_mode && epoch > 0) {
    k_p2p_control<<<1, 32, 0, st>>>(p->deltas, p->world, epoch, p->ctrl, static_cast<double>(p->V), p->eps,
                                    p->iterations);
    PLATO_LAUNCHED("k_p2p_control");
  }
  const size_t base = static_cast<size_t>(p->rank) * p->n;
  const plato_b200::peer_list peers = p2p_peers(p, par ^ 1);
  PLATO_TRY(pull_epoch_partition_bcast(p->g, p->s[par], p->s[par] + base, p->s[par ^ 1] + base, peers.p,
                                       p->world - 1, static_cast<float>((1.0 - damping) / p->V),
                                       static_cast<float>(damping), epoch + 1 == p->iterations,
                                       eps_mode ? p->ctrl + 1 : nullptr, st, eps_mode ? p->d_part : nullptr));
  k_p2p_signal<<<1, 32, 0, st>>>(p2p_flags(p), p2p_deltas(p), p->world, p->rank, epoch + 2,
                                 eps_mode ? p->d_part : nullptr, epoch & 1u);
  PLATO_LAUNCHED("k_p2p_signal");
  return PLATO_OK;
}

extern "C" int plato_partition_p2p_state(plato_partition* p, void* stream, const float** d_state, uint32_t* epochs) {
  if (!p || !p->p2p_ready || p->iterations == 0 || !d_state)
    return set_error(PLATO_EINVAL, "plato_partition_p2p_state: bad argument");
  PLATO_CUDA_TRY(cudaSetDevice(p->g->device));
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  k_p2p_wait<<<1, 32, 0, st>>>(p->flags, p->world, p->iterations + 1, p->ctrl, p->timeout_ns);
  PLATO_LAUNCHED("k_p2p_wait");
  int c[3] = {0, 0, 0};
  PLATO_CUDA_TRY(cudaMemcpyAsync(c, p->ctrl, sizeof(c), cudaMemcpyDeviceToHost, st));
  PLATO_CUDA_TRY(cudaStreamSynchronize(st));
  if (c[0])
    return set_error(PLATO_ETIMEDOUT, "partition p2p: a partition did not publish its epoch within the timeout");
  // fixed epochs: all ran; with eps: those counted by the control, plus a
  // final epoch that no later control counted
  const uint32_t ran = p->eps > 0.0 ? static_cast<uint32_t>(c[2]) + (c[1] == 1 ? 1u : 0u) : p->iterations;
  if (epochs) *epochs = ran;
  *d_state = p->s[ran & 1u];
  return PLATO_OK;
}

extern "C" int plato_partition_p2p_ranks(plato_partition* p, void* stream, float* ranks, uint32_t* epochs) {
  if (!ranks) return set_error(PLATO_EINVAL, "plato_partition_p2p_ranks: null argument");
  const float* d_state = nullptr;
  PLATO_TRY(plato_partition_p2p_state(p, stream, &d_state, epochs));
  std::vector<float> h(static_cast<size_t>(p->world) * p->n);
  PLATO_CUDA_TRY(cudaMemcpy(h.data(), d_state, h.size() * sizeof(float), cudaMemcpyDeviceToHost));
  return plato_partition_ranks(p, h.data(), ranks);
}
