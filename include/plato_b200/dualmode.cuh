/*
 * dualmode.cuh — header-only device form of plato::dualmode_engine_t.
 *
 * Mirrors the reference engine (plato/engine/dualmode.hpp:75-166) on a graph
 * resident in HBM (plato_graph from include/plato_b200.h):
 *
 *   plato_b200::dualmode_engine_t engine(graph);            // dualmode.hpp:93-97
 *   auto rank   = engine.alloc_v_state<double>();           // :232-236
 *   auto active = engine.alloc_v_subset();                  // :238-242
 *   R r = engine.foreach_edges<MSG, R>(push_signal, push_slot,
 *                                      pull_signal, pull_slot, active);  // :245-297
 *   R r = engine.foreach_edges<MSG, R>(push_signal, push_slot, active);  // push only
 *   R r = engine.foreach_edges<MSG, R>(pull_signal, pull_slot);          // pull only
 *
 * Functors are __device__ (extended) lambdas with the reference's shapes
 * (dualmode.hpp:119-124):
 *   push_signal  void(const push_context<MSG>&, vid_t v)        ctx.send(MSG)
 *   push_slot    R(int p, MSG& msg)
 *   pull_signal  void(const pull_context<MSG>&, vid_t v, const adj_unit_list_t& adjs)
 *                                                                ctx.send(mepa_ag_message_t<MSG>)
 *   pull_slot    R(int p, mepa_ag_message_t<MSG>& msg)
 * context.send() applies the slot on the device right away (the reference
 * ships the message through MPI, message_passing.hpp:88-144, :286-335), and
 * the call returns the sum of the slot returns, like the reference.
 *
 * Execution model (what "thread safe" means here, as in the reference where
 * functors run concurrently on OpenMP threads):
 *   pull  every vertex with in-edges is visited; its in-adjacency is split into
 *         chunks of at most kPullChunk edges and each chunk is one signal call,
 *         exactly like the reference's per-partition pieces of a DCSC column,
 *         so a vertex may receive several messages and the slot must combine
 *         them (atomics), as the reference's write_add / CAS slots do.
 *   push  one signal call per active vertex (thread per vertex, frontier
 *         compacted with ballot/popc); the slot reaches out-edges through
 *         engine.out_edges().neighbours(v).
 *   switch  active_edges = sum of out-degrees over `actives`; push iff
 *         active_edges / edges < push_threshold, edges doubled for undirected
 *         graphs (dualmode.hpp:261-279).
 *   pull with a combiner (opt-in: the overloads that take
 *         make_combiner(f), f(MSG& into, const MSG& from)): the in-adjacency
 *         is split into pieces of at most kPiece (4) edges, consecutive
 *         lanes of a warp take consecutive pieces (a warp reads up to 128
 *         contiguous ids), each piece is one signal call, and the messages
 *         of one vertex within a warp are folded with f in lane order before
 *         one slot call per vertex and warp.  f must be associative; a
 *         signal's messages must be for its own vertex v.  Without a
 *         combiner the 64-edge path above runs.
 * Vertex ids seen by functors are the engine's internal ids; states copied to
 * the host with to_host() are returned in caller ids.
 */
#pragma once

#include <cuda_runtime.h>

#include <cub/device/device_scan.cuh>

#include <cstdint>
#include <cstring>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "plato_b200.h"

namespace plato_b200 {

using vid_t = uint32_t;
using eid_t = uint64_t;

constexpr uint32_t kPullChunk = 64;
constexpr uint32_t kPiece = 4;  // edges per signal call on the combined pull

// Message combiner of the combined pull: f(MSG& into, const MSG& from).
template <typename F>
struct combiner {
  F f;
};
template <typename F>
combiner<F> make_combiner(F f) {
  return combiner<F>{f};
}

struct adj_unit_t {  // adj_unit_t<empty_t> (plato/graph/base.hpp)
  vid_t neighbour_;
};

struct adj_unit_list_t {  // adj_unit_list_t (plato/graph/base.hpp)
  const adj_unit_t* begin_;
  const adj_unit_t* end_;
};

template <typename MSG>
struct mepa_ag_message_t {  // plato/graph/message_passing.hpp:47-56
  vid_t v_i_;
  MSG message_;
};

struct dualmode_engine_opts_t {  // plato/engine/dualmode.hpp:41-43
  double push_threshold_ = 0.05;
};

inline void check_cuda(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

// Device memory of the engine (states, bitmaps, work lists, scratch) comes
// from a stream-ordered pool on the legacy default stream, where the
// engine's kernels run: a freed block returns to the pool without a
// device-wide synchronisation, and the next engine, state or bitmap reuses
// it.  The pool keeps up to kPoolKeepBytes of freed memory per device.
constexpr uint64_t kPoolKeepBytes = 1ull << 30;

inline cudaMemPool_t engine_pool() {
  static cudaMemPool_t pools[64] = {};
  static std::mutex mu;
  int dev = 0;
  check_cuda(cudaGetDevice(&dev), "engine pool: device");
  std::lock_guard<std::mutex> lock(mu);
  if (dev < 0 || dev >= 64) throw std::runtime_error("engine pool: device index out of range");
  if (!pools[dev]) {
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    check_cuda(cudaMemPoolCreate(&pools[dev], &props), "engine pool: create");
    uint64_t keep = kPoolKeepBytes;
    check_cuda(cudaMemPoolSetAttribute(pools[dev], cudaMemPoolAttrReleaseThreshold, &keep),
               "engine pool: release threshold");
  }
  return pools[dev];
}

template <typename T>
inline void dev_alloc(T** p, size_t bytes, const char* what) {
  check_cuda(cudaMallocFromPoolAsync(reinterpret_cast<void**>(p), bytes ? bytes : 1, engine_pool(), 0), what);
}

inline void dev_free(void* p) {
  if (p) cudaFreeAsync(p, 0);
}

// Out-edge view usable inside device functors (bcsr_t::neighbours, bcsr.hpp:225-240).
struct out_edges_view {
  const uint64_t* off;
  const vid_t* adj;
  __device__ adj_unit_list_t neighbours(vid_t v) const {
    return adj_unit_list_t{reinterpret_cast<const adj_unit_t*>(adj + off[v]),
                           reinterpret_cast<const adj_unit_t*>(adj + off[v + 1])};
  }
};

// Device bitmap (bitmap_t, plato/util/bitmap.hpp:43-350), 32-bit words.
class bitmap_t {
 public:
  bitmap_t() = default;
  explicit bitmap_t(uint32_t n) : n_(n) {
    dev_alloc(&w_, words() * sizeof(uint32_t), "bitmap alloc");
    clear();
  }
  bitmap_t(bitmap_t&& o) noexcept : w_(o.w_), n_(o.n_) { o.w_ = nullptr; }
  bitmap_t& operator=(bitmap_t&& o) noexcept {
    std::swap(w_, o.w_);
    std::swap(n_, o.n_);
    return *this;
  }
  bitmap_t(const bitmap_t&) = delete;
  bitmap_t& operator=(const bitmap_t&) = delete;
  ~bitmap_t() {
    dev_free(w_);
  }
  size_t words() const { return (static_cast<size_t>(n_) + 31) / 32; }
  void clear() { check_cuda(cudaMemset(w_, 0, words() * 4), "bitmap clear"); }
  uint32_t size() const { return n_; }
  uint32_t* data() const { return w_; }
  // host-side single bit set (bitmap.hpp:207-222)
  void set_bit_host(vid_t v) {
    uint32_t w = 0;
    check_cuda(cudaMemcpy(&w, w_ + (v >> 5), 4, cudaMemcpyDeviceToHost), "bitmap read");
    w |= 1u << (v & 31);
    check_cuda(cudaMemcpy(w_ + (v >> 5), &w, 4, cudaMemcpyHostToDevice), "bitmap write");
  }
  // popcount (bitmap.hpp:229-238)
  uint64_t count() const;

  struct view {
    uint32_t* w;
    __device__ void set_bit(vid_t v) const { atomicOr(w + (v >> 5), 1u << (v & 31)); }
    __device__ bool get_bit(vid_t v) const { return (w[v >> 5] >> (v & 31)) & 1u; }
  };
  view dev() const { return view{w_}; }

 private:
  uint32_t* w_ = nullptr;
  uint32_t n_ = 0;
};

// Device vertex state (dense_state_t, plato/graph/state/dense_state.hpp:43-425).
template <typename T>
class dense_state_t {
 public:
  dense_state_t() = default;
  explicit dense_state_t(uint32_t n) : n_(n) {
    dev_alloc(&p_, sizeof(T) * (n ? n : 1), "state alloc");
  }
  dense_state_t(dense_state_t&& o) noexcept : p_(o.p_), n_(o.n_) { o.p_ = nullptr; }
  dense_state_t& operator=(dense_state_t&& o) noexcept {
    std::swap(p_, o.p_);
    std::swap(n_, o.n_);
    return *this;
  }
  dense_state_t(const dense_state_t&) = delete;
  dense_state_t& operator=(const dense_state_t&) = delete;
  ~dense_state_t() {
    dev_free(p_);
  }
  T* data() const { return p_; }
  uint32_t size() const { return n_; }
  void fill(const T& v);  // dense_state.hpp:241-254
  // raw copy in the engine's internal vertex order
  std::vector<T> to_host_internal() const {
    std::vector<T> h(n_);
    check_cuda(cudaMemcpy(h.data(), p_, sizeof(T) * n_, cudaMemcpyDeviceToHost), "state copy");
    return h;
  }

 private:
  T* p_ = nullptr;
  uint32_t n_ = 0;
};

namespace detail {

template <typename T>
__global__ void k_fill(T* p, uint32_t n, T v) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x)
    p[i] = v;
}

static __global__ void k_popc(const uint32_t* w, size_t nw, unsigned long long* out) {
  unsigned long long c = 0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < nw;
       i += (size_t)gridDim.x * blockDim.x)
    c += __popc(w[i]);
  atomicAdd(out, c);
}

// Frontier compaction + active-edge count (dualmode.hpp:264-277).  Warps
// reserve queue slots in shared memory and one thread per block and round
// takes the block's range from the global counter, so a dense frontier does
// not serialise on one address.
static __global__ void __launch_bounds__(256) k_compact(const uint32_t* bits, uint32_t n,
                                                        const uint32_t* deg, vid_t* queue,
                                                        unsigned long long* counters) {
  __shared__ unsigned long long s_base, s_deg;
  __shared__ uint32_t s_cnt;
  const unsigned lane = threadIdx.x & 31;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  const uint64_t rounds = (n + stride - 1) / stride;
  for (uint64_t r = 0; r < rounds; ++r) {  // block-uniform trip count
    const uint64_t v = r * stride + blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    const bool on = v < n && ((bits[v >> 5] >> (v & 31)) & 1u);
    if (threadIdx.x == 0) {
      s_cnt = 0;
      s_deg = 0;
    }
    __syncthreads();
    const unsigned m = __ballot_sync(0xffffffffu, on);
    unsigned long long de = on ? deg[v] : 0ull;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) de += __shfl_xor_sync(0xffffffffu, de, o);
    uint32_t wbase = 0;
    if (lane == 0 && m) {
      wbase = atomicAdd(&s_cnt, static_cast<uint32_t>(__popc(m)));
      if (de) atomicAdd(&s_deg, de);
    }
    wbase = __shfl_sync(0xffffffffu, wbase, 0);
    __syncthreads();
    if (threadIdx.x == 0) {
      if (s_cnt) s_base = atomicAdd(&counters[0], static_cast<unsigned long long>(s_cnt));
      if (s_deg) atomicAdd(&counters[1], s_deg);
    }
    __syncthreads();
    if (on) queue[s_base + wbase + __popc(m & ((1u << lane) - 1u))] = static_cast<vid_t>(v);
  }
}

// Pull chunk list: (vertex, first edge) for every kPullChunk edges of every column.
static __global__ void k_count_chunks(const uint64_t* off, uint32_t V, uint64_t* cnt) {
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < V;
       v += (uint64_t)gridDim.x * blockDim.x)
    cnt[v] = (off[v + 1] - off[v] + kPullChunk - 1) / kPullChunk;
}

static __global__ void k_fill_chunks(const uint64_t* off, uint32_t V, const uint64_t* cstart,
                                     uint2* chunks) {
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < V;
       v += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t n = (off[v + 1] - off[v] + kPullChunk - 1) / kPullChunk;
    for (uint64_t k = 0; k < n; ++k) chunks[cstart[v] + k] = make_uint2(static_cast<uint32_t>(v), static_cast<uint32_t>(k));
  }
}

template <typename R>
__device__ inline void reduce_add(R v, R* out) {
  atomicAdd(out, v);
}

}  // namespace detail

// Contexts handed to the signal functors.
template <typename MSG, typename R, typename SLOT>
struct pull_context {
  const SLOT* slot;
  R* acc;
  __device__ void send(const mepa_ag_message_t<MSG>& m) const {
    mepa_ag_message_t<MSG> msg = m;
    *acc += (*slot)(0, msg);
  }
};

template <typename MSG, typename R, typename SLOT>
struct push_context {
  const SLOT* slot;
  R* acc;
  __device__ void send(const MSG& m) const {
    MSG msg = m;
    *acc += (*slot)(0, msg);
  }
};

namespace detail {

template <typename MSG, typename R, typename SIG, typename SLOT>
__global__ void k_pull(const uint2* chunks, uint64_t nchunks, const uint64_t* off, const vid_t* adj,
                       SIG sig, SLOT slot, R* result) {
  R acc = R();
  pull_context<MSG, R, SLOT> ctx{&slot, &acc};
  for (uint64_t c = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; c < nchunks;
       c += (uint64_t)gridDim.x * blockDim.x) {
    const uint2 ch = chunks[c];
    const uint64_t b = off[ch.x] + static_cast<uint64_t>(ch.y) * kPullChunk;
    const uint64_t e = min(b + kPullChunk, off[ch.x + 1]);
    const adj_unit_list_t adjs{reinterpret_cast<const adj_unit_t*>(adj + b),
                               reinterpret_cast<const adj_unit_t*>(adj + e)};
    sig(ctx, static_cast<vid_t>(ch.x), adjs);
  }
  if (acc != R()) reduce_add(acc, result);
}

template <typename MSG, typename R, typename SIG, typename SLOT>
__global__ void k_push(const vid_t* queue, uint64_t n, SIG sig, SLOT slot, R* result) {
  R acc = R();
  push_context<MSG, R, SLOT> ctx{&slot, &acc};
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x)
    sig(ctx, queue[i]);
  if (acc != R()) reduce_add(acc, result);
}

// Pieces of the combined pull.  Columns with in-edges are listed in vertex
// order (colv) with the index of their first piece (pstart, a column of d
// edges has ceil(d / kPiece) pieces); wstart[w] is the column holding piece
// 32w, the first piece of warp w.
static __global__ void k_piece_flags(const uint64_t* off, uint32_t V, uint32_t* flag) {
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < V;
       v += (uint64_t)gridDim.x * blockDim.x)
    flag[v] = off[v + 1] > off[v] ? 1u : 0u;
}

static __global__ void k_piece_cols(const uint64_t* off, uint32_t V, const uint32_t* cidx, vid_t* colv,
                                    uint64_t* npieces) {
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < V;
       v += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t d = off[v + 1] - off[v];
    if (d == 0) continue;
    colv[cidx[v]] = static_cast<vid_t>(v);
    npieces[cidx[v]] = (d + kPiece - 1) / kPiece;
  }
}

static __global__ void k_piece_warps(const uint64_t* pstart, uint32_t ncols, uint32_t* wstart) {
  for (uint64_t c = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; c < ncols;
       c += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t ps = pstart[c], pe = pstart[c + 1];
    for (uint64_t w = (ps + 31) / 32; w * 32 < pe; ++w) wstart[w] = static_cast<uint32_t>(c);
  }
}

// Lane-to-lane shift of any trivially copyable message (whole 32-bit words).
template <typename T>
__device__ __forceinline__ T shfl_up_any(const T& v, unsigned d) {
  static_assert(sizeof(T) % 4 == 0, "combined pull: message size must be a multiple of 4 bytes");
  constexpr int kWords = sizeof(T) / 4;
  uint32_t w[kWords];
  memcpy(w, &v, sizeof(T));
#pragma unroll
  for (int i = 0; i < kWords; ++i) w[i] = __shfl_up_sync(0xffffffffu, w[i], d);
  T out;
  memcpy(&out, w, sizeof(T));
  return out;
}

// Context of a combined pull signal: its messages fold into one per lane.
template <typename MSG, typename COMB>
struct combine_context {
  const COMB* comb;
  MSG* msg;
  bool* has;
  __device__ void send(const mepa_ag_message_t<MSG>& m) const {
    if (*has) {
      comb->f(*msg, m.message_);
    } else {
      *msg = m.message_;
      *has = true;
    }
  }
};

template <typename MSG, typename R, typename SIG, typename SLOT, typename COMB>
__global__ void __launch_bounds__(256) k_pull_combined(const vid_t* __restrict__ colv,
                                                       const uint64_t* __restrict__ pstart,
                                                       const uint32_t* __restrict__ wstart, uint32_t ncols,
                                                       uint64_t npieces, const uint64_t* __restrict__ off,
                                                       const vid_t* __restrict__ adj, SIG sig, SLOT slot,
                                                       COMB comb, R* result) {
  const unsigned lane = threadIdx.x & 31;
  const uint64_t nwarps = (uint64_t)gridDim.x * (blockDim.x >> 5);
  R acc = R();
  for (uint64_t w = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5; w * 32 < npieces; w += nwarps) {
    const uint64_t p = w * 32 + lane;
    const bool valid = p < npieces;
    // column of each lane: c0 holds piece 32w; a later column starting at
    // relative piece r sets bit r, and lane l lies in column c0 + (bits <= l)
    const uint32_t c0 = wstart[w];
    const uint32_t cb = c0 + 1 + lane;
    const uint64_t b = cb <= ncols ? pstart[cb] : ~0ull;
    const uint64_t r = b - w * 32;
    const uint32_t bits = __reduce_or_sync(0xffffffffu, r < 32 ? (1u << r) : 0u);
    const uint32_t upto = lane == 31 ? 0xffffffffu : ((2u << lane) - 1u);
    const uint32_t col = c0 + static_cast<uint32_t>(__popc(bits & upto));
    MSG msg{};
    bool has = false;
    vid_t v = 0;
    if (valid) {
      v = colv[col];
      const uint64_t e0 = off[v] + (p - pstart[col]) * kPiece;
      const uint64_t e1 = min(e0 + kPiece, off[v + 1]);
      const adj_unit_list_t adjs{reinterpret_cast<const adj_unit_t*>(adj + e0),
                                 reinterpret_cast<const adj_unit_t*>(adj + e1)};
      combine_context<MSG, COMB> ctx{&comb, &msg, &has};
      sig(ctx, v, adjs);
    }
    // segmented inclusive scan over lanes of the same column, in lane order
    const uint32_t key = valid ? col : 0xffffffffu;
#pragma unroll
    for (unsigned d = 1; d < 32; d <<= 1) {
      const MSG om = shfl_up_any(msg, d);
      const uint32_t ok = __shfl_up_sync(0xffffffffu, key, d);
      const bool oh = __shfl_up_sync(0xffffffffu, has ? 1u : 0u, d) != 0u;
      if (lane >= d && ok == key && oh) {
        if (has) {
          MSG t = om;
          comb.f(t, msg);
          msg = t;
        } else {
          msg = om;
          has = true;
        }
      }
    }
    const uint32_t nk = __shfl_down_sync(0xffffffffu, key, 1);
    const bool tail = lane == 31 || nk != key;
    if (valid && has && tail) {
      mepa_ag_message_t<MSG> m{v, msg};
      acc += slot(0, m);
    }
  }
  if (acc != R()) reduce_add(acc, result);
}

}  // namespace detail

template <typename T>
void dense_state_t<T>::fill(const T& v) {
  detail::k_fill<T><<<592, 256>>>(p_, n_, v);
  check_cuda(cudaGetLastError(), "fill");
}

inline uint64_t bitmap_t::count() const {
  unsigned long long* d = nullptr;
  dev_alloc(&d, sizeof(*d), "count alloc");
  check_cuda(cudaMemsetAsync(d, 0, sizeof(*d), 0), "count clear");
  detail::k_popc<<<296, 256>>>(w_, words(), d);
  unsigned long long h = 0;
  check_cuda(cudaMemcpy(&h, d, sizeof(h), cudaMemcpyDeviceToHost), "count read");
  dev_free(d);
  return h;
}

class dualmode_engine_t {
 public:
  explicit dualmode_engine_t(plato_graph* g, dualmode_engine_opts_t opts = dualmode_engine_opts_t())
      : g_(g), opts_(opts) {
    if (plato_graph_get_device_view(g, &view_) != PLATO_OK) throw std::runtime_error(plato_last_error());
    plato_graph_get_info(g, &info_);
  }
  dualmode_engine_t(const dualmode_engine_t&) = delete;
  dualmode_engine_t& operator=(const dualmode_engine_t&) = delete;
  ~dualmode_engine_t() {
    for (auto& pi : pieces_) {
      dev_free(pi.colv);
      dev_free(pi.pstart);
      dev_free(pi.wstart);
    }
    dev_free(chunks_);
    dev_free(queue_);
    dev_free(counters_);
    dev_free(result_);
  }

  const plato_graph_info& graph_info() const { return info_; }
  uint32_t vertices() const { return view_.vertices; }

  template <typename T>
  dense_state_t<T> alloc_v_state() const { return dense_state_t<T>(view_.vertices); }
  bitmap_t alloc_v_subset() const { return bitmap_t(view_.vertices); }

  out_edges_view out_edges() const {
    return reversed_ ? out_edges_view{view_.in_offsets, view_.in_adj}
                     : out_edges_view{view_.out_offsets, view_.out_adj};
  }
  const uint32_t* out_degrees() const { return view_.out_degree; }
  void reverse() { reversed_ = !reversed_; }
  bool is_reversed() const { return reversed_; }

  // caller id <-> internal id (identity when the graph was not relabelled)
  vid_t to_internal(vid_t ext) const {
    if (!view_.to_internal) return ext;
    vid_t v = 0;
    check_cuda(cudaMemcpy(&v, view_.to_internal + ext, 4, cudaMemcpyDeviceToHost), "to_internal");
    return v;
  }
  template <typename T>
  std::vector<T> to_host(const dense_state_t<T>& s) const {
    std::vector<T> in = s.to_host_internal();
    if (!view_.to_external) return in;
    std::vector<vid_t> ext(view_.vertices);
    check_cuda(cudaMemcpy(ext.data(), view_.to_external, 4ull * view_.vertices, cudaMemcpyDeviceToHost),
               "to_external");
    std::vector<T> out(in.size());
    for (size_t i = 0; i < in.size(); ++i) out[ext[i]] = in[i];
    return out;
  }

  // pull only (dualmode.hpp:299-309)
  template <typename MSG, typename R, typename PULL_SIGNAL, typename PULL_SLOT>
  R foreach_edges(PULL_SIGNAL signal, PULL_SLOT slot) {
    ensure_chunks();
    R* res = result_buf<R>();
    detail::k_pull<MSG, R><<<grid(nchunks_), 256>>>(chunks_, nchunks_, in_off(), in_adj(), signal,
                                                     slot, res);
    check_cuda(cudaGetLastError(), "pull launch");
    return read_result<R>(res);
  }

  // pull only, the sum of the slot returns added into *d_result (device
  // memory, not cleared here) instead of read back: the call does not
  // synchronise, so a loop whose epochs are decided on the device can be
  // enqueued back to back.
  template <typename MSG, typename R, typename PULL_SIGNAL, typename PULL_SLOT>
  void foreach_edges_device(PULL_SIGNAL signal, PULL_SLOT slot, R* d_result) {
    ensure_chunks();
    detail::k_pull<MSG, R><<<grid(nchunks_), 256>>>(chunks_, nchunks_, in_off(), in_adj(), signal,
                                                     slot, d_result);
    check_cuda(cudaGetLastError(), "pull launch");
  }

  // pull only with a message combiner (see the header comment)
  template <typename MSG, typename R, typename PULL_SIGNAL, typename PULL_SLOT, typename F>
  R foreach_edges(PULL_SIGNAL signal, PULL_SLOT slot, combiner<F> comb) {
    R* res = result_buf<R>();
    pull_combined<MSG, R>(signal, slot, comb, res);
    return read_result<R>(res);
  }

  // as foreach_edges_device above, with a message combiner
  template <typename MSG, typename R, typename PULL_SIGNAL, typename PULL_SLOT, typename F>
  void foreach_edges_device(PULL_SIGNAL signal, PULL_SLOT slot, combiner<F> comb, R* d_result) {
    pull_combined<MSG, R>(signal, slot, comb, d_result);
  }

  // push only (dualmode.hpp:311-322)
  template <typename MSG, typename R, typename PUSH_SIGNAL, typename PUSH_SLOT>
  R foreach_edges(PUSH_SIGNAL signal, PUSH_SLOT slot, bitmap_t& actives) {
    uint64_t n = 0, ae = 0;
    compact(actives, &n, &ae);
    return push_queue<MSG, R>(signal, slot, n);
  }

  // push + pull, engine-chosen (dualmode.hpp:245-297)
  template <typename MSG, typename R, typename PUSH_SIGNAL, typename PUSH_SLOT,
            typename PULL_SIGNAL, typename PULL_SLOT>
  R foreach_edges(PUSH_SIGNAL push_signal, PUSH_SLOT push_slot, PULL_SIGNAL pull_signal,
                  PULL_SLOT pull_slot, bitmap_t& actives) {
    uint64_t n = 0, active_edges = 0;
    compact(actives, &n, &active_edges);
    uint64_t edges = info_.edges;
    if (!info_.is_directed) edges *= 2;
    last_push_ = (static_cast<double>(active_edges) / static_cast<double>(edges)) < opts_.push_threshold_;
    if (last_push_) return push_queue<MSG, R>(push_signal, push_slot, n);
    return foreach_edges<MSG, R>(pull_signal, pull_slot);
  }

  // push + pull, engine-chosen, the pull with a message combiner
  template <typename MSG, typename R, typename PUSH_SIGNAL, typename PUSH_SLOT,
            typename PULL_SIGNAL, typename PULL_SLOT, typename F>
  R foreach_edges(PUSH_SIGNAL push_signal, PUSH_SLOT push_slot, PULL_SIGNAL pull_signal,
                  PULL_SLOT pull_slot, bitmap_t& actives, combiner<F> comb) {
    uint64_t n = 0, active_edges = 0;
    compact(actives, &n, &active_edges);
    uint64_t edges = info_.edges;
    if (!info_.is_directed) edges *= 2;
    last_push_ = (static_cast<double>(active_edges) / static_cast<double>(edges)) < opts_.push_threshold_;
    if (last_push_) return push_queue<MSG, R>(push_signal, push_slot, n);
    return foreach_edges<MSG, R>(pull_signal, pull_slot, comb);
  }

  bool last_was_push() const { return last_push_; }

 private:
  const uint64_t* in_off() const { return reversed_ ? view_.out_offsets : view_.in_offsets; }
  const vid_t* in_adj() const { return reversed_ ? view_.out_adj : view_.in_adj; }
  static unsigned grid(uint64_t n) {
    uint64_t b = (n + 255) / 256;
    if (b < 1) b = 1;
    if (b > 148 * 16) b = 148 * 16;
    return static_cast<unsigned>(b);
  }

  // The chunk list of the pull direction, built on the device (counts, a
  // scan for the start of each column's chunks, then the fill).
  void ensure_chunks() {
    if (chunks_ && chunks_reversed_ == reversed_) return;
    dev_free(chunks_);
    chunks_ = nullptr;
    const uint32_t V = view_.vertices;
    uint64_t* cnt = nullptr;
    uint64_t* start = nullptr;
    void* tmp = nullptr;
    size_t tmp_bytes = 0;
    dev_alloc(&cnt, 8ull * (V ? V : 1), "chunks");
    dev_alloc(&start, 8ull * (V + 1), "chunks");
    detail::k_count_chunks<<<grid(V), 256>>>(in_off(), V, cnt);
    check_cuda(cudaMemset(start, 0, sizeof(uint64_t)), "chunks");
    check_cuda(cub::DeviceScan::InclusiveSum(nullptr, tmp_bytes, cnt, start + 1, static_cast<int64_t>(V)),
               "chunks");
    dev_alloc(&tmp, tmp_bytes, "chunks");
    check_cuda(cub::DeviceScan::InclusiveSum(tmp, tmp_bytes, cnt, start + 1, static_cast<int64_t>(V)),
               "chunks");
    uint64_t total = 0;
    check_cuda(cudaMemcpy(&total, start + V, sizeof(total), cudaMemcpyDeviceToHost), "chunks");
    nchunks_ = total;
    dev_alloc(&chunks_, sizeof(uint2) * (nchunks_ ? nchunks_ : 1), "chunks");
    detail::k_fill_chunks<<<grid(V), 256>>>(in_off(), V, start, chunks_);
    check_cuda(cudaGetLastError(), "chunks");
    dev_free(tmp);
    dev_free(cnt);
    dev_free(start);
    chunks_reversed_ = reversed_;
  }

  // The piece index of the pull direction (combined pull), built on the
  // device: non-empty columns compacted with a scan, their piece counts
  // scanned into first-piece offsets, then the first column of every warp.
  void ensure_pieces() {
    piece_index& pi = pieces_[reversed_ ? 1 : 0];
    if (pi.built) return;
    const uint32_t V = view_.vertices;
    uint32_t* flag = nullptr;
    uint32_t* cidx = nullptr;
    uint64_t* cnt = nullptr;
    void* tmp = nullptr;
    size_t tmp_bytes = 0, t2 = 0;
    dev_alloc(&flag, 4ull * (V ? V : 1), "pieces");
    dev_alloc(&cidx, 4ull * (V + 1), "pieces");
    detail::k_piece_flags<<<grid(V), 256>>>(in_off(), V, flag);
    check_cuda(cudaMemset(cidx, 0, 4), "pieces");
    check_cuda(cub::DeviceScan::InclusiveSum(nullptr, tmp_bytes, flag, cidx + 1, static_cast<int64_t>(V)), "pieces");
    dev_alloc(&tmp, tmp_bytes, "pieces");
    check_cuda(cub::DeviceScan::InclusiveSum(tmp, tmp_bytes, flag, cidx + 1, static_cast<int64_t>(V)), "pieces");
    uint32_t ncols = 0;
    check_cuda(cudaMemcpy(&ncols, cidx + V, 4, cudaMemcpyDeviceToHost), "pieces");
    pi.ncols = ncols;
    dev_alloc(&pi.colv, 4ull * (ncols ? ncols : 1), "pieces");
    dev_alloc(&cnt, 8ull * (ncols ? ncols : 1), "pieces");
    dev_alloc(&pi.pstart, 8ull * (ncols + 1), "pieces");
    detail::k_piece_cols<<<grid(V), 256>>>(in_off(), V, cidx, pi.colv, cnt);
    check_cuda(cudaMemset(pi.pstart, 0, 8), "pieces");
    check_cuda(cub::DeviceScan::InclusiveSum(nullptr, t2, cnt, pi.pstart + 1, static_cast<int64_t>(ncols)), "pieces");
    if (t2 > tmp_bytes) {
      dev_free(tmp);
      dev_alloc(&tmp, t2, "pieces");
    }
    if (ncols)
      check_cuda(cub::DeviceScan::InclusiveSum(tmp, t2, cnt, pi.pstart + 1, static_cast<int64_t>(ncols)), "pieces");
    uint64_t np = 0;
    check_cuda(cudaMemcpy(&np, pi.pstart + ncols, 8, cudaMemcpyDeviceToHost), "pieces");
    pi.npieces = np;
    const uint64_t nw = (np + 31) / 32;
    dev_alloc(&pi.wstart, 4ull * (nw ? nw : 1), "pieces");
    if (ncols) detail::k_piece_warps<<<grid(ncols), 256>>>(pi.pstart, ncols, pi.wstart);
    check_cuda(cudaGetLastError(), "pieces");
    dev_free(tmp);
    dev_free(flag);
    dev_free(cidx);
    dev_free(cnt);
    pi.built = true;
  }

  template <typename MSG, typename R, typename SIG, typename SLOT, typename F>
  void pull_combined(SIG signal, SLOT slot, combiner<F> comb, R* res) {
    ensure_pieces();
    const piece_index& pi = pieces_[reversed_ ? 1 : 0];
    if (pi.npieces == 0) return;
    const uint64_t threads = (pi.npieces + 31) / 32 * 32;
    detail::k_pull_combined<MSG, R><<<grid(threads), 256>>>(pi.colv, pi.pstart, pi.wstart, pi.ncols, pi.npieces,
                                                             in_off(), in_adj(), signal, slot, comb, res);
    check_cuda(cudaGetLastError(), "combined pull launch");
  }

  void compact(bitmap_t& actives, uint64_t* n, uint64_t* active_edges) {
    const uint32_t V = view_.vertices;
    if (!queue_) dev_alloc(&queue_, 4ull * (V ? V : 1), "queue");
    if (!counters_) dev_alloc(&counters_, 16, "counters");
    check_cuda(cudaMemset(counters_, 0, 16), "counters");
    const uint32_t* deg = reversed_ ? view_.in_degree : view_.out_degree;
    detail::k_compact<<<grid(V), 256>>>(actives.data(), V, deg, queue_, counters_);
    unsigned long long h[2];
    check_cuda(cudaMemcpy(h, counters_, 16, cudaMemcpyDeviceToHost), "counters");
    *n = h[0];
    *active_edges = h[1];
  }

  template <typename MSG, typename R, typename SIG, typename SLOT>
  R push_queue(SIG signal, SLOT slot, uint64_t n) {
    R* res = result_buf<R>();
    if (n) {
      detail::k_push<MSG, R><<<grid(n), 256>>>(queue_, n, signal, slot, res);
      check_cuda(cudaGetLastError(), "push launch");
    }
    return read_result<R>(res);
  }

  template <typename R>
  R* result_buf() {
    if (!result_) dev_alloc(&result_, 16, "result");
    check_cuda(cudaMemset(result_, 0, 16), "result");
    return reinterpret_cast<R*>(result_);
  }
  template <typename R>
  R read_result(R* res) {
    R h{};
    check_cuda(cudaMemcpy(&h, res, sizeof(R), cudaMemcpyDeviceToHost), "result");
    return h;
  }

  struct piece_index {
    bool built = false;
    uint32_t ncols = 0;
    uint64_t npieces = 0;
    vid_t* colv = nullptr;
    uint64_t* pstart = nullptr;
    uint32_t* wstart = nullptr;
  };

  plato_graph* g_;
  dualmode_engine_opts_t opts_;
  plato_graph_device_view view_{};
  plato_graph_info info_{};
  bool reversed_ = false, chunks_reversed_ = false, last_push_ = false;
  uint2* chunks_ = nullptr;
  uint64_t nchunks_ = 0;
  vid_t* queue_ = nullptr;
  unsigned long long* counters_ = nullptr;
  void* result_ = nullptr;
  piece_index pieces_[2];  // by direction: in-edges, out-edges (reversed)
};

}  // namespace plato_b200
