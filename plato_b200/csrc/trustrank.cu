// TrustRank: good-seed selection, then seed-set personalized PageRank.
//
// Mirrors plato/algo/trustrank/trustrank.hpp:
//   select (select_good_seeds, :88-146)
//     V <= seed_num       every good vertex is a seed;
//     method 0 / 1        the seed_num vertices of highest inverse PageRank
//                         (PageRank of the transposed graph, generate_rank_pairs
//                         over the out-edges, :52-71) or PageRank, ordered by
//                         rank descending then id ascending, that are good;
//     method 2            seed_num distinct vertices drawn uniformly, the good
//                         ones kept (the reference seeds its generator from
//                         std::random_device; here the caller's seed is used,
//                         so a run can be repeated).
//   trust (trustrank, :163-259)  seed-set PPR with those seeds: init 1/|S|
//                         (divided by the out-degree) on seeds, teleport
//                         (1-d)/|S| on seeds, eps early exit into a final
//                         epoch -- plato_seedset_ppr on the binned pull.
// The selection PageRank is the reference's default run (pagerank_opts_t:
// 100 epochs, damping 0.85, eps 0.001; pagerank.hpp:39-46, 81-146) in double
// precision, written with the reference's functor bodies for
// include/plato_b200/dualmode.cuh (engine.reverse() for the transposed
// graph), so the order of the ranks is the reference's up to FP64 rounding.
// Its pulls run on the engine's combined path: the sums of a vertex's
// 4-edge pieces in one warp are added in lane order before one write_add.
#include <algorithm>
#include <exception>
#include <mutex>
#include <random>
#include <unordered_set>
#include <vector>

#include <cub/device/device_radix_sort.cuh>

#include "graph.cuh"
#include "plato_b200/dualmode.cuh"

namespace plato_b200 {
namespace {

__global__ void k_tr_init(double* x, const uint32_t* __restrict__ deg, uint32_t V) {
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < V;
       v += (uint64_t)gridDim.x * blockDim.x)
    x[v] = deg[v] > 0 ? 1.0 / deg[v] : 1.0;  // pagerank.hpp:90-98
}

// pagerank.hpp:118-135: r = (1-d) + d*y; non-final epochs divide by the degree
// and sum |x' - x| * deg, one partial per block (summed in a fixed order by
// k_tr_control, so the exit epoch does not depend on atomic order).  The
// epoch is final when it is the last one or when ctrl[1] says so; nothing
// runs once ctrl[0] is set.
__global__ void __launch_bounds__(256) k_tr_update(double* n, const double* __restrict__ c,
                                                   const uint32_t* __restrict__ deg, uint32_t V, double d,
                                                   int last_epoch, double* partials, const uint32_t* ctrl) {
  __shared__ double s_red[32];
  if (ctrl[0]) return;
  const bool last = last_epoch || ctrl[1];
  double dl = 0.0;
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < V;
       v += (uint64_t)gridDim.x * blockDim.x) {
    double r = (1.0 - d) + d * n[v];
    if (!last) {
      if (deg[v] > 0) {
        r /= deg[v];
        dl += fabs(r - c[v]) * deg[v];
      } else {
        dl += fabs(r - c[v]);
      }
    }
    n[v] = r;
  }
  dl = block_sum<256>(dl, s_red);
  if (threadIdx.x == 0) partials[blockIdx.x] = dl;
}

// next.fill(0) of the epoch, skipped like the rest once the final epoch has
// run (the buffer it would clear may hold the result).
__global__ void k_tr_zero(double* n, uint32_t V, const uint32_t* ctrl) {
  if (ctrl[0]) return;
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < V;
       v += (uint64_t)gridDim.x * blockDim.x)
    n[v] = 0.0;
}

// The eps early exit of pagerank.hpp:137-139 decided on the device, so the
// host enqueues every epoch without waiting: the epoch's delta is the sum of
// the update's n block partials in a fixed order; after a non-final epoch
// with delta < eps the next epoch is the final one (ctrl[1]); after the
// final epoch ctrl[0] stops the rest and ctrl[2] records which epoch it was.
__global__ void __launch_bounds__(1024) k_tr_control(const double* __restrict__ partials, uint32_t n,
                                                     double eps, uint32_t epoch, int last_epoch,
                                                     uint32_t* ctrl) {
  __shared__ double s_red[32];
  if (ctrl[0]) return;  // grid-uniform
  const uint32_t per = (n + 1023) / 1024;
  const uint32_t b = threadIdx.x * per, e = min(n, b + per);
  double s = 0.0;
  for (uint32_t i = b; i < e; ++i) s += partials[i];
  s = block_sum<1024>(s, s_red);
  if (threadIdx.x != 0) return;
  if (last_epoch || ctrl[1]) {
    ctrl[0] = 1;
    ctrl[2] = epoch;
  } else if (s < eps) {
    ctrl[1] = 1;
  }
}

// Selection ranks laid out by caller id, with the caller ids beside them.
__global__ void k_tr_keys(const double* __restrict__ r, const uint32_t* __restrict__ to_ext, uint32_t V,
                          double* keys, uint32_t* ids) {
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < V;
       v += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t e = to_ext ? to_ext[v] : static_cast<uint32_t>(v);
    keys[e] = r[v];
    ids[e] = e;
  }
}

// The k caller ids of highest rank, ties by smaller id (trustrank.hpp:108-112),
// chosen on the device: a stable descending radix sort of (rank, id) pairs
// laid out by ascending id keeps equal ranks in id order.  Ranks are
// positive and finite, where the radix order of doubles is their numeric
// order.
std::vector<uint32_t> top_ids(const double* r, const uint32_t* to_ext, uint32_t V, uint32_t k) {
  double *ka = nullptr, *kb = nullptr;
  uint32_t *ia = nullptr, *ib = nullptr;
  void* tmp = nullptr;
  size_t bytes = 0;
  std::vector<uint32_t> out(k);
  check_cuda(cub::DeviceRadixSort::SortPairsDescending(nullptr, bytes, ka, kb, ia, ib, static_cast<int64_t>(V)),
             "top ids");
  try {
    dev_alloc(&ka, 8ull * V, "top ids");
    dev_alloc(&kb, 8ull * V, "top ids");
    dev_alloc(&ia, 4ull * V, "top ids");
    dev_alloc(&ib, 4ull * V, "top ids");
    dev_alloc(&tmp, bytes, "top ids");
    k_tr_keys<<<grid_for(V, 256), 256>>>(r, to_ext, V, ka, ia);
    check_cuda(cudaGetLastError(), "k_tr_keys");
    count_launch();
    check_cuda(cub::DeviceRadixSort::SortPairsDescending(tmp, bytes, ka, kb, ia, ib, static_cast<int64_t>(V)),
               "top ids");
    if (k) check_cuda(cudaMemcpy(out.data(), ib, 4ull * k, cudaMemcpyDeviceToHost), "top ids");
  } catch (...) {
    dev_free(ka);
    dev_free(kb);
    dev_free(ia);
    dev_free(ib);
    dev_free(tmp);
    throw;
  }
  dev_free(ka);
  dev_free(kb);
  dev_free(ia);
  dev_free(ib);
  dev_free(tmp);
  return out;
}

// The k caller ids of highest rank under the reference's default PageRank on
// the graph (transposed when `inverse`).
std::vector<uint32_t> selection_top(plato_graph* g, bool inverse, uint32_t k) {
  constexpr uint32_t kIterations = 100;
  constexpr double kDamping = 0.85, kEps = 0.001;
  dualmode_engine_t engine(g);
  plato_graph_device_view view{};
  if (plato_graph_get_device_view(g, &view) != PLATO_OK) throw std::runtime_error(plato_last_error());
  if (inverse) engine.reverse();
  // out-degrees of the structure the pull walks: in-degrees when transposed
  const uint32_t* deg = inverse ? view.in_degree : view.out_degree;
  const uint32_t V = engine.vertices();
  dense_state_t<double> x[2] = {engine.alloc_v_state<double>(), engine.alloc_v_state<double>()};
  double* delta = nullptr;  // the update's block partials
  uint32_t* ctrl = nullptr;
  int* unused = nullptr;
  const unsigned upd_blocks = grid_for(V, 256);
  dev_alloc(&delta, upd_blocks * sizeof(double), "trustrank delta");
  uint32_t final_epoch = 0;
  try {
    dev_alloc(&ctrl, 3 * sizeof(uint32_t), "trustrank control");
    dev_alloc(&unused, sizeof(int), "trustrank slot sum");
    check_cuda(cudaMemset(ctrl, 0, 3 * sizeof(uint32_t)), "trustrank control");
    k_tr_init<<<grid_for(V, 256), 256>>>(x[0].data(), deg, V);
    check_cuda(cudaGetLastError(), "k_tr_init");
    count_launch();
    for (uint32_t epoch = 0; epoch < kIterations; ++epoch) {
      const double* c = x[epoch & 1].data();
      double* n = x[(epoch & 1) ^ 1].data();
      k_tr_zero<<<grid_for(V, 256), 256>>>(n, V, ctrl);
      check_cuda(cudaGetLastError(), "k_tr_zero");
      const uint32_t* done = ctrl;
      engine.foreach_edges_device<double, int>(
          [c, done] __device__(const auto& context, vid_t v_i, const adj_unit_list_t& adjs) {
            if (*done) return;
            double rank_sum = 0.0;
            for (auto it = adjs.begin_; adjs.end_ != it; ++it) rank_sum += c[it->neighbour_];
            context.send(mepa_ag_message_t<double>{v_i, rank_sum});
          },
          [n] __device__(int, mepa_ag_message_t<double>& msg) -> int {
            atomicAdd(n + msg.v_i_, msg.message_);  // write_add (atomic.hpp:97-104)
            return 0;
          },
          make_combiner([] __device__(double& into, const double& from) { into += from; }), unused);
      const int last = epoch + 1 == kIterations ? 1 : 0;
      k_tr_update<<<upd_blocks, 256>>>(n, c, deg, V, kDamping, last, delta, ctrl);
      check_cuda(cudaGetLastError(), "k_tr_update");
      k_tr_control<<<1, 1024>>>(delta, upd_blocks, kEps, epoch, last, ctrl);
      check_cuda(cudaGetLastError(), "k_tr_control");
      count_launch(5);
    }
    check_cuda(cudaMemcpy(&final_epoch, ctrl + 2, sizeof(uint32_t), cudaMemcpyDeviceToHost), "trustrank control");
  } catch (...) {
    dev_free(delta);
    dev_free(ctrl);
    dev_free(unused);
    throw;
  }
  dev_free(delta);
  dev_free(ctrl);
  dev_free(unused);
  return top_ids(x[(final_epoch & 1) ^ 1].data(), view.to_external, V, k);
}

int select_seeds(plato_graph* g, const plato_trustrank_opts* o, const uint8_t* good,
                 std::vector<plato_vid_t>* seeds) {
  const uint32_t V = g->info.vertices;
  auto is_good = [good](uint32_t v) { return good == nullptr || good[v] != 0; };
  seeds->clear();
  if (static_cast<uint64_t>(g->info.max_v_i) + 1 <= o->seed_num) {  // trustrank.hpp:98-102
    for (uint32_t v = 0; v < V; ++v)
      if (is_good(v)) seeds->push_back(v);
    return PLATO_OK;
  }
  if (o->select_method == 2) {  // trustrank.hpp:124-143
    std::mt19937_64 gen(o->random_seed);
    std::uniform_int_distribution<uint32_t> dist(0, g->info.max_v_i);
    std::unordered_set<uint32_t> picked;
    while (picked.size() < o->seed_num) {
      const uint32_t v = dist(gen);
      if (picked.insert(v).second && is_good(v)) seeds->push_back(v);
    }
    std::sort(seeds->begin(), seeds->end());
    return PLATO_OK;
  }
  const uint32_t k = std::min<uint32_t>(o->seed_num, V);
  const std::vector<uint32_t> order = selection_top(g, o->select_method == 0, k);
  for (uint32_t i = 0; i < k; ++i)
    if (is_good(order[i])) seeds->push_back(order[i]);
  std::sort(seeds->begin(), seeds->end());
  return PLATO_OK;
}

}  // namespace
}  // namespace plato_b200

using namespace plato_b200;

extern "C" int plato_trustrank(plato_graph* g, const plato_trustrank_opts* opts,
                               const uint8_t* good_vertices, float* ranks, plato_vid_t* seeds_out,
                               uint32_t* n_seeds, plato_run_stats* stats) {
  if (!g || !opts) return set_error(PLATO_EINVAL, "plato_trustrank: null argument");
  if (opts->select_method > 2) return set_error(PLATO_EINVAL, "plato_trustrank: select_method must be 0, 1 or 2");
  if (opts->seed_num == 0) return set_error(PLATO_EINVAL, "plato_trustrank: seed_num must be >= 1");
  std::vector<plato_vid_t> seeds;
  {
    std::lock_guard<std::mutex> lock(g->mu);
    PLATO_CUDA_TRY(cudaSetDevice(g->device));
    PLATO_CUDA_TRY(cudaStreamSynchronize(g->stream));  // the selection runs on the default stream
    try {
      PLATO_TRY(select_seeds(g, opts, good_vertices, &seeds));
    } catch (const std::exception& e) {
      return set_error(PLATO_ECUDA, std::string("plato_trustrank: ") + e.what());
    }
  }
  if (n_seeds) *n_seeds = static_cast<uint32_t>(seeds.size());
  if (seeds_out) std::copy(seeds.begin(), seeds.end(), seeds_out);
  if (seeds.empty())
    return set_error(PLATO_EINVAL, "plato_trustrank: no good vertex among the selected seeds");
  const plato_ppr_opts po{opts->iteration, opts->damping, 0, opts->eps};
  return plato_seedset_ppr(g, seeds.data(), static_cast<uint32_t>(seeds.size()), &po, ranks, stats);
}
