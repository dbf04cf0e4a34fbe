// Host driver of the batched PPR kernels (batch.cuh): state buffers, seed
// index, one-iteration CUDA graphs, column admission / retirement, top-k.
// Used by plato_ppr_batch (fixed batch) and plato_server_* (continuous batching).
#pragma once

#include <vector>

#include "graph.cuh"

namespace plato_b200 {

struct batch_seed {  // one seed of one column, in caller ids
  uint32_t col;
  uint32_t vertex;
};

class batch_engine {
 public:
  explicit batch_engine(plato_graph* g) : g_(g) {}
  ~batch_engine();
  batch_engine(const batch_engine&) = delete;
  batch_engine& operator=(const batch_engine&) = delete;

  // Allocates state for K columns with kt columns per tile (kt in 8/16/32/64/128).
  int init(uint32_t K, uint32_t kt, uint32_t max_iterations, double damping, double eps,
           cudaStream_t st);
  // Starts columns `cols` with the given seed lists (seeds[i] for cols[i]).
  int admit(const std::vector<uint32_t>& cols, const std::vector<std::vector<uint32_t>>& seeds);
  // n iterations over all live columns, then one host poll; *live = columns
  // still running, retired = columns that finished during these iterations.
  int step(uint32_t* live, std::vector<uint32_t>* retired, uint32_t n = 1);
  // Top-k (caller ids, descending rank, ties by smaller id) of finished columns.
  int topk(const std::vector<uint32_t>& cols, uint32_t k, uint32_t* ids, float* vals);
  // Full rank vectors of finished columns, caller-id order, [cols.size()][V].
  int ranks(const std::vector<uint32_t>& cols, float* out);
  // Epochs each column ran.
  int iterations(std::vector<uint32_t>* out);
  // Frees the columns (state FREE); their slots may be admitted again.
  int release(const std::vector<uint32_t>& cols);

  uint32_t kt() const { return kt_; }
  uint32_t columns() const { return K_; }
  // HBM bytes per column of state (two V-vectors).
  static uint64_t bytes_per_column(uint32_t V) { return 8ull * V; }

 private:
  int capture();
  int launch_iteration(int parity);
  int rebuild_seed_index();

  plato_graph* g_;
  cudaStream_t st_ = nullptr;
  uint32_t K_ = 0, Kp_ = 0, kt_ = 0, ntiles_ = 0, rows_ = 0;
  uint32_t max_iterations_ = 0;
  uint64_t hot_l2_bytes_ = 0;  // L2 bytes of hot rows the row gathers keep (half of L2)
  double eps_ = 0.0, damping_ = 0.85;
  int cur_ = 0;
  dbuf<float> X_[2];
  dbuf<uint8_t> state_, parity_;
  dbuf<uint32_t> iters_;
  dbuf<double> delta_;
  dbuf<float> tcarry_, thead_;
  dbuf<double> partials_;
  dbuf<uint32_t> seed_off_, seed_col_;
  dbuf<float> seed_tele_;
  // seed-index build on the device: per-vertex counts, scan scratch and the
  // uploaded entry list (vertex, column, rank within the vertex, teleport)
  dbuf<uint32_t> seed_cnt_;
  dbuf<unsigned char> scan_tmp_;
  size_t scan_bytes_ = 0;
  dbuf<uint32_t> ent_v_, ent_q_, ent_r_;
  dbuf<float> ent_t_;
  // admission / release / top-k scratch (grow-only, so no allocation per request)
  dbuf<uint32_t> adm_cols_, adm_sv_, adm_sq_;
  dbuf<float> adm_init_;
  dbuf<uint32_t> tk_cols_, tk_hist_, tk_ids_, tk_undone_;
  dbuf<unsigned char> tk_state_;  // topk_col per column
  dbuf<unsigned long long> tk_cand_;
  dbuf<float> tk_vals_;
  dbuf<uint32_t> counters_;  // [0] live, [1] retired count
  dbuf<uint32_t> retired_;
  uint32_t* h_counters_ = nullptr;
  uint32_t h_counters_cap_ = 0;
  std::vector<uint32_t> h_retired_;
  // live seeds by column (internal ids), for the seed index
  std::vector<std::vector<uint32_t>> col_seeds_;
  cudaGraphExec_t exec_[2] = {nullptr, nullptr};
};

// Columns per tile chosen by measurement for this graph and batch size.
int batch_autotune(plato_graph* g, uint32_t K, cudaStream_t st, uint32_t* kt);

}  // namespace plato_b200
