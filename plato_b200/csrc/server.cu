// Continuous-batching personalized PageRank server.
//
// Each live query owns one column (slot) of a batch_engine.  A server step
//   1. admits queued requests into free slots (zeroed column + seeds),
//   2. runs one iteration over every live column (one CUDA graph replay),
//   3. retires the columns that finished their final epoch: on-device top-k,
//      result queued for plat_server_poll, slot freed.
// Requests that arrive while others are running join at the next step, so
// their iterations overlap on the device with the older queries'.  Each
// column's arithmetic is independent of which other columns are live (the
// per-column sums run in a fixed order over the same tiles), so a query's
// result does not depend on the mix it ran in.
// The number of slots is bounded by the HBM budget: each slot costs two
// V-float columns of state.
#include <deque>
#include <mutex>
#include <new>
#include <vector>

#include "batch_engine.hpp"

namespace {

struct pending {
  uint64_t id;
  std::vector<uint32_t> seeds;
};

struct finished {
  uint64_t id;
  std::vector<uint32_t> ids;
  std::vector<float> vals;
  uint32_t iterations;
};

}  // namespace

struct plato_server {
  plato_graph* g = nullptr;
  plato_server_opts opts{};
  plato_b200::batch_engine* eng = nullptr;
  uint32_t slots = 0;
  std::vector<int64_t> slot_req;  // request id per slot, -1 = free
  std::deque<pending> queue;
  std::deque<finished> done;
  uint64_t next_id = 1;
  uint64_t completed = 0;
  uint32_t live = 0;
  std::mutex mu;
  ~plato_server() { delete eng; }
};

using namespace plato_b200;

extern "C" int plato_server_create(plato_graph* g, const plato_server_opts* opts,
                                   plato_server** out) {
  if (!g || !opts || !out) return set_error(PLATO_EINVAL, "plato_server_create: null argument");
  *out = nullptr;
  if (opts->max_slots == 0) return set_error(PLATO_EINVAL, "plato_server_create: max_slots 0");
  if (opts->topk == 0 || opts->topk > 1024)
    return set_error(PLATO_EINVAL, "plato_server_create: topk must be in [1, 1024]");
  const uint64_t per = batch_engine::bytes_per_column(g->info.vertices);
  const uint64_t by_budget = opts->hbm_budget_bytes / per;
  if (by_budget == 0)
    return set_error(PLATO_ENOMEM, "plato_server_create: HBM budget below one query's state");
  auto* s = new (std::nothrow) plato_server();
  if (!s) return set_error(PLATO_ENOMEM, "plato_server_create: host allocation failed");
  s->g = g;
  s->opts = *opts;
  s->slots = static_cast<uint32_t>(std::min<uint64_t>(opts->max_slots, by_budget));
  std::lock_guard<std::mutex> glock(g->mu);
  int rc = PLATO_OK;
  do {
    if (cudaSetDevice(g->device) != cudaSuccess) {
      rc = set_error(PLATO_ECUDA, "plato_server_create: cudaSetDevice failed");
      break;
    }
    uint32_t kt = 0;
    rc = batch_autotune(g, s->slots, g->stream, &kt);
    if (rc != PLATO_OK) break;
    s->eng = new (std::nothrow) batch_engine(g);
    if (!s->eng) {
      rc = set_error(PLATO_ENOMEM, "plato_server_create: host allocation failed");
      break;
    }
    rc = s->eng->init(s->slots, kt, opts->max_iterations, opts->damping, opts->eps, g->stream);
  } while (false);
  if (rc != PLATO_OK) {
    delete s;
    return rc;
  }
  s->slot_req.assign(s->slots, -1);
  *out = s;
  return PLATO_OK;
}

extern "C" int plato_server_submit(plato_server* s, const plato_vid_t* seeds, uint32_t n,
                                   uint64_t* request_id) {
  if (!s || !seeds || !request_id) return set_error(PLATO_EINVAL, "plato_server_submit: null argument");
  if (n == 0) return set_error(PLATO_EINVAL, "plato_server_submit: empty seed set");
  for (uint32_t i = 0; i < n; ++i)
    if (seeds[i] >= s->g->info.vertices)
      return set_error(PLATO_EINVAL, "plato_server_submit: seed vertex out of range");
  std::lock_guard<std::mutex> lock(s->mu);
  pending p;
  p.id = s->next_id++;
  p.seeds.assign(seeds, seeds + n);
  s->queue.push_back(std::move(p));
  *request_id = s->queue.back().id;
  return PLATO_OK;
}

extern "C" int plato_server_step(plato_server* s) {
  if (!s) return set_error(PLATO_EINVAL, "plato_server_step: null server");
  std::lock_guard<std::mutex> lock(s->mu);
  std::lock_guard<std::mutex> glock(s->g->mu);
  PLATO_CUDA_TRY(cudaSetDevice(s->g->device));
  // 1. admission into free slots
  std::vector<uint32_t> cols;
  std::vector<std::vector<uint32_t>> seeds;
  for (uint32_t q = 0; q < s->slots && !s->queue.empty(); ++q) {
    if (s->slot_req[q] >= 0) continue;
    pending& p = s->queue.front();
    s->slot_req[q] = static_cast<int64_t>(p.id);
    cols.push_back(q);
    seeds.push_back(std::move(p.seeds));
    s->queue.pop_front();
  }
  if (!cols.empty()) {
    const int rc = s->eng->admit(cols, seeds);
    if (rc != PLATO_OK) return rc;
    s->live += static_cast<uint32_t>(cols.size());
  }
  if (s->live == 0) return PLATO_OK;
  // 2. one iteration over every live column
  uint32_t live = 0;
  std::vector<uint32_t> retired;
  PLATO_TRY(s->eng->step(&live, &retired));
  s->live = live;
  if (retired.empty()) return PLATO_OK;
  // 3. retire: top-k, results, free the slots
  const uint32_t k = s->opts.topk;
  std::vector<uint32_t> ids(retired.size() * k);
  std::vector<float> vals(retired.size() * k);
  PLATO_TRY(s->eng->topk(retired, k, ids.data(), vals.data()));
  std::vector<uint32_t> iters;
  PLATO_TRY(s->eng->iterations(&iters));
  for (size_t i = 0; i < retired.size(); ++i) {
    const uint32_t q = retired[i];
    finished f;
    f.id = static_cast<uint64_t>(s->slot_req[q]);
    f.ids.assign(ids.begin() + i * k, ids.begin() + (i + 1) * k);
    f.vals.assign(vals.begin() + i * k, vals.begin() + (i + 1) * k);
    f.iterations = iters[q];
    s->done.push_back(std::move(f));
    s->slot_req[q] = -1;
    ++s->completed;
  }
  return s->eng->release(retired);
}

extern "C" int plato_server_poll(plato_server* s, uint64_t* request_id, plato_vid_t* topk_ids,
                                 float* topk_vals, uint32_t* iterations) {
  if (!s || !request_id) return set_error(PLATO_EINVAL, "plato_server_poll: null argument");
  std::lock_guard<std::mutex> lock(s->mu);
  if (s->done.empty()) return PLATO_ENOTFOUND;
  finished& f = s->done.front();
  *request_id = f.id;
  if (topk_ids) std::copy(f.ids.begin(), f.ids.end(), topk_ids);
  if (topk_vals) std::copy(f.vals.begin(), f.vals.end(), topk_vals);
  if (iterations) *iterations = f.iterations;
  s->done.pop_front();
  return PLATO_OK;
}

extern "C" int plato_server_stats(const plato_server* s, uint32_t* live, uint32_t* queued,
                                  uint64_t* completed) {
  if (!s) return set_error(PLATO_EINVAL, "plato_server_stats: null server");
  auto* m = const_cast<plato_server*>(s);
  std::lock_guard<std::mutex> lock(m->mu);
  uint32_t occupied = 0;
  for (int64_t r : m->slot_req) occupied += (r >= 0);
  if (live) *live = occupied;
  if (queued) *queued = static_cast<uint32_t>(m->queue.size());
  if (completed) *completed = m->completed;
  return PLATO_OK;
}

extern "C" int plato_server_destroy(plato_server* s) {
  if (!s) return PLATO_OK;
  {
    std::lock_guard<std::mutex> glock(s->g->mu);
    cudaSetDevice(s->g->device);
    cudaStreamSynchronize(s->g->stream);
    delete s->eng;
    s->eng = nullptr;
  }
  delete s;
  return PLATO_OK;
}
