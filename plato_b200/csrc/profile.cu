// Event-based kernel timing for the hot kernels (opt-in, see plato_profile_*).
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

#include "common.cuh"
#include "profile.cuh"

namespace plato_b200 {
namespace {

struct kernel_record {
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> pending;
  double total_ms = 0.0;
  uint64_t launches = 0;
};

std::mutex g_mu;
bool g_on = false;
std::unordered_map<std::string, kernel_record> g_records;

void drain(kernel_record& r) {
  for (auto& ev : r.pending) {
    float ms = 0.f;
    if (cudaEventSynchronize(ev.second) == cudaSuccess &&
        cudaEventElapsedTime(&ms, ev.first, ev.second) == cudaSuccess)
      r.total_ms += ms;
    cudaEventDestroy(ev.first);
    cudaEventDestroy(ev.second);
    ++r.launches;
  }
  r.pending.clear();
}

}  // namespace

bool profile_on() { return g_on; }

prof_scope::prof_scope(const char* name, cudaStream_t st) : name_(name), st_(st) {
  if (!g_on) return;
  if (cudaEventCreate(&a_) != cudaSuccess || cudaEventCreate(&b_) != cudaSuccess) {
    a_ = b_ = nullptr;
    return;
  }
  cudaEventRecord(a_, st_);
}

prof_scope::~prof_scope() {
  if (!a_) return;
  cudaEventRecord(b_, st_);
  std::lock_guard<std::mutex> lock(g_mu);
  auto& r = g_records[name_];
  r.pending.emplace_back(a_, b_);
  if (r.pending.size() > 4096) drain(r);
}

}  // namespace plato_b200

using namespace plato_b200;

extern "C" int plato_profile_enable(int on) {
  std::lock_guard<std::mutex> lock(g_mu);
  g_on = on != 0;
  return PLATO_OK;
}

extern "C" int plato_profile_reset(void) {
  std::lock_guard<std::mutex> lock(g_mu);
  for (auto& kv : g_records) {
    drain(kv.second);
    kv.second.total_ms = 0.0;
    kv.second.launches = 0;
  }
  return PLATO_OK;
}

extern "C" int plato_profile_read(const char* kernel, double* total_ms, uint64_t* launches) {
  if (!kernel) return set_error(PLATO_EINVAL, "plato_profile_read: null kernel name");
  std::lock_guard<std::mutex> lock(g_mu);
  auto it = g_records.find(kernel);
  if (it == g_records.end()) {
    if (total_ms) *total_ms = 0.0;
    if (launches) *launches = 0;
    return PLATO_OK;
  }
  drain(it->second);
  if (total_ms) *total_ms = it->second.total_ms;
  if (launches) *launches = it->second.launches;
  return PLATO_OK;
}
