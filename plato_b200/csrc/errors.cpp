// Error reporting and launch accounting of the C ABI.
#include <atomic>
#include <string>

#include "host_common.hpp"
#include "plato_b200.h"

namespace plato_b200 {

namespace {
thread_local std::string g_last_error;
std::atomic<uint64_t> g_launches{0};
}  // namespace

int set_error(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

void count_launch(uint64_t n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

}  // namespace plato_b200

extern "C" const char* plato_last_error(void) { return plato_b200::g_last_error.c_str(); }

extern "C" uint64_t plato_kernel_launches(void) {
  return plato_b200::g_launches.load(std::memory_order_relaxed);
}

extern "C" const char* plato_version(void) { return "plato_b200 0.1.0 (sm_100a)"; }
