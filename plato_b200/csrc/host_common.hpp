// Host-side helpers shared by every translation unit of libplato_b200:
// thread-local last-error message and the kernel launch counter.
#pragma once

#include <atomic>
#include <cstdint>
#include <cstdio>
#include <string>

namespace plato_b200 {

// Records `msg` as the calling thread's last error and returns `code`.
int set_error(int code, const std::string& msg);
// Counts one kernel launch (reported by plato_kernel_launches()).
void count_launch(uint64_t n = 1);

}  // namespace plato_b200
