// RAII event bracket around one kernel launch (active only when profiling is on).
#pragma once

#include <cuda_runtime.h>

namespace plato_b200 {

bool profile_on();

class prof_scope {
 public:
  prof_scope(const char* name, cudaStream_t st);
  ~prof_scope();
  prof_scope(const prof_scope&) = delete;
  prof_scope& operator=(const prof_scope&) = delete;

 private:
  const char* name_;
  cudaStream_t st_;
  cudaEvent_t a_ = nullptr, b_ = nullptr;
};

}  // namespace plato_b200
