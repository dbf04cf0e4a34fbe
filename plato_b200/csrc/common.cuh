// Shared CUDA helpers for libplato_b200 (sm_100a only).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "host_common.hpp"
#include "plato_b200.h"

#define PLATO_TRY(expr)                    \
  do {                                     \
    int plato_s_ = (expr);                 \
    if (plato_s_ != PLATO_OK) return plato_s_; \
  } while (0)

#define PLATO_CUDA_TRY(call)                                                        \
  do {                                                                              \
    cudaError_t plato_e_ = (call);                                                  \
    if (plato_e_ != cudaSuccess)                                                    \
      return ::plato_b200::set_error(PLATO_ECUDA, std::string(#call) + " failed: " + \
                                                      cudaGetErrorString(plato_e_)); \
  } while (0)

// Call right after a <<<...>>> launch: counts it and surfaces launch errors.
#define PLATO_LAUNCHED(name)                                                            \
  do {                                                                                  \
    ::plato_b200::count_launch();                                                       \
    cudaError_t plato_e_ = cudaGetLastError();                                          \
    if (plato_e_ != cudaSuccess)                                                        \
      return ::plato_b200::set_error(PLATO_ECUDA, std::string("launch of ") + (name) +   \
                                                      " failed: " + cudaGetErrorString(plato_e_)); \
  } while (0)

namespace plato_b200 {

constexpr int kWarp = 32;
constexpr int kNumSMs = 148;  // B200; the runtime value is queried where it matters

// Device buffer owned by the library (cudaMalloc / cudaFree), move-only.
template <typename T>
struct dbuf {
  T* p = nullptr;
  size_t n = 0;
  dbuf() = default;
  dbuf(const dbuf&) = delete;
  dbuf& operator=(const dbuf&) = delete;
  dbuf(dbuf&& o) noexcept : p(o.p), n(o.n) { o.p = nullptr; o.n = 0; }
  dbuf& operator=(dbuf&& o) noexcept {
    if (this != &o) { release(); p = o.p; n = o.n; o.p = nullptr; o.n = 0; }
    return *this;
  }
  ~dbuf() { release(); }
  int alloc(size_t count) {
    if (count <= n && p) return PLATO_OK;
    release();
    if (count == 0) return PLATO_OK;
    cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&p), count * sizeof(T));
    if (e != cudaSuccess) {
      p = nullptr;
      cudaGetLastError();
      return set_error(e == cudaErrorMemoryAllocation ? PLATO_ENOMEM : PLATO_ECUDA,
                       std::string("cudaMalloc of ") + std::to_string(count * sizeof(T)) +
                           " bytes failed: " + cudaGetErrorString(e));
    }
    n = count;
    return PLATO_OK;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  size_t bytes() const { return n * sizeof(T); }
};

inline unsigned grid_for(uint64_t items, unsigned block, unsigned max_blocks = 148u * 16u) {
  uint64_t g = (items + block - 1) / block;
  if (g < 1) g = 1;
  if (g > max_blocks) g = max_blocks;
  return static_cast<unsigned>(g);
}

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ unsigned long long warp_sum(unsigned long long v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Block-wide sum of a double; result valid in thread 0. `scratch` >= 32 doubles.
template <int NT>
__device__ __forceinline__ double block_sum(double v, double* scratch) {
  v = warp_sum(v);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) scratch[wid] = v;
  __syncthreads();
  double r = 0.0;
  if (wid == 0) {
    r = (lane < NT / 32) ? scratch[lane] : 0.0;
    r = warp_sum(r);
  }
  __syncthreads();
  return r;
}

template <int NT>
__device__ __forceinline__ unsigned long long block_sum_u64(unsigned long long v,
                                                            unsigned long long* scratch) {
  v = warp_sum(v);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) scratch[wid] = v;
  __syncthreads();
  unsigned long long r = 0;
  if (wid == 0) {
    r = (lane < NT / 32) ? scratch[lane] : 0ull;
    r = warp_sum(r);
  }
  __syncthreads();
  return r;
}

}  // namespace plato_b200
