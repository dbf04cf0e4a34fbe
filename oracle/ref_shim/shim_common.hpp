// shim_common.hpp — helpers shared by the oracle shim's translation units
// (test infrastructure only): one-time cluster set-up, capture of the
// reference's INFO lines, per-epoch deltas, state copies.
#pragma once

#include <cstdint>
#include <cstdio>
#include <mutex>
#include <string>
#include <vector>

#include "glog/logging.h"
#include "plato/graph/base.hpp"

namespace plato_ref_shim {

// captured log lines of the current call (defined in plato_ref_shim.cpp)
extern std::mutex g_log_mu;
extern std::vector<std::string> g_lines;

inline void capture(int severity, const char* text) {
  if (severity != 0) return;
  std::lock_guard<std::mutex> lock(g_log_mu);
  g_lines.emplace_back(text);
}

inline void start_capture() {
  std::lock_guard<std::mutex> lock(g_log_mu);
  g_lines.clear();
  plato_shim_log_sink() = &capture;
}

inline std::vector<std::string> stop_capture() {
  std::lock_guard<std::mutex> lock(g_log_mu);
  plato_shim_log_sink() = nullptr;
  return std::move(g_lines);
}

inline void init_once() {
  static std::once_flag once;
  std::call_once(once, [] {
    int argc = 1;
    static char name[] = "plato_ref_shim";
    static char* args[] = {name, nullptr};
    char** argv = args;
    plato::cluster_info_t::get_instance().initialize(&argc, &argv);
  });
}

template <typename STATE>
void copy_out(const STATE& st, uint32_t V, double* out) {
  for (uint32_t v = 0; v < V; ++v) out[v] = st[v];
}

template <typename STATE>
void copy_out_u32(const STATE& st, uint32_t V, uint32_t* out) {
  for (uint32_t v = 0; v < V; ++v) out[v] = st[v];
}

// "[epoch-i], delta: X, ..." lines (pagerank.hpp:141-144 and the like)
inline uint32_t epoch_deltas(const std::vector<std::string>& lines, double* deltas, uint32_t cap) {
  uint32_t n = 0;
  for (const auto& l : lines) {
    int e = 0;
    double d = 0.0;
    if (std::sscanf(l.c_str(), "[epoch-%d], delta: %lf", &e, &d) == 2) {
      if (deltas && n < cap) deltas[n] = d;
      ++n;
    }
  }
  return n;
}

}  // namespace plato_ref_shim
