// Reference-shaped functors on the header-only dualmode engine.
//
// Test infrastructure: built into tests/engine/libengine_kat.so and driven by
// tests/test_gpu_engine.py.  Each entry point restates one reference client
// of dualmode_engine_t::foreach_edges with the same functor bodies:
//   kat_aggregate   plato/graph/test/message_passing.cc:62-87 (AggregateMessage),
//                   also on the combined pull (messages of a vertex summed)
//   kat_pagerank    plato/algo/pagerank/pagerank.hpp:81-146 (double state, write_add),
//                   on the 64-edge or the combined pull, on the graph or its
//                   transpose (engine.reverse())
//   kat_bfs         plato/algo/bfs/bfs.hpp:70-151 (CAS parents, push/pull switch)
#include <cstdio>
#include <exception>

#include "plato_b200/dualmode.cuh"

using namespace plato_b200;

namespace {
thread_local std::string g_err;
int fail(const std::exception& e) {
  g_err = e.what();
  return 1;
}
}  // namespace

extern "C" const char* kat_error() { return g_err.c_str(); }

extern "C" int kat_aggregate(plato_graph* g, int combined, int32_t* values_out, int64_t* sum_out) {
  try {
    dualmode_engine_t engine(g);
    auto values = engine.alloc_v_state<int32_t>();
    values.fill(0);
    int32_t* vals = values.data();
    auto signal = [] __device__(const auto& context, vid_t v_i, const adj_unit_list_t& adjs) {
      for (auto it = adjs.begin_; adjs.end_ != it; ++it) context.send(mepa_ag_message_t<uint32_t>{v_i, 1});
    };
    auto slot = [vals] __device__(int, mepa_ag_message_t<uint32_t>& msg) -> int32_t {
      atomicAdd(vals + msg.v_i_, static_cast<int32_t>(msg.message_));
      return static_cast<int32_t>(msg.message_);  // the messages this call stands for
    };
    const int32_t sum =
        combined ? engine.foreach_edges<uint32_t, int32_t>(
                       signal, slot, make_combiner([] __device__(uint32_t& a, const uint32_t& b) { a += b; }))
                 : engine.foreach_edges<uint32_t, int32_t>(signal, slot);
    auto h = engine.to_host(values);
    for (size_t i = 0; i < h.size(); ++i) values_out[i] = h[i];
    *sum_out = sum;
    return 0;
  } catch (const std::exception& e) {
    return fail(e);
  }
}

extern "C" int kat_pagerank(plato_graph* g, uint32_t iterations, double damping, int combined, int reversed,
                            double* out) {
  try {
    dualmode_engine_t engine(g);
    if (reversed) engine.reverse();
    auto curt = engine.alloc_v_state<double>();
    auto next = engine.alloc_v_state<double>();
    const uint32_t V = engine.vertices();
    // out-degrees of the direction the pull walks (in-degrees on the transpose)
    plato_graph_device_view view{};
    plato_graph_get_device_view(g, &view);
    const uint32_t* odeg = reversed ? view.in_degree : engine.out_degrees();
    // x = 1 / deg (pagerank.hpp:90-98): done with a push-only sweep over all vertices
    auto all = engine.alloc_v_subset();
    {
      std::vector<uint32_t> w((V + 31) / 32, 0xFFFFFFFFu);
      if (V % 32) w.back() = (1u << (V % 32)) - 1u;
      check_cuda(cudaMemcpy(all.data(), w.data(), 4 * w.size(), cudaMemcpyHostToDevice), "all");
    }
    double* c = curt.data();
    double* n = next.data();
    const double d = damping;
    engine.foreach_edges<int, int>(
        [c, odeg] __device__(const auto&, vid_t v) { c[v] = odeg[v] > 0 ? 1.0 / odeg[v] : 1.0; },
        [] __device__(int, int&) -> int { return 0; }, all);
    for (uint32_t epoch = 0; epoch < iterations; ++epoch) {
      next.fill(0.0);
      auto signal = [c] __device__(const auto& context, vid_t v_i, const adj_unit_list_t& adjs) {
        double rank_sum = 0.0;
        for (auto it = adjs.begin_; adjs.end_ != it; ++it) rank_sum += c[it->neighbour_];
        context.send(mepa_ag_message_t<double>{v_i, rank_sum});
      };
      auto slot = [n] __device__(int, mepa_ag_message_t<double>& msg) -> int {
        atomicAdd(n + msg.v_i_, msg.message_);  // write_add (atomic.hpp:97-104)
        return 0;
      };
      if (combined)
        engine.foreach_edges<double, int>(signal, slot,
                                          make_combiner([] __device__(double& a, const double& b) { a += b; }));
      else
        engine.foreach_edges<double, int>(signal, slot);
      const bool last = epoch + 1 == iterations;
      engine.foreach_edges<int, int>(
          [n, odeg, d, last] __device__(const auto&, vid_t v) {
            n[v] = 1.0 - d + d * n[v];
            if (!last && odeg[v] > 0) n[v] = n[v] / odeg[v];
          },
          [] __device__(int, int&) -> int { return 0; }, all);
      std::swap(c, n);
      std::swap(curt, next);
      c = curt.data();
      n = next.data();
    }
    auto h = engine.to_host(curt);
    for (size_t i = 0; i < h.size(); ++i) out[i] = h[i];
    return 0;
  } catch (const std::exception& e) {
    return fail(e);
  }
}

extern "C" int kat_bfs(plato_graph* g, uint32_t root_ext, uint32_t* levels_out, uint64_t* visited_out,
                       uint64_t* trace_out) {
  try {
    dualmode_engine_t engine(g);
    const uint32_t V = engine.vertices();
    const vid_t root = engine.to_internal(root_ext);
    auto visited = engine.alloc_v_subset();
    auto active_current = engine.alloc_v_subset();
    auto active_next = engine.alloc_v_subset();
    auto parent = engine.alloc_v_state<vid_t>();
    auto level = engine.alloc_v_state<uint32_t>();
    const vid_t invalid_parent = engine.graph_info().max_v_i + 1;  // bfs.hpp:79
    parent.fill(invalid_parent);
    level.fill(0xFFFFFFFFu);
    check_cuda(cudaMemcpy(parent.data() + root, &root, 4, cudaMemcpyHostToDevice), "root");
    const uint32_t zero = 0;
    check_cuda(cudaMemcpy(level.data() + root, &zero, 4, cudaMemcpyHostToDevice), "root");
    visited.set_bit_host(root);
    active_current.set_bit_host(root);
    vid_t* par = parent.data();
    uint32_t* lev = level.data();
    const out_edges_view out_edges = engine.out_edges();
    uint64_t trace = 0;
    vid_t actives = 1;
    for (uint32_t epoch = 0; actives != 0; ++epoch) {
      active_next.clear();
      const auto nxt = active_next.dev();
      const auto vis = visited.dev();
      const auto cur = active_current.dev();
      const uint32_t lvl = epoch + 1;
      actives = engine.foreach_edges<vid_t, vid_t>(
          [] __device__(const auto& context, vid_t v_i) { context.send(v_i); },
          [=] __device__(int, vid_t& msg) -> vid_t {
            vid_t activated = 0;
            auto neighbours = out_edges.neighbours(msg);
            for (auto it = neighbours.begin_; neighbours.end_ != it; ++it) {
              const vid_t dst = it->neighbour_;
              if (par[dst] == invalid_parent && atomicCAS(par + dst, invalid_parent, msg) == invalid_parent) {
                lev[dst] = lvl;
                nxt.set_bit(dst);
                vis.set_bit(dst);
                ++activated;
              }
            }
            return activated;
          },
          [=] __device__(const auto& context, vid_t v_i, const adj_unit_list_t& adjs) {
            if (vis.get_bit(v_i)) return;
            for (auto it = adjs.begin_; adjs.end_ != it; ++it) {
              const vid_t src = it->neighbour_;
              if (cur.get_bit(src)) {
                context.send(mepa_ag_message_t<vid_t>{v_i, src});
                break;
              }
            }
          },
          [=] __device__(int, mepa_ag_message_t<vid_t>& msg) -> vid_t {
            if (atomicCAS(par + msg.v_i_, invalid_parent, msg.message_) == invalid_parent) {
              lev[msg.v_i_] = lvl;
              nxt.set_bit(msg.v_i_);
              vis.set_bit(msg.v_i_);
              return 1;
            }
            return 0;
          },
          active_current);
      if (engine.last_was_push() && epoch < 64) trace |= 1ull << epoch;
      std::swap(active_current, active_next);
    }
    auto h = engine.to_host(level);
    for (uint32_t i = 0; i < V; ++i) levels_out[i] = h[i];
    *visited_out = visited.count();
    *trace_out = trace;
    return 0;
  } catch (const std::exception& e) {
    return fail(e);
  }
}
