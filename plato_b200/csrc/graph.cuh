// Resident graph object: CSC (in-edges) + CSR (out-edges) in HBM, internal
// vertex order, plus lazily built per-algorithm metadata and workspaces.
#pragma once

#include <map>
#include <memory>
#include <mutex>
#include <vector>

#include "common.cuh"

namespace plato_b200 {

// Merge-path partition of the CSC into tiles of `items` (vertices + edges)
// merge items each: tile t covers vertices [row[t], row[t+1]] and edges
// [edge[t], edge[t+1]).  Static per graph and tile size.
struct merge_tiles {
  uint32_t items = 0;
  uint32_t count = 0;
  dbuf<uint32_t> row;   // [count + 1]
  dbuf<uint64_t> edge;  // [count + 1]
};

struct rank_workspace;   // rank.cu
struct bfs_workspace;    // bfs.cu
class batch_engine;      // ppr_batch.cu
struct hll_workspace;    // hll.cu
void destroy_rank_workspace(rank_workspace*);
void destroy_bfs_workspace(bfs_workspace*);
void destroy_hll_workspace(hll_workspace*);
void destroy_batch_engine(batch_engine*);

}  // namespace plato_b200

struct plato_graph {
  int device = 0;
  plato_graph_info info{};
  uint64_t stored_edges = 0;  // directed edges held in CSC/CSR
  bool relabeled = false;

  plato_b200::dbuf<uint64_t> in_off, out_off;
  plato_b200::dbuf<uint32_t> in_adj, out_adj;
  plato_b200::dbuf<uint32_t> out_deg, in_deg;
  plato_b200::dbuf<uint32_t> to_int, to_ext;  // empty when not relabeled
  bool weighted = false;
  plato_b200::dbuf<float> in_w;      // [E] weight of each CSC edge (weighted graphs)
  plato_b200::dbuf<float> out_wsum;  // [V] sum of each vertex's out-edge weights

  cudaStream_t stream = nullptr;  // stream of the host-buffer entry points
  std::mutex mu;                  // one algorithm call at a time per graph

  std::map<uint32_t, plato_b200::merge_tiles> tiles;  // merge-path tiles by items per tile
  plato_b200::rank_workspace* rank_ws = nullptr;
  plato_b200::bfs_workspace* bfs_ws = nullptr;
  plato_b200::hll_workspace* hll_ws = nullptr;  // HyperLogLog buffers (hll.cu)
  plato_b200::batch_engine* batch_cache = nullptr;  // plato_ppr_batch state, kept between calls
  std::vector<uint32_t> h_to_int;             // host copy of to_int (lazily)
  std::map<uint32_t, uint32_t> batch_tuned;   // K bucket -> columns per tile (kt)

  ~plato_graph();
};

namespace plato_b200 {

// Builds (once) the merge-path tiles of the CSC for `items` per tile.
int ensure_pull_tiles(plato_graph* g, uint32_t items, cudaStream_t st,
                      const merge_tiles** out = nullptr);

// out_ext[to_ext[i]] = in_int[i] (identity when the graph is not relabeled).
int scatter_to_external_f32(const plato_graph* g, const float* in_int, float* out_ext,
                            cudaStream_t st);
int scatter_to_external_u32(const plato_graph* g, const uint32_t* in_int, uint32_t* out_ext,
                            cudaStream_t st);

inline uint32_t to_internal_host(const plato_graph* g, uint32_t v, const uint32_t* h_to_int) {
  return (g->relabeled && h_to_int) ? h_to_int[v] : v;
}

// Maps one caller id to the internal id (device lookup, synchronous).
int lookup_internal(const plato_graph* g, uint32_t ext, uint32_t* internal, cudaStream_t st);

// Host copy of to_int (caller id -> internal id), fetched once per graph.
int host_to_internal(plato_graph* g, const std::vector<uint32_t>** map, cudaStream_t st);

}  // namespace plato_b200
