/*
 * ref_cpu.c — CPU restatement of the reference's dual-mode engine path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the oracle: tests, the smoke check
 * and bench.py's CPU-baseline leg call it to check or time against.  Nothing
 * in the plato_b200 package links or calls it.
 *
 * It restates, at one partition (mpirun -np 1) and in double precision, what
 * the reference computes (the reference itself cannot be built here: it needs
 * MPI, glog, gflags, boost, yas and bazel):
 *   graph      DCSC of in-edges with only non-empty columns
 *              (plato/graph/structure/dcsc.hpp:148-152, build :201-348, undirected
 *              doubling :365-385) and BCSR of out-edges with a row bitmap
 *              (plato/graph/structure/bcsr.hpp:167-174, :243-376)
 *   degrees    generate_dense_out_degrees_fg from the in-edges
 *              (plato/graph/structure.hpp:291-346)
 *   engine     dualmode_engine_t::foreach_edges switch
 *              (plato/engine/dualmode.hpp:245-297): push iff
 *              active_edges / edges < push_threshold, edges doubled when undirected
 *   pagerank   plato/algo/pagerank/pagerank.hpp:81-146
 *   ppr        plato/algo/ppr/personalized_pagerank.hpp:61-131 (pull-only)
 *              and :158-272 (push/pull, sticky switch on active_edges > edges/20)
 *   seed sets  plato/algo/trustrank/trustrank.hpp:194-256 (explicit seeds)
 *   bfs        plato/algo/bfs/bfs.hpp:70-151, levels = epoch + 1
 *   write_add  CAS loop on doubles (plato/util/atomic.hpp:97-104)
 *   bitmaps    64-bit words (plato/util/bitmap.hpp:43-350)
 * The MPI message transport (bsp.hpp, broadcast.hpp) is a self-send at one
 * partition; it is replaced by direct calls of the slot functions.
 *
 * Parity status: the reference ships no golden vectors for pagerank, ppr,
 * bfs or trustrank results, so the algorithm outputs are unpinned by the
 * reference's own tests; the graph substrate (DCSC column/edge counts,
 * out-degrees, aggregate-message sums) is pinned against the reference's
 * substrate tests (tests/golden/).
 */
#include <math.h>
#include <omp.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define EXPORT __attribute__((visibility("default")))

typedef struct {
  uint32_t vertices;      /* graph_info.vertices_ */
  uint32_t max_v_i;
  uint64_t input_edges;   /* graph_info.edges_    */
  int is_directed;
  /* DCSC (in-edges) */
  uint64_t nnzcol;
  uint64_t* col_index;    /* [nnzcol + 1] index_        */
  uint32_t* col_vertex;   /* [nnzcol]     local_vertex_ */
  uint32_t* in_adjs;      /* [E]          adjs_ (sources) */
  /* BCSR (out-edges) */
  uint64_t* row_bitmap;   /* rows with out-edges */
  uint64_t* row_index;    /* [V + 1] */
  uint32_t* out_adjs;     /* [E] */
  uint64_t stored_edges;
  uint32_t* out_degree;   /* from in-edges */
  /* rank-loop state kept between calls (two V-vectors and two bitmaps), so a
   * timed call is the epochs alone, like the device side's resident state */
  double* ws_a;
  double* ws_b;
  uint64_t* ws_actives;
  uint64_t* ws_walk;
} ref_graph;

/* ---------------- bitmap (bitmap.hpp) ------------------------------------ */
static inline void bm_set(uint64_t* b, uint32_t v) {
  __atomic_fetch_or(&b[v >> 6], 1ull << (v & 63), __ATOMIC_RELAXED);
}
static inline int bm_get(const uint64_t* b, uint32_t v) { return (b[v >> 6] >> (v & 63)) & 1ull; }
static inline uint64_t bm_words(uint32_t n) { return ((uint64_t)n + 63) / 64 + 1; }

/* ---------------- atomics (atomic.hpp) ------------------------------------ */
static inline void write_add(double* p, double v) {
  const uint64_t ob0 = __atomic_load_n((uint64_t*)p, __ATOMIC_RELAXED);
  double old;
  memcpy(&old, &ob0, 8);
  for (;;) {
    double nv = old + v;
    uint64_t ob, nb;
    memcpy(&ob, &old, 8);
    memcpy(&nb, &nv, 8);
    if (__atomic_compare_exchange_n((uint64_t*)p, &ob, nb, 0, __ATOMIC_RELAXED, __ATOMIC_RELAXED))
      return;
    memcpy(&old, &ob, 8);
  }
}
static inline int cas_u32(uint32_t* p, uint32_t expect, uint32_t val) {
  return __atomic_compare_exchange_n(p, &expect, val, 0, __ATOMIC_RELAXED, __ATOMIC_RELAXED);
}

/* ---------------- graph build --------------------------------------------- */
static int cmp_u32(const void* a, const void* b) {
  const uint32_t x = *(const uint32_t*)a, y = *(const uint32_t*)b;
  return (x > y) - (x < y);
}

/* Counting sort by key (stable), so each adjacency list keeps input order;
 * inputs sorted by (src, dst) give ascending adjacency lists. */
EXPORT ref_graph* ref_graph_build(uint32_t V, uint64_t n, const uint32_t* src, const uint32_t* dst,
                                  int is_directed) {
  ref_graph* g = (ref_graph*)calloc(1, sizeof(ref_graph));
  if (!g) return NULL;
  g->vertices = V;
  g->max_v_i = V ? V - 1 : 0;
  g->input_edges = n;
  g->is_directed = is_directed;
  const uint64_t E = is_directed ? n : 2 * n;
  g->stored_edges = E;
  uint64_t* in_cnt = (uint64_t*)calloc((size_t)V + 1, 8);
  uint64_t* out_cnt = (uint64_t*)calloc((size_t)V + 1, 8);
  g->in_adjs = (uint32_t*)malloc((E ? E : 1) * 4);
  g->out_adjs = (uint32_t*)malloc((E ? E : 1) * 4);
  g->row_index = (uint64_t*)calloc((size_t)V + 1, 8);
  g->row_bitmap = (uint64_t*)calloc(bm_words(V), 8);
  g->out_degree = (uint32_t*)calloc(V ? V : 1, 4);
  for (uint64_t i = 0; i < n; ++i) {
    in_cnt[dst[i]]++;
    out_cnt[src[i]]++;
    if (!is_directed) {
      in_cnt[src[i]]++;
      out_cnt[dst[i]]++;
    }
  }
  /* CSC offsets over all vertices, then compress empty columns (DCSC) */
  uint64_t* in_off = (uint64_t*)calloc((size_t)V + 1, 8);
  for (uint32_t v = 0; v < V; ++v) in_off[v + 1] = in_off[v] + in_cnt[v];
  for (uint32_t v = 0; v < V; ++v) g->row_index[v + 1] = g->row_index[v] + out_cnt[v];
  uint64_t* in_pos = (uint64_t*)malloc(((size_t)V + 1) * 8);
  uint64_t* out_pos = (uint64_t*)malloc(((size_t)V + 1) * 8);
  memcpy(in_pos, in_off, ((size_t)V + 1) * 8);
  memcpy(out_pos, g->row_index, ((size_t)V + 1) * 8);
  /* directed edges in (src, dst) order; the reversed copies of an undirected
   * graph are placed so that every list stays ascending when the input is
   * sorted: process all (u -> v) edges in ascending (u, v) of the stored set. */
  if (is_directed) {
    for (uint64_t i = 0; i < n; ++i) {
      g->in_adjs[in_pos[dst[i]]++] = src[i];
      g->out_adjs[out_pos[src[i]]++] = dst[i];
    }
  } else {
    /* stored edges are {(s,d), (d,s)}; emit in ascending source order by
     * walking sources: first build the out lists, then derive in lists. */
    for (uint64_t i = 0; i < n; ++i) {
      g->out_adjs[out_pos[src[i]]++] = dst[i];
      g->out_adjs[out_pos[dst[i]]++] = src[i];
    }
    /* sort each out list (already ascending for (min, max)-sorted input) */
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t v = 0; v < (int64_t)V; ++v) {
      uint32_t* a = g->out_adjs + g->row_index[v];
      const uint64_t m = g->row_index[v + 1] - g->row_index[v];
      int sorted = 1;
      for (uint64_t x = 1; x < m && sorted; ++x) sorted = a[x - 1] <= a[x];
      if (!sorted) qsort(a, m, sizeof(uint32_t), cmp_u32);
    }
    for (uint32_t u = 0; u < V; ++u)
      for (uint64_t e = g->row_index[u]; e < g->row_index[u + 1]; ++e)
        g->in_adjs[in_pos[g->out_adjs[e]]++] = u;
  }
  /* DCSC compression */
  uint64_t nnz = 0;
  for (uint32_t v = 0; v < V; ++v) nnz += (in_cnt[v] > 0);
  g->nnzcol = nnz;
  g->col_index = (uint64_t*)malloc((nnz + 1) * 8);
  g->col_vertex = (uint32_t*)malloc((nnz ? nnz : 1) * 4);
  uint64_t c = 0;
  for (uint32_t v = 0; v < V; ++v) {
    if (in_cnt[v] == 0) continue;
    g->col_index[c] = in_off[v];
    g->col_vertex[c] = v;
    ++c;
  }
  g->col_index[nnz] = E;
  for (uint32_t v = 0; v < V; ++v)
    if (out_cnt[v]) bm_set(g->row_bitmap, v);
  /* generate_dense_out_degrees_fg(is_out_edge=false): count each source
   * occurrence in the in-edge lists */
#pragma omp parallel for schedule(static)
  for (int64_t e = 0; e < (int64_t)E; ++e) __atomic_fetch_add(&g->out_degree[g->in_adjs[e]], 1u, __ATOMIC_RELAXED);
  free(in_cnt);
  free(out_cnt);
  free(in_off);
  free(in_pos);
  free(out_pos);
  return g;
}

EXPORT void ref_graph_free(ref_graph* g) {
  if (!g) return;
  free(g->col_index);
  free(g->col_vertex);
  free(g->in_adjs);
  free(g->row_bitmap);
  free(g->row_index);
  free(g->out_adjs);
  free(g->out_degree);
  free(g->ws_a);
  free(g->ws_b);
  free(g->ws_actives);
  free(g->ws_walk);
  free(g);
}

EXPORT uint64_t ref_graph_dcsc_columns(const ref_graph* g) { return g->nnzcol; }
EXPORT uint64_t ref_graph_stored_edges(const ref_graph* g) { return g->stored_edges; }
EXPORT void ref_out_degrees(const ref_graph* g, uint32_t* out) {
  memcpy(out, g->out_degree, (size_t)g->vertices * 4);
}
EXPORT void ref_in_adjacency(const ref_graph* g, uint64_t* col_index, uint32_t* col_vertex,
                             uint32_t* adjs) {
  memcpy(col_index, g->col_index, (g->nnzcol + 1) * 8);
  memcpy(col_vertex, g->col_vertex, g->nnzcol * 4);
  memcpy(adjs, g->in_adjs, g->stored_edges * 4);
}

/* aggregate_message with the KAT functors of plato/graph/test/message_passing.cc:62-87:
 * signal sends 1 per in-edge, slot adds it to values[v] and returns 1;
 * returns the sum of slot returns. */
EXPORT uint64_t ref_aggregate_count(const ref_graph* g, int32_t* values) {
  uint64_t sum = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : sum)
  for (int64_t c = 0; c < (int64_t)g->nnzcol; ++c) {
    const uint32_t v = g->col_vertex[c];
    for (uint64_t e = g->col_index[c]; e < g->col_index[c + 1]; ++e) {
      __atomic_fetch_add(&values[v], 1, __ATOMIC_RELAXED);
      sum += 1;
    }
  }
  return sum;
}

/* ---------------- rank algorithms ------------------------------------------ */
/* teleport kinds */
enum { TELE_UNIFORM = 0, TELE_SINGLE = 1, TELE_SEEDS = 2 };

/* pull: next[v] += sum_{src in in(v)} curt[src] over DCSC columns (CIRCLE
 * chunks of 64 columns, message_passing.hpp:116-117); write_add slot. */
static void pull_sum(const ref_graph* g, const double* curt, double* next) {
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t c = 0; c < (int64_t)g->nnzcol; ++c) {
    double rank_sum = 0.0;
    for (uint64_t e = g->col_index[c]; e < g->col_index[c + 1]; ++e) rank_sum += curt[g->in_adjs[e]];
    write_add(&next[g->col_vertex[c]], rank_sum);
  }
}

/* one vertex update; returns the delta term (pagerank.hpp:118-135) */
static inline double update(double* pval, double tele, double d, uint32_t deg, double old,
                            int final_epoch) {
  *pval = tele + d * (*pval);
  if (final_epoch) return 0.0;
  if (deg > 0) {
    *pval = *pval / deg;
    return fabs(*pval - old) * deg;
  }
  return fabs(*pval - old);
}

/* Generic rank loop.  tele_kind selects pagerank / single-source / seed set.
 * pushpull: personalized_pagerank.hpp:158-272 push epochs while
 * active_edges <= edges/20 (sticky). */
static int rank_loop(ref_graph* g, int tele_kind, uint32_t src, const uint8_t* is_seed,
                     double seed_tele, uint32_t iteration, double damping, double eps,
                     int pushpull, double* out, uint32_t* epochs_out, uint32_t* push_epochs_out,
                     uint64_t* trace_out, double* delta_out) {
  const uint32_t V = g->vertices;
  if (!g->ws_a) {
    g->ws_a = (double*)malloc(((size_t)V + 1) * 8);
    g->ws_b = (double*)malloc(((size_t)V + 1) * 8);
    g->ws_actives = (uint64_t*)malloc(bm_words(V) * 8);
    g->ws_walk = (uint64_t*)malloc(bm_words(V) * 8);
    if (!g->ws_a || !g->ws_b || !g->ws_actives || !g->ws_walk) return 2;
  }
  double* curt = g->ws_a;
  double* next = g->ws_b;
  uint64_t* actives = g->ws_actives;
  uint64_t* walk = g->ws_walk;
  memset(actives, 0, bm_words(V) * 8);
  const uint32_t* odeg = g->out_degree;
  /* init */
#pragma omp parallel for schedule(static)
  for (int64_t v = 0; v < (int64_t)V; ++v) {
    double x;
    if (tele_kind == TELE_UNIFORM) x = 1.0;
    else if (tele_kind == TELE_SINGLE) x = ((uint32_t)v == src) ? 1.0 : 0.0;
    else x = is_seed[v] ? seed_tele : 0.0;  /* trustrank.hpp:197-206: init_dist */
    if (tele_kind != TELE_SINGLE && odeg[v] > 0) x = x / odeg[v];
    curt[v] = x;
  }
  if (tele_kind == TELE_SINGLE && odeg[src] > 0) curt[src] = 1.0 / odeg[src];
  if (pushpull) bm_set(actives, src);
  uint64_t edges = g->input_edges;
  if (!g->is_directed) edges *= 2;
  int do_pull = !pushpull;
  uint32_t epochs = 0, push_epochs = 0;
  uint64_t trace = 0;
  double delta = 0.0;
  for (uint32_t epoch = 0; epoch < iteration; ++epoch) {
    if (!do_pull) {
      uint64_t active_edges = 0;
#pragma omp parallel for schedule(static) reduction(+ : active_edges)
      for (int64_t v = 0; v < (int64_t)V; ++v)
        if (bm_get(actives, (uint32_t)v)) active_edges += odeg[v];
      do_pull = active_edges > edges / 20;
    }
#pragma omp parallel for schedule(static)
    for (int64_t v = 0; v < (int64_t)V; ++v) next[v] = 0.0;
    if (do_pull) {
      pull_sum(g, curt, next);
    } else {
      /* broadcast over active vertices; slot scatters to out-neighbours and
       * marks them active (personalized_pagerank.hpp:225-239).  The slot sets
       * bits in the bitmap the broadcast is scanning, from other threads, so
       * in the reference a vertex reached in this epoch may or may not be
       * broadcast in this epoch too, by thread timing.  Its rank is still 0,
       * so the ranks are the same either way; only the active-edge count of
       * the next switch test can differ.  This restatement takes the one
       * order that does not depend on timing: the epoch broadcasts the
       * actives it started with. */
      const uint64_t words = bm_words(V);
      memcpy(walk, actives, words * 8);
#pragma omp parallel for schedule(dynamic, 64)
      for (int64_t w = 0; w < (int64_t)words; ++w) {
        uint64_t bits = walk[w];
        while (bits) {
          const int b = __builtin_ctzll(bits);
          bits &= bits - 1;
          const uint32_t v = (uint32_t)(w * 64 + b);
          if (v >= V) break;
          const double msg = curt[v];
          for (uint64_t e = g->row_index[v]; e < g->row_index[v + 1]; ++e) {
            const uint32_t dst = g->out_adjs[e];
            bm_set(actives, dst);
            write_add(&next[dst], msg);
          }
        }
      }
      if (epoch < 64) trace |= 1ull << epoch;
      ++push_epochs;
    }
    const int final_epoch = (epoch == iteration - 1);
    double dsum = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : dsum)
    for (int64_t v = 0; v < (int64_t)V; ++v) {
      double tele;
      if (tele_kind == TELE_UNIFORM) tele = 1.0 - damping;
      else if (tele_kind == TELE_SINGLE) tele = ((uint32_t)v == src) ? 1.0 - damping : 0.0;
      else tele = is_seed[v] ? (1.0 - damping) * seed_tele : 0.0;
      dsum += update(&next[v], tele, damping, odeg[v], curt[v], final_epoch);
    }
    ++epochs;
    if (!final_epoch) {
      delta = dsum;
      if (eps > 0.0 && delta < eps) epoch = iteration - 2;
    }
    double* t = curt;
    curt = next;
    next = t;
  }
  memcpy(out, curt, (size_t)V * 8);
  if (epochs_out) *epochs_out = epochs;
  if (push_epochs_out) *push_epochs_out = push_epochs;
  if (trace_out) *trace_out = trace;
  if (delta_out) *delta_out = delta;
  return 0;
}

/* algo::pagerank — reference units (ranks start at 1.0). */
EXPORT int ref_pagerank(ref_graph* g, uint32_t iteration, double damping, double eps,
                        double* out, uint32_t* epochs, double* delta) {
  return rank_loop(g, TELE_UNIFORM, 0, NULL, 0.0, iteration, damping, eps, 0, out, epochs, NULL,
                   NULL, delta);
}

/* algo::personalized_pagerank — pull-only (pushpull = 0) or dual-mode (1). */
EXPORT int ref_ppr(ref_graph* g, uint32_t src, uint32_t iteration, double damping, double eps,
                   int pushpull, double* out, uint32_t* epochs, uint32_t* push_epochs,
                   uint64_t* trace, double* delta) {
  if (src >= g->vertices) return 1;
  return rank_loop(g, TELE_SINGLE, src, NULL, 0.0, iteration, damping, eps, pushpull, out, epochs,
                   push_epochs, trace, delta);
}

/* Seed-set PPR with trustrank's semantics (trustrank.hpp:197-245): init
 * 1/|S| on seeds (divided by degree), teleport (1-d)/|S| on seeds. */
EXPORT int ref_seedset_ppr(ref_graph* g, uint32_t nseeds, const uint32_t* seeds,
                           uint32_t iteration, double damping, double eps, double* out,
                           uint32_t* epochs, double* delta) {
  const uint32_t V = g->vertices;
  uint8_t* is_seed = (uint8_t*)calloc(V ? V : 1, 1);
  uint32_t count = 0;
  for (uint32_t i = 0; i < nseeds; ++i) {
    if (seeds[i] >= V) { free(is_seed); return 1; }
    if (!is_seed[seeds[i]]) { is_seed[seeds[i]] = 1; ++count; }
  }
  if (count == 0) { free(is_seed); return 1; }
  int r = rank_loop(g, TELE_SEEDS, 0, is_seed, 1.0 / count, iteration, damping, eps, 0, out,
                    epochs, NULL, NULL, delta);
  free(is_seed);
  return r;
}

/* ---------------- breadth first search (bfs.hpp:70-151) -------------------- */
EXPORT int ref_bfs(const ref_graph* g, uint32_t root, double push_threshold, uint32_t* levels,
                   uint32_t* parents, uint64_t* visited_count, uint64_t* trace_out,
                   uint32_t* epochs_out) {
  const uint32_t V = g->vertices;
  if (root >= V) return 1;
  const uint64_t words = bm_words(V);
  uint64_t* visited = (uint64_t*)calloc(words, 8);
  uint64_t* cur = (uint64_t*)calloc(words, 8);
  uint64_t* nxt = (uint64_t*)calloc(words, 8);
  uint32_t* parent = parents;
  const uint32_t invalid_parent = g->max_v_i + 1;
  const uint32_t* odeg = g->out_degree;
  for (uint32_t v = 0; v < V; ++v) {
    parent[v] = invalid_parent;
    levels[v] = 0xFFFFFFFFu;
  }
  parent[root] = root;
  levels[root] = 0;
  bm_set(visited, root);
  bm_set(cur, root);
  uint64_t edges = g->input_edges;
  if (!g->is_directed) edges *= 2;
  uint64_t actives = 1, trace = 0;
  uint32_t epoch = 0;
  for (epoch = 0; actives != 0; ++epoch) {
    memset(nxt, 0, words * 8);
    uint64_t active_edges = 0;
#pragma omp parallel for schedule(static) reduction(+ : active_edges)
    for (int64_t w = 0; w < (int64_t)words; ++w) {
      uint64_t bits = cur[w];
      while (bits) {
        const int b = __builtin_ctzll(bits);
        bits &= bits - 1;
        const uint64_t v = (uint64_t)w * 64 + b;
        if (v < V) active_edges += odeg[v];
      }
    }
    const int is_sparse = ((double)active_edges / (double)edges) < push_threshold;
    uint64_t activated = 0;
    if (is_sparse) {
#pragma omp parallel for schedule(dynamic, 16) reduction(+ : activated)
      for (int64_t w = 0; w < (int64_t)words; ++w) {
        uint64_t bits = cur[w];
        while (bits) {
          const int b = __builtin_ctzll(bits);
          bits &= bits - 1;
          const uint32_t u = (uint32_t)(w * 64 + b);
          if (u >= V) break;
          for (uint64_t e = g->row_index[u]; e < g->row_index[u + 1]; ++e) {
            const uint32_t dst = g->out_adjs[e];
            if (__atomic_load_n(&parent[dst], __ATOMIC_RELAXED) == invalid_parent &&
                cas_u32(&parent[dst], invalid_parent, u)) {
              bm_set(nxt, dst);
              bm_set(visited, dst);
              levels[dst] = epoch + 1;
              ++activated;
            }
          }
        }
      }
      if (epoch < 64) trace |= 1ull << epoch;
    } else {
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : activated)
      for (int64_t c = 0; c < (int64_t)g->nnzcol; ++c) {
        const uint32_t v = g->col_vertex[c];
        if (bm_get(visited, v)) continue;
        for (uint64_t e = g->col_index[c]; e < g->col_index[c + 1]; ++e) {
          const uint32_t s = g->in_adjs[e];
          if (bm_get(cur, s)) {
            if (cas_u32(&parent[v], invalid_parent, s)) {
              bm_set(nxt, v);
              bm_set(visited, v);
              levels[v] = epoch + 1;
              ++activated;
            }
            break;
          }
        }
      }
    }
    actives = activated;
    uint64_t* t = cur;
    cur = nxt;
    nxt = t;
  }
  uint64_t count = 0;
  for (uint64_t w = 0; w < words; ++w) count += (uint64_t)__builtin_popcountll(visited[w]);
  if (visited_count) *visited_count = count;
  if (trace_out) *trace_out = trace;
  if (epochs_out) *epochs_out = epoch;
  free(visited);
  free(cur);
  free(nxt);
  return 0;
}

EXPORT int ref_max_threads(void) { return omp_get_max_threads(); }
