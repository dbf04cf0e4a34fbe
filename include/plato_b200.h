/*
 * plato_b200.h — C ABI of the B200-native dual-mode push/pull graph engine.
 *
 * Plain C types only (no torch, no C++): every entry point returns an int
 * status (PLATO_OK == 0) and never aborts; the message of the last failure on
 * the calling thread is available from plato_last_error().
 *
 * Vertex ids are the caller's ids, which must be compact (every id in
 * [0, vertices) — the reference requires the same, see
 * plato/graph/structure/dcsc.hpp:48-49 "vertexId must be compacted" and
 * plato/graph/partition/sequence.hpp:67).  Internally the engine may renumber
 * vertices (unless PLATO_GRAPH_NO_RELABEL); every result crosses the ABI in caller ids.
 *
 * Numeric conventions (parity with the reference):
 *  - PageRank ranks are returned normalised: initial rank 1/V, teleport
 *    (1-d)/V.  The reference (plato/algo/pagerank/pagerank.hpp:90-146) starts
 *    at 1.0 with teleport (1-d); every iterate of the reference equals ours
 *    times V.  opts->eps keeps the reference's units (the sum of rank changes
 *    over the un-normalised ranks), so early exit triggers on the same
 *    iteration in exact arithmetic.
 *  - Personalized PageRank is already normalised in the reference
 *    (plato/algo/ppr/personalized_pagerank.hpp:71-81): values are returned as is.
 *  - BFS levels are exact; unreached vertices get PLATO_LEVEL_UNREACHED;
 *    parents use the reference's invalid marker max_v_i + 1
 *    (plato/algo/bfs/bfs.hpp:79).
 */
#ifndef PLATO_B200_H
#define PLATO_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define PLATO_OK          0
#define PLATO_EINVAL      1  /* bad argument (null pointer, id out of range, ...) */
#define PLATO_ENOMEM      2  /* device or host allocation failed / over budget     */
#define PLATO_ECUDA       3  /* a CUDA runtime call failed                          */
#define PLATO_ETIMEDOUT   4  /* a bounded device wait for another partition ran out
                                (plato_partition_p2p_state)                          */
#define PLATO_EBUSY       5  /* server full: no slot or HBM budget for the request  */
#define PLATO_ENOTFOUND   6  /* nothing ready / unknown request id                  */

#define PLATO_LEVEL_UNREACHED 0xFFFFFFFFu

/* graph creation flags.  By default the engine renumbers vertices by
 * descending in-degree inside the graph (results still cross the ABI in
 * caller ids): the pull kernels then work on contiguous degree bins.
 * PLATO_GRAPH_NO_RELABEL keeps the caller's order (the device view's CSC is
 * then indexed by caller ids); pull epochs on such a graph take the
 * merge-path kernel, about 2.5x slower.  PLATO_GRAPH_RELABEL asks for the
 * default explicitly; both together -> PLATO_EINVAL. */
#define PLATO_GRAPH_RELABEL    0x1u
#define PLATO_GRAPH_NO_RELABEL 0x2u

/* personalized pagerank modes */
#define PLATO_PPR_PULL      0 /* pull-only engine: personalized_pagerank.hpp:40-134     */
#define PLATO_PPR_PUSHPULL  1 /* push until active edges > E/20, then pull: :137-275   */

typedef uint32_t plato_vid_t; /* plato/graph/base.hpp vid_t */
typedef uint64_t plato_eid_t; /* plato/graph/base.hpp eid_t */

typedef struct plato_graph plato_graph;
typedef struct plato_server plato_server;

/* Mirrors graph_info_t (plato/graph/base.hpp:241-257). */
typedef struct {
  int32_t     is_directed;
  plato_vid_t vertices;  /* number of vertices (ids are [0, vertices)) */
  plato_eid_t edges;     /* input edges; undirected edges count once   */
  plato_vid_t max_v_i;   /* largest vertex id == vertices - 1          */
} plato_graph_info;

/* Mirrors pagerank_opts_t (plato/algo/pagerank/pagerank.hpp:39-46). */
typedef struct {
  uint32_t iteration;
  double   damping;
  double   eps;        /* 0 forces `iteration` epochs */
} plato_pagerank_opts;

/* Mirrors personalized_pagerank_opts_t (plato/algo/ppr/personalized_pagerank.hpp:18-26). */
typedef struct {
  uint32_t    iteration;
  double      damping;
  plato_vid_t src;
  double      eps;
} plato_ppr_opts;

/* Mirrors bfs_opts_t (plato/algo/bfs/bfs.hpp:37-39). */
typedef struct {
  plato_vid_t root;
} plato_bfs_opts;

/* Mirrors dualmode_engine_opts_t (plato/engine/dualmode.hpp:41-43). */
typedef struct {
  double push_threshold; /* push iff active_edges / edges < push_threshold (default 0.05) */
} plato_dualmode_opts;

/* Per-run statistics (the reference logs the same per epoch, e.g. pagerank.hpp:141-144). */
typedef struct {
  uint32_t iterations;      /* epochs executed (including the final non-dividing one) */
  uint32_t push_iterations; /* epochs run in push mode                                */
  uint32_t pull_iterations; /* epochs run in pull mode                                */
  uint32_t reserved;
  double   delta;           /* last delta (reference units)                           */
  uint64_t visited;         /* BFS: visited vertex count (bfs.hpp:153-154)            */
  uint64_t mode_trace;      /* bit i set = epoch i ran in push mode (first 64 epochs) */
} plato_run_stats;

/* Raw device view of a resident graph in the engine's internal vertex order,
 * for header-only device code (include/plato_b200/dualmode.cuh). */
typedef struct {
  plato_vid_t        vertices;
  int32_t            is_directed;
  plato_eid_t        edges;        /* graph_info.edges (input edges)              */
  plato_eid_t        stored_edges; /* directed edges stored (2*edges undirected)  */
  const uint64_t*    in_offsets;   /* [V+1] CSC (DCSC without the empty-column compression) */
  const plato_vid_t* in_adj;       /* [stored_edges] sources, ascending per column */
  const uint64_t*    out_offsets;  /* [V+1] CSR */
  const plato_vid_t* out_adj;      /* [stored_edges] destinations, ascending per row */
  const uint32_t*    out_degree;   /* [V] */
  const uint32_t*    in_degree;    /* [V] */
  const plato_vid_t* to_internal;  /* [V] caller id -> internal id (NULL if identity) */
  const plato_vid_t* to_external;  /* [V] internal id -> caller id (NULL if identity) */
} plato_graph_device_view;

/* ---- errors / diagnostics ---------------------------------------------- */
const char* plato_last_error(void);
/* Number of kernels this library has launched in this process. */
uint64_t    plato_kernel_launches(void);
/* Library version string. */
const char* plato_version(void);

/* ---- kernel timing ---------------------------------------------------------
 * When enabled, the hot kernels are bracketed by CUDA events on their launch
 * stream (the device analogue of the reference's per-epoch stop_watch_t,
 * plato/util/perf.hpp:71-103).  plato_profile_read synchronises those events
 * and returns the summed device time and launch count of one kernel name
 * since the last reset. */
int plato_profile_enable(int on);
int plato_profile_reset(void);
int plato_profile_read(const char* kernel, double* total_ms, uint64_t* launches);

/* ---- graph ---------------------------------------------------------------
 * Replaces create_dualmode_seq_from_path (plato/graph/structure.hpp:983-1086)
 * for an edge list already in memory: builds CSC (in-edges, the DCSC of
 * dcsc.hpp:148-152) and CSR (out-edges, the BCSR of bcsr.hpp:167-174) in HBM.
 * Undirected input is stored in both directions (dcsc.hpp:365-385).  Host
 * arrays src/dst hold info->edges entries.  Ids >= info->vertices -> EINVAL. */
int plato_graph_create(const plato_graph_info* info, const plato_vid_t* src,
                       const plato_vid_t* dst, uint32_t flags, plato_graph** out);
/* Same with a double weight per input edge (create_dcsc_seqs_from_path<double>
 * with double_decoder, as example/pagerank_weighted.cc:71-74 loads weighted
 * graphs): each edge keeps its weight (float) in the CSC, and every vertex
 * the sum of its out-edge weights (summed in double, in CSR row order).
 * weights: host [info->edges], input order. */
int plato_graph_create_weighted(const plato_graph_info* info, const plato_vid_t* src,
                                const plato_vid_t* dst, const double* weights, uint32_t flags,
                                plato_graph** out);
int plato_graph_destroy(plato_graph* g);
int plato_graph_get_info(const plato_graph* g, plato_graph_info* info);
int plato_graph_get_device_view(const plato_graph* g, plato_graph_device_view* view);
/* Out-degrees computed from the in-edge structure, in caller ids
 * (generate_dense_out_degrees_fg, plato/graph/structure.hpp:291-346). */
int plato_graph_out_degrees(plato_graph* g, uint32_t* degrees_out /* host [V] */);
/* Bytes of HBM held by the graph. */
int plato_graph_device_bytes(const plato_graph* g, uint64_t* bytes);

/* ---- algorithms (host output buffers) ------------------------------------ */
/* algo::pagerank (plato/algo/pagerank/pagerank.hpp:60-149).  ranks: host [V]. */
int plato_pagerank(plato_graph* g, const plato_pagerank_opts* opts, float* ranks,
                   plato_run_stats* stats);
/* algo::personalized_pagerank, pull-only (personalized_pagerank.hpp:40-134) or
 * dual-mode (:137-275) by `mode`.  ranks: host [V]. */
int plato_personalized_pagerank(plato_graph* g, const plato_ppr_opts* opts, int mode,
                                float* ranks, plato_run_stats* stats);
/* algo::trustrank (plato/algo/trustrank/trustrank.hpp:163-259) with the seed
 * set given instead of selected: one seed-set PPR query on the pull engine
 * (init 1/|S| on seeds, teleport (1-d)/|S| on seeds; opts->src is ignored). */
int plato_seedset_ppr(plato_graph* g, const plato_vid_t* seeds, uint32_t n,
                      const plato_ppr_opts* opts, float* ranks, plato_run_stats* stats);

/* Mirrors trustrank_opts_t (plato/algo/trustrank/trustrank.hpp:24-33). */
typedef struct {
  uint32_t iteration;      /* 100 */
  double   damping;        /* 0.85 */
  uint32_t seed_num;       /* 100 */
  uint32_t select_method;  /* 0 inverse PageRank, 1 PageRank, 2 random */
  double   eps;            /* 0.001 */
  uint64_t random_seed;    /* method 2 only (the reference draws from std::random_device) */
} plato_trustrank_opts;
/* algo::trustrank with select_good_seeds (trustrank.hpp:88-259): seeds are
 * the good vertices among the top seed_num by (inverse) PageRank (ranks of
 * the reference's default PageRank run, FP64; ties by smaller id), or drawn
 * at random, or every good vertex when V <= seed_num; then one seed-set PPR.
 * good_vertices: host [V] 0/1 bytes, NULL = every vertex is good.
 * seeds_out: host [seed_num] (sorted caller ids) or NULL; *n_seeds = count.
 * No good seed among the selected -> PLATO_EINVAL (the reference divides
 * by zero). */
int plato_trustrank(plato_graph* g, const plato_trustrank_opts* opts, const uint8_t* good_vertices,
                    float* ranks, plato_vid_t* seeds_out, uint32_t* n_seeds, plato_run_stats* stats);
/* algo::weighted_pagerank (plato/algo/pagerank/weighted_pagerank.hpp:60-149)
 * on a graph made by plato_graph_create_weighted (else PLATO_EINVAL): ranks
 * start at 1, rank' = 1 - d + d * sum of rank[u] * w / weight_sum[u] over
 * in-edges; eps > 0 and the epoch's sum |rank' - rank| < eps jumps to the last
 * epoch.  ranks: host [V], caller ids, in the reference's units (not
 * normalised).  stats->delta = the last delta read (eps > 0). */
int plato_weighted_pagerank(plato_graph* g, const plato_pagerank_opts* opts, float* ranks,
                            plato_run_stats* stats);
/* algo::breadth_first_search (plato/algo/bfs/bfs.hpp:55-155) with the engine's
 * push/pull switch (dualmode.hpp:245-297).  levels/parents: host [V] or NULL. */
int plato_bfs(plato_graph* g, const plato_bfs_opts* opts, const plato_dualmode_opts* engine_opts,
              uint32_t* levels, plato_vid_t* parents, plato_run_stats* stats);

/* plato::algo::connected_component_t (plato/algo/cgm/connected_component.hpp):
 * label propagation with the engine's push/pull switch (:173-245) and the
 * component summary (:247-340).  labels: host [V] or NULL, each vertex's
 * label = the smallest caller id that reaches it along edges (its
 * component's smallest id on undirected graphs).  stats->iterations = epochs. */
typedef struct {
  uint64_t    components;      /* distinct labels                                      */
  plato_vid_t major_label;     /* label of the largest component (ties: smallest label) */
  uint64_t    major_vertices;
  uint64_t    major_edges;     /* in-edges whose source has the major label; undirected: halved */
} plato_cc_summary;
int plato_connected_components(plato_graph* g, const plato_dualmode_opts* engine_opts,
                               plato_vid_t* labels, plato_cc_summary* summary,
                               plato_run_stats* stats);

/* ---- HyperLogLog propagation (hyperloglog_t<P>, plato/util/hyperloglog.hpp:32-142;
 * ids hashed with murmurhash3, plato/util/hash.hpp:33-88) -------------------- */
/* Mirrors hyperanf_opts_t (plato/algo/hyperanf/hyperanf.hpp:43-46). */
typedef struct {
  uint32_t iteration; /* 20 */
  uint32_t bits;      /* register-count exponent P in [4, 16] (the CLI's --bits, default 6) */
} plato_hyperanf_opts;
/* algo::hyperanf (hyperanf.hpp:83-195): *avg_distance = GetAvgDistance of the
 * ANF series (NaN when the series never grows).  anfs: host [iteration + 1] or
 * NULL, *n_anfs = entries written.  registers: host [V << bits] or NULL, the
 * final register rows in caller-id order.  stats: epochs and the engine's
 * push/pull choice per epoch. */
int plato_hyperanf(plato_graph* g, const plato_hyperanf_opts* opts, const plato_dualmode_opts* engine_opts,
                   double* avg_distance, double* anfs, uint32_t* n_anfs, uint8_t* registers,
                   plato_run_stats* stats);

#define PLATO_NSTEP_IN 1
#define PLATO_NSTEP_OUT 2
#define PLATO_NSTEP_BOTH 3
/* Mirrors nstepdegree_opts_t (plato/algo/nstepdegrees/nstepdegrees.hpp:47-51)
 * plus the register width the reference takes as a template argument. */
typedef struct {
  uint32_t step;        /* epochs per phase; 0xFFFFFFFF = until nothing changes (the CLI's -1) */
  uint32_t bits;        /* P in [4, 16] (CLI default 6) */
  uint32_t type;        /* PLATO_NSTEP_IN / _OUT / _BOTH ("in" / "out" / "both") */
  int32_t  is_directed; /* nstepdegree_opts_t::is_directed: with type BOTH and 0, out = in */
} plato_nstep_opts;
/* nstepdegrees_t::compute (nstepdegrees.hpp:380-402): for each target, the
 * estimated number of vertices within `step` hops towards it (in) or from it
 * (out), excluding itself.  targets: host [V] 0/1 bytes by caller id, NULL =
 * every vertex (the CLI's "ALL").  in_degrees / out_degrees: host [V] or NULL,
 * caller ids, 0 for non-targets.  The engine's switch and the reference's
 * forward push in reversed phases are reproduced (see nstepdegrees.hpp:217-229,
 * 316-327). */
int plato_nstep_degrees(plato_graph* g, const plato_nstep_opts* opts, const plato_dualmode_opts* engine_opts,
                        const uint8_t* targets, plato_vid_t* in_degrees, plato_vid_t* out_degrees,
                        plato_run_stats* stats);

/* ---- algorithms (device output buffers, caller's CUDA stream) ------------- */
/* Same as plato_pagerank but writes the ranks to device memory d_ranks [V]
 * (caller ids) on `stream` (a cudaStream_t; NULL = legacy default stream).
 * With opts->eps == 0 nothing is read back and the call does not synchronise. */
int plato_pagerank_device(plato_graph* g, const plato_pagerank_opts* opts, float* d_ranks,
                          void* stream, plato_run_stats* stats);

/* ---- PageRank without allocation -----------------------------------------
 * No counterpart in the reference.  For callers that must not have a library
 * call cudaMalloc (an application whose pooling allocator owns all of HBM, a
 * plugin under a fixed memory budget, a loop that cannot take an
 * allocation's device-wide synchronisation): PageRank over the caller's own
 * CSC in device memory (d_in_offsets [V+1], d_in_adj [edges] sources,
 * d_out_degree [V]; edges = directed edges stored, both directions for an
 * undirected graph), ranks written to device memory d_ranks [V] in the
 * caller's vertex order, normalised as plato_pagerank, on `stream`.
 * d_ranks must be 16-byte aligned (it also holds the ranks between epochs
 * and is read with vector loads), d_in_offsets 8-byte, d_in_adj and
 * d_out_degree 4-byte aligned; otherwise PLATO_EINVAL before any launch.
 * Every temporary lives in one static device array of
 * PLATO_NOALLOC_SCRATCH_BYTES held by each GPU that loads the library until
 * exit; a graph needing more (about 4V + 12(V+E)/224 bytes) gets EINVAL.
 * The first call on a device looks up that array's device address (and sets
 * the kernel's shared-memory limit); make it before any stream capture.
 * With eps > 0 the early exit is decided on the device; a non-NULL `stats`
 * then makes the call wait for its own work at the end to read the epoch
 * count and the last delta (stats->delta: the delta of the last non-final
 * epoch, 0 with eps == 0, as plato_pagerank reports it).
 * Calls that overlap on the GPU race on the shared array: serialise them. */
#define PLATO_NOALLOC_SCRATCH_BYTES (32u << 20)
int plato_pagerank_csc_noalloc(uint32_t vertices, uint64_t edges, const uint64_t* d_in_offsets,
                               const uint32_t* d_in_adj, const uint32_t* d_out_degree,
                               const plato_pagerank_opts* opts, float* d_ranks, void* stream,
                               plato_run_stats* stats);

/* ---- 1D-partitioned PageRank over several GPUs ---------------------------
 * The reference's multi-partition pull (create_dcsc_seqs_from_path with
 * sequence_balanced_by_destination_t, plato/graph/structure.hpp:471-555,
 * plato/graph/partition/sequence.hpp:43-75; one process per partition).
 * Partition `rank` of `world` owns a set of destination vertices with all of
 * their in-edges; the rank state the pull gathers is replicated on every GPU
 * as a world x rows float array (internal global ids), each partition writes
 * its slice [rank*rows, (rank+1)*rows) of the next state, and the caller
 * assembles the next state with an all-gather (in place, equal counts: e.g.
 * NCCL over NVLink) before the next epoch.  Vertices are ranked by descending
 * in-degree (ties by caller id) and rank i goes to partition i % world at row
 * i / world, so partitions hold equal row counts (some end in padding rows)
 * and near-equal edge counts, and run the single-GPU degree-binned kernels.
 * Every process passes the whole edge list (host memory) and derives the
 * same layout.  PageRank semantics and units are plato_pagerank's. */
typedef struct plato_partition plato_partition;
/* Global internal id of every caller vertex (host [V]) and rows per partition,
 * host-only (no GPU needed). */
int plato_partition_layout(const plato_graph_info* info, const plato_vid_t* src, const plato_vid_t* dst,
                           uint32_t world, plato_vid_t* global_ids, uint32_t* rows_per_partition);
/* Builds partition `rank` on the current device. */
int plato_partition_create(const plato_graph_info* info, const plato_vid_t* src, const plato_vid_t* dst,
                           uint32_t rank, uint32_t world, plato_partition** out);
int plato_partition_destroy(plato_partition* p);
/* vertices = V of the whole graph, rows = rows per partition, real_rows = this
 * partition's vertices (rows minus padding), edges = its in-edges. */
int plato_partition_info(const plato_partition* p, uint32_t* vertices, uint32_t* rows, uint32_t* real_rows,
                         uint64_t* edges);
/* Writes this partition's slice of the initial state (pagerank.hpp:90-98,
 * normalised) into d_state [world*rows] on `stream`. */
int plato_partition_pagerank_init(plato_partition* p, float* d_state, double damping, void* stream);
/* One pull epoch: gathers d_state [world*rows] (the assembled state), writes
 * this partition's slice of d_next; final_epoch != 0 stores the ranks
 * (pagerank.hpp:118-124).  d_delta (device, 1 double, or NULL) receives this
 * partition's delta in normalised units (the reference's = sum over
 * partitions x V); the caller sums it over partitions for the eps exit. */
int plato_partition_pagerank_epoch(plato_partition* p, const float* d_state, float* d_next, double damping,
                                   int final_epoch, double* d_delta, void* stream);
/* Caller-id ranks (host [V]) from an assembled state copied to the host
 * (h_state [world*rows]). */
int plato_partition_ranks(const plato_partition* p, const float* h_state, float* ranks);

/* Fused exchange over peer memory, in place of the all-gather: the same
 * epoch (the reference's per-epoch message exchange, message_passing.hpp:
 * 88-144), with each partition's pull storing its new rows straight into the
 * state replicas of every partition (NVLink peer stores) and a flag per
 * partition published after each epoch; the next epoch starts once every
 * partition has published (a bounded wait on the device).  With eps > 0 each
 * partition also publishes its delta, and every partition sums them in rank
 * order and applies the eps exit of pagerank.hpp:137-139 on the device.  No
 * collective and no host round trip per epoch; at most 8 partitions.
 * Between processes: every partition calls plato_partition_p2p_alloc
 * (two state replicas of world*rows floats and a flag/delta block, in its
 * own HBM; writes 3 CUDA IPC handles of PLATO_IPC_HANDLE_BYTES each), the
 * handles of all partitions are exchanged in rank order, then
 * plato_partition_p2p_connect maps the others'.  Partitions of one process
 * (on one GPU, or on several with peer access): plato_partition_p2p_connect_local.
 * A run: reset (flags to 0 on every partition, then a barrier, before any
 * init; alloc leaves them 0), init on every partition, then
 * plato_partition_p2p_epoch for epoch 0 .. iterations-1 (epochs after an eps
 * exit only pass the barrier), then plato_partition_p2p_state, which waits
 * for every partition's last epoch and returns the replica that holds the
 * ranks (world*rows floats, device) and the epochs that ran; or
 * plato_partition_p2p_ranks for the ranks in caller ids on the host.  A wait
 * gives up after timeout_ms (0: 5000) and the run reports PLATO_ETIMEDOUT
 * from plato_partition_p2p_state; later waits of the run return at once.
 * With partitions of one process on one GPU, call each epoch for every
 * partition before the next epoch (each epoch's waits are then already
 * satisfied). */
#define PLATO_IPC_HANDLE_BYTES 64
int plato_partition_p2p_alloc(plato_partition* p, void* handles_out);
int plato_partition_p2p_connect(plato_partition* p, const void* all_handles, uint32_t timeout_ms);
int plato_partition_p2p_connect_local(plato_partition* const* parts, uint32_t world, uint32_t timeout_ms);
int plato_partition_p2p_reset(plato_partition* p);
int plato_partition_p2p_init(plato_partition* p, uint32_t iterations, double damping, double eps, void* stream);
int plato_partition_p2p_epoch(plato_partition* p, uint32_t epoch, double damping, void* stream);
int plato_partition_p2p_state(plato_partition* p, void* stream, const float** d_state, uint32_t* epochs);
/* plato_partition_p2p_state, then the ranks in caller ids (host [V]). */
int plato_partition_p2p_ranks(plato_partition* p, void* stream, float* ranks, uint32_t* epochs);

/* ---- diagnostics -----------------------------------------------------------
 * No counterpart in the reference.  The memory system's rate on this graph's
 * long-bin pull gather stream (the CSC source ids of rows with in-degree > 64,
 * one 4-byte rank gathered per id), with the row bookkeeping and the update
 * taken out: mode 0 the id stream alone; 1 / 2 / 3 ids + random gathers with
 * 4 / 8 / 16 in flight per lane; 4 gathers folded into the first 64K ranks
 * (L1-resident); 5 gathers at the edge position mod V (coalesced).
 * *ms_per_launch = CUDA-event average over `reps` launches after 3 warm-ups;
 * *edges = ids in the stream; *checksum keeps the loads live.  The graph must
 * be relabelled (the default).  Allocates and synchronises: not for hot
 * paths. */
int plato_diag_pull_ceiling(plato_graph* g, uint32_t mode, uint32_t reps, double* ms_per_launch,
                            uint64_t* edges, double* checksum);
/* No counterpart in the reference.  The batched PPR pull's row-gather stream
 * at column-tile width kt (16/32/64/128): every CSC edge gathers its source's
 * kt-float row (a float4 per lane, 4 rows in flight per lane, as the batched
 * pull), with the row sums, update and delta taken out: mode 0 the real
 * source rows; 1 rows at the edge position mod V (sequential rows); 2 sources
 * folded into the first 16 MB of rows (L2-resident).  Mode 3 times the real
 * batched iteration over kt live columns that never converge.  Same outputs
 * and caveats as plato_diag_pull_ceiling (*edges = all stored edges); any
 * vertex order. */
int plato_diag_batch_ceiling(plato_graph* g, uint32_t kt, uint32_t mode, uint32_t reps, double* ms_per_launch,
                             uint64_t* edges, double* checksum);

/* ---- batched multi-source personalized pagerank --------------------------
 * K queries, query q's seed set is seeds[seed_offsets[q] .. seed_offsets[q+1]).
 * Each query follows the seed-set semantics of algo::trustrank
 * (plato/algo/trustrank/trustrank.hpp:197-245: init 1/|S| on seeds, teleport
 * (1-d)/|S| on seeds); a query stops once its own L1 delta < eps (plus the
 * reference's one final non-dividing epoch, pagerank.hpp:137-139). */
typedef struct {
  uint32_t max_iterations;
  double   damping;
  double   eps;
  uint32_t topk;       /* 0 = no top-k */
  uint32_t k_tile;     /* 0 = autotune */
} plato_ppr_batch_opts;

int plato_ppr_batch(plato_graph* g, uint32_t K, const uint64_t* seed_offsets /* host [K+1] */,
                    const plato_vid_t* seeds /* host */, const plato_ppr_batch_opts* opts,
                    float* ranks /* host [K*V] query-major, or NULL */,
                    plato_vid_t* topk_ids /* host [K*topk] or NULL */,
                    float* topk_vals /* host [K*topk] or NULL */,
                    uint32_t* iterations /* host [K] or NULL */);

/* The column-tile width plato_ppr_batch uses for K columns when
 * opts->k_tile == 0: autotuned on first use (a few timed iterations per
 * candidate width), then cached per graph and power-of-two bucket of K.
 * No reference counterpart (the reference runs one query at a time). */
int plato_ppr_batch_k_tile(plato_graph* g, uint32_t K, uint32_t* k_tile);

/* ---- continuous-batching PPR server -------------------------------------- */
typedef struct {
  uint32_t max_slots;        /* upper bound of live queries (columns)            */
  uint64_t hbm_budget_bytes; /* admission budget for per-query state             */
  uint32_t max_iterations;
  double   damping;
  double   eps;
  uint32_t topk;
} plato_server_opts;

int plato_server_create(plato_graph* g, const plato_server_opts* opts, plato_server** out);
/* Queue a request (seed set of n caller ids). Returns its id. */
int plato_server_submit(plato_server* s, const plato_vid_t* seeds, uint32_t n,
                        uint64_t* request_id);
/* Run one engine step: admit queued requests into free slots, run one
 * iteration over all live slots, retire converged ones. */
int plato_server_step(plato_server* s);
/* Fetch one finished result (any request). PLATO_ENOTFOUND if none is ready. */
int plato_server_poll(plato_server* s, uint64_t* request_id, plato_vid_t* topk_ids,
                      float* topk_vals, uint32_t* iterations);
/* live = queries on the device, queued = waiting for admission. */
int plato_server_stats(const plato_server* s, uint32_t* live, uint32_t* queued,
                       uint64_t* completed);
int plato_server_destroy(plato_server* s);

/* ---- synthetic input ------------------------------------------------------
 * Seeded RMAT edge list (Chakrabarti et al. 2004), self-loops and duplicates
 * removed, ids compacted to [0, V) (required by the reference, see above),
 * optionally symmetrised (one entry per unordered pair, is_directed = 0) and
 * optionally relabelled by a seeded permutation.  Host-side, multithreaded. */
typedef struct {
  uint32_t scale;
  uint32_t edgefactor;
  uint64_t seed;
  double   a, b, c;   /* d = 1 - a - b - c */
  int32_t  symmetrize;
  int32_t  permute;
} plato_rmat_params;

typedef struct plato_edge_list plato_edge_list;
int plato_rmat_generate(const plato_rmat_params* p, plato_edge_list** out);
int plato_edge_list_info(const plato_edge_list* el, plato_vid_t* vertices, uint64_t* edges);
/* Pointers stay valid until plato_edge_list_free.  RMAT lists are sorted by
 * (src, dst); lists read from files keep file order. */
int plato_edge_list_data(const plato_edge_list* el, const plato_vid_t** src,
                         const plato_vid_t** dst);
int plato_edge_list_free(plato_edge_list* el);

/* ---- files ------------------------------------------------------------------
 * Edge list from CSV text.  Replaces load_edges_cache + csv_parser
 * (plato/graph/structure.hpp:190-237, plato/graph/parsers.hpp:226-290,
 * plato/graph/detail.hpp:82-108, 196-212):
 *   path   one file, or a directory whose regular files are read in name
 *          order; names ending in ".gz" are gzip-compressed;
 *   lines  "src,dst": fields split at commas (empty fields skipped), each id
 *          read as strtoul(field, 10) reads it; empty lines and lines without
 *          a destination are skipped; an id above 2^32-1 -> PLATO_EINVAL
 *          (the reference aborts);
 *   info   edges = lines parsed, vertices = largest id + 1 (the reference's
 *          distinct-id count on the compact ids it requires).
 * The result feeds plato_graph_create like an RMAT list. */
int plato_edge_list_read_csv(const char* path, plato_edge_list** out);
/* As plato_edge_list_read_csv for weighted edges (csv_parser with
 * double_decoder, parsers.hpp:84-88, 226-290): a line needs a third field,
 * read as strtod reads it; lines without one are skipped. */
int plato_edge_list_read_csv_weighted(const char* path, plato_edge_list** out);
/* Weights of a weighted list in edge order (valid until plato_edge_list_free),
 * NULL for an unweighted list. */
int plato_edge_list_weights(const plato_edge_list* el, const double** weights);

/* Per-vertex results as CSV, the layout the reference's examples write
 * (example/pagerank.cc:191-200, plato/util/foutput.cc:95-101):
 * `files` files <dir>/<prefix><NNNN>.csv (".csv.gz" when gzip != 0), each
 * holding a contiguous vertex range, one "v,value" line per vertex; float
 * values printed as %g (ostream's default for double), uint32 values as
 * integers.  `values` is host memory indexed by caller vertex id. */
#define PLATO_VALUE_F32 0
#define PLATO_VALUE_U32 1
int plato_write_vertex_csv(const char* dir, const char* prefix, const void* values,
                           int value_type, uint32_t n, uint32_t files, int gzip);

#ifdef __cplusplus
}  /* extern "C" */
#endif

#endif /* PLATO_B200_H */
