"""plato_b200 — B200-native dual-mode push/pull graph engine (host-side mirror).

Python mirror of the reference's operator surface for the hot path, over the C
ABI of ``include/plato_b200.h``:

* option structs ``pagerank_opts_t``, ``personalized_pagerank_opts_t``,
  ``bfs_opts_t``, ``dualmode_engine_opts_t`` with the reference's field names
  and defaults (plato/algo/pagerank/pagerank.hpp:39-46,
  plato/algo/ppr/personalized_pagerank.hpp:18-26, plato/algo/bfs/bfs.hpp:37-39,
  plato/engine/dualmode.hpp:41-43);
* ``pagerank``, ``personalized_pagerank``, ``breadth_first_search`` with the
  reference's argument meaning and return values (ranks in reference units,
  visited count for BFS);
* ``Graph`` — a resident single-partition graph in HBM (``graph_info_t`` via
  ``Graph.info``).

Every call runs the CUDA kernels of libplato_b200.so; there is no CPU path.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from ._lib import (PLATO_GRAPH_NO_RELABEL, PLATO_GRAPH_RELABEL, PLATO_LEVEL_UNREACHED, PLATO_PPR_PULL, PLATO_PPR_PUSHPULL,
                   PlatoError, check, load)

__all__ = [
    "Graph", "GraphInfo", "PlatoError", "rmat", "read_csv", "write_vertex_csv", "pagerank", "personalized_pagerank",
    "breadth_first_search", "pagerank_opts_t", "personalized_pagerank_opts_t", "bfs_opts_t",
    "dualmode_engine_opts_t", "PLATO_LEVEL_UNREACHED", "PLATO_PPR_PULL", "PLATO_PPR_PUSHPULL",
    "kernel_launches",
]


@dataclass
class pagerank_opts_t:  # noqa: N801 — reference name
    iteration_: int = 100
    damping_: float = 0.85
    eps_: float = 0.001


@dataclass
class personalized_pagerank_opts_t:  # noqa: N801
    iteration_: int = 100
    damping_: float = 0.85
    src_: int = 0
    eps_: float = 0.001


@dataclass
class bfs_opts_t:  # noqa: N801
    root_: int = 0


@dataclass
class dualmode_engine_opts_t:  # noqa: N801
    push_threshold_: float = 0.05


@dataclass
class GraphInfo:
    """graph_info_t (plato/graph/base.hpp:241-257)."""
    is_directed_: bool
    vertices_: int
    edges_: int
    max_v_i_: int


@dataclass
class RunStats:
    iterations: int = 0
    push_iterations: int = 0
    pull_iterations: int = 0
    delta: float = 0.0
    visited: int = 0
    mode_trace: list = field(default_factory=list)  # "push"/"pull" per epoch (first 64)

    @classmethod
    def from_c(cls, s: _lib.RunStats) -> "RunStats":
        n = min(int(s.iterations), 64)
        trace = ["push" if (int(s.mode_trace) >> i) & 1 else "pull" for i in range(n)]
        return cls(int(s.iterations), int(s.push_iterations), int(s.pull_iterations),
                   float(s.delta), int(s.visited), trace)


def kernel_launches() -> int:
    return int(load().plato_kernel_launches())


def _u32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.uint32)


def _ptr(a: np.ndarray) -> C.c_void_p:
    return C.c_void_p(a.ctypes.data)


def _take_edge_list(lib, h, weighted: bool = False):
    """Copies an edge-list handle into numpy arrays and frees it."""
    try:
        V = C.c_uint32()
        E = C.c_uint64()
        check(lib.plato_edge_list_info(h, C.byref(V), C.byref(E)), "plato_edge_list_info")
        ps, pd = C.c_void_p(), C.c_void_p()
        check(lib.plato_edge_list_data(h, C.byref(ps), C.byref(pd)), "plato_edge_list_data")
        n = int(E.value)
        src = np.empty(n, dtype=np.uint32)
        dst = np.empty(n, dtype=np.uint32)
        if n:
            C.memmove(src.ctypes.data, ps.value, 4 * n)
            C.memmove(dst.ctypes.data, pd.value, 4 * n)
        if not weighted:
            return int(V.value), src, dst
        pw = C.c_void_p()
        check(lib.plato_edge_list_weights(h, C.byref(pw)), "plato_edge_list_weights")
        w = np.empty(n, dtype=np.float64)
        if n:
            C.memmove(w.ctypes.data, pw.value, 8 * n)
        return int(V.value), src, dst, w
    finally:
        lib.plato_edge_list_free(h)


def rmat(scale: int, edgefactor: int = 16, seed: int = 1, a: float = 0.57, b: float = 0.19,
         c: float = 0.19, symmetrize: bool = False, permute: bool = False):
    """Seeded RMAT edge list -> (V, src, dst) numpy uint32 arrays sorted by (src, dst).

    Self-loops and duplicates removed, ids compacted to [0, V); symmetrised
    graphs keep one (min, max) entry per unordered pair."""
    lib = load()
    p = _lib.RmatParams(scale, edgefactor, seed, a, b, c, int(symmetrize), int(permute))
    h = C.c_void_p()
    check(lib.plato_rmat_generate(C.byref(p), C.byref(h)), "plato_rmat_generate")
    return _take_edge_list(lib, h)


def read_csv(path, weighted: bool = False) -> tuple:
    """Edge list from CSV text -> (V, src, dst), or (V, src, dst, weights
    float64) when weighted, the reference's csv_parser rules
    (plato/graph/parsers.hpp:226-290; weights with double_decoder, :84-88):
    `path` is a file or a directory of files (read in name order, ".gz"
    inflated); V = largest id + 1."""
    lib = load()
    h = C.c_void_p()
    fn = lib.plato_edge_list_read_csv_weighted if weighted else lib.plato_edge_list_read_csv
    check(fn(os.fsencode(str(path)), C.byref(h)), "plato_edge_list_read_csv")
    return _take_edge_list(lib, h, weighted)


def write_vertex_csv(directory, values, prefix: str = "", files: int = 1, gzip: bool = False) -> None:
    """Writes `v,value` lines for every vertex into `files` CSV files
    <directory>/<prefix><NNNN>.csv[.gz] (float32 -> %g, uint32 -> integer),
    the result layout of the reference's examples (example/pagerank.cc:191-200)."""
    a = np.ascontiguousarray(values)
    if a.dtype == np.float32:
        kind = _lib.PLATO_VALUE_F32
    elif a.dtype == np.uint32:
        kind = _lib.PLATO_VALUE_U32
    else:
        raise TypeError("write_vertex_csv: values must be float32 or uint32")
    check(load().plato_write_vertex_csv(os.fsencode(str(directory)), prefix.encode(), _ptr(a), kind,
                                        a.size, files, int(gzip)), "plato_write_vertex_csv")


class Graph:
    """A graph resident in HBM: CSC (in-edges) + CSR (out-edges), single partition.

    Replaces create_dualmode_seq_from_path (plato/graph/structure.hpp:983-1086)
    for an in-memory edge list.  ``relabel`` lets the engine renumber vertices
    internally by out-degree; results always come back in caller ids."""

    def __init__(self, vertices: int, src, dst, is_directed: bool = True, relabel: bool = True,
                 weights=None):
        self._lib = load()
        src = _u32(src)
        dst = _u32(dst)
        if src.shape != dst.shape:
            raise ValueError("src and dst must have the same length")
        info = _lib.GraphInfo(1 if is_directed else 0, int(vertices), int(src.size),
                              max(int(vertices) - 1, 0))
        h = C.c_void_p()
        flags = PLATO_GRAPH_RELABEL if relabel else PLATO_GRAPH_NO_RELABEL
        if weights is None:
            check(self._lib.plato_graph_create(C.byref(info), _ptr(src), _ptr(dst), flags, C.byref(h)),
                  "plato_graph_create")
        else:
            w = np.ascontiguousarray(weights, dtype=np.float64)
            if w.shape != src.shape:
                raise ValueError("weights must have one entry per edge")
            check(self._lib.plato_graph_create_weighted(C.byref(info), _ptr(src), _ptr(dst), _ptr(w), flags,
                                                        C.byref(h)), "plato_graph_create_weighted")
        self._h = h

    # -- lifetime ---------------------------------------------------------
    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.plato_graph_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self) -> C.c_void_p:
        if not self._h:
            raise ValueError("graph is closed")
        return self._h

    # -- info ---------------------------------------------------------------
    @property
    def info(self) -> GraphInfo:
        i = _lib.GraphInfo()
        check(self._lib.plato_graph_get_info(self.handle, C.byref(i)), "plato_graph_get_info")
        return GraphInfo(bool(i.is_directed), int(i.vertices), int(i.edges), int(i.max_v_i))

    @property
    def vertices(self) -> int:
        return self.info.vertices_

    def device_view(self) -> _lib.GraphDeviceView:
        v = _lib.GraphDeviceView()
        check(self._lib.plato_graph_get_device_view(self.handle, C.byref(v)),
              "plato_graph_get_device_view")
        return v

    def device_bytes(self) -> int:
        b = C.c_uint64()
        check(self._lib.plato_graph_device_bytes(self.handle, C.byref(b)), "plato_graph_device_bytes")
        return int(b.value)

    def out_degrees(self) -> np.ndarray:
        out = np.empty(self.vertices, dtype=np.uint32)
        check(self._lib.plato_graph_out_degrees(self.handle, _ptr(out)), "plato_graph_out_degrees")
        return out

    # -- algorithms (normalised FP32 outputs) -------------------------------
    def pagerank(self, iteration: int = 100, damping: float = 0.85, eps: float = 0.0):
        """Normalised ranks (sum ~ 1; the reference's values are these times V)."""
        out = np.empty(self.vertices, dtype=np.float32)
        o = _lib.PagerankOpts(iteration, damping, eps)
        s = _lib.RunStats()
        check(self._lib.plato_pagerank(self.handle, C.byref(o), _ptr(out), C.byref(s)),
              "plato_pagerank")
        return out, RunStats.from_c(s)

    def pagerank_device(self, d_out: int, iteration: int, damping: float = 0.85,
                        eps: float = 0.0, stream: int = 0):
        """PageRank into device memory `d_out` (a CUDA pointer) on `stream`."""
        o = _lib.PagerankOpts(iteration, damping, eps)
        s = _lib.RunStats()
        check(self._lib.plato_pagerank_device(self.handle, C.byref(o), C.c_void_p(d_out),
                                              C.c_void_p(stream), C.byref(s)),
              "plato_pagerank_device")
        return RunStats.from_c(s)

    def weighted_pagerank(self, iteration: int = 100, damping: float = 0.85, eps: float = 0.001):
        """algo::weighted_pagerank (plato/algo/pagerank/weighted_pagerank.hpp:60-149)
        on a graph built with weights -> (ranks float32 [V] in the reference's
        units, stats)."""
        out = np.empty(self.vertices, dtype=np.float32)
        o = _lib.PagerankOpts(iteration, damping, eps)
        s = _lib.RunStats()
        check(self._lib.plato_weighted_pagerank(self.handle, C.byref(o), _ptr(out), C.byref(s)),
              "plato_weighted_pagerank")
        return out, RunStats.from_c(s)

    def personalized_pagerank(self, src: int, iteration: int = 100, damping: float = 0.85,
                              eps: float = 0.0, mode: int = PLATO_PPR_PULL):
        out = np.empty(self.vertices, dtype=np.float32)
        o = _lib.PprOpts(iteration, damping, src, eps)
        s = _lib.RunStats()
        check(self._lib.plato_personalized_pagerank(self.handle, C.byref(o), mode, _ptr(out),
                                                    C.byref(s)),
              "plato_personalized_pagerank")
        return out, RunStats.from_c(s)

    def seedset_ppr(self, seeds, iteration: int = 100, damping: float = 0.85, eps: float = 0.0):
        """One seed-set PPR query on the pull engine (trustrank with explicit seeds)."""
        s = _u32(seeds)
        out = np.empty(self.vertices, dtype=np.float32)
        o = _lib.PprOpts(iteration, damping, 0, eps)
        st = _lib.RunStats()
        check(self._lib.plato_seedset_ppr(self.handle, _ptr(s), s.size, C.byref(o), _ptr(out),
                                          C.byref(st)), "plato_seedset_ppr")
        return out, RunStats.from_c(st)

    def trustrank(self, good=None, iteration: int = 100, damping: float = 0.85, seed_num: int = 100,
                  select_method: int = 0, eps: float = 0.001, random_seed: int = 0):
        """algo::trustrank with select_good_seeds (trustrank.hpp:88-259) ->
        (ranks float32 [V], seeds uint32 (sorted caller ids), stats).
        good: bool/uint8 [V] or None (every vertex good); select_method 0
        inverse PageRank, 1 PageRank, 2 random (seeded by random_seed)."""
        V = self.vertices
        out = np.empty(V, dtype=np.float32)
        gv = None if good is None else np.ascontiguousarray(np.asarray(good).astype(np.uint8))
        if gv is not None and gv.size != V:
            raise ValueError("trustrank: good must have one entry per vertex")
        seeds = np.empty(max(seed_num, V if V <= seed_num else 0, 1), dtype=np.uint32)
        n = C.c_uint32()
        o = _lib.TrustrankOpts(iteration, damping, seed_num, select_method, eps, random_seed)
        st = _lib.RunStats()
        check(self._lib.plato_trustrank(self.handle, C.byref(o), _ptr(gv) if gv is not None else None,
                                        _ptr(out), _ptr(seeds), C.byref(n), C.byref(st)), "plato_trustrank")
        return out, seeds[:n.value].copy(), RunStats.from_c(st)

    def ppr_batch_k_tile(self, K: int) -> int:
        """Column-tile width the autotuner picks for K columns (cached per graph)."""
        kt = C.c_uint32()
        _lib.check(_lib.load().plato_ppr_batch_k_tile(self.handle, K, C.byref(kt)), "plato_ppr_batch_k_tile")
        return int(kt.value)

    def ppr_batch(self, seed_sets, max_iterations: int = 100, damping: float = 0.85,
                  eps: float = 1e-6, topk: int = 0, k_tile: int = 0, ranks: bool = False):
        """Batched multi-source PPR: one query per seed set (trustrank seed-set
        semantics).  -> dict(iterations [K], ranks [K, V] or None,
        topk_ids [K, topk], topk_vals [K, topk])."""
        K = len(seed_sets)
        off = np.zeros(K + 1, dtype=np.uint64)
        off[1:] = np.cumsum([len(s) for s in seed_sets])
        flat = _u32(np.concatenate([np.asarray(s, dtype=np.uint32) for s in seed_sets])
                    if K else np.zeros(0, np.uint32))
        V = self.vertices
        out_r = np.empty((K, V), dtype=np.float32) if ranks else None
        ids = np.empty((K, topk), dtype=np.uint32) if topk else None
        vals = np.empty((K, topk), dtype=np.float32) if topk else None
        its = np.empty(K, dtype=np.uint32)
        o = _lib.PprBatchOpts(max_iterations, damping, eps, topk, k_tile)
        check(self._lib.plato_ppr_batch(self.handle, K, _ptr(off), _ptr(flat), C.byref(o),
                                        _ptr(out_r) if ranks else None,
                                        _ptr(ids) if topk else None,
                                        _ptr(vals) if topk else None, _ptr(its)),
              "plato_ppr_batch")
        return {"iterations": its, "ranks": out_r, "topk_ids": ids, "topk_vals": vals}

    def bfs(self, root: int, push_threshold: float = 0.05, parents: bool = True,
            levels: bool = True):
        """-> (levels uint32 [V] with PLATO_LEVEL_UNREACHED or None, parents or None, stats)."""
        V = self.vertices
        lev = np.empty(V, dtype=np.uint32) if levels else None
        par = np.empty(V, dtype=np.uint32) if parents else None
        o = _lib.BfsOpts(root)
        eo = _lib.DualmodeOpts(push_threshold)
        s = _lib.RunStats()
        check(self._lib.plato_bfs(self.handle, C.byref(o), C.byref(eo),
                                  _ptr(lev) if levels else None,
                                  _ptr(par) if parents else None, C.byref(s)), "plato_bfs")
        return lev, par, RunStats.from_c(s)

    def connected_components(self, push_threshold: float = 0.05, labels: bool = True):
        """Label propagation (plato/algo/cgm/connected_component.hpp) ->
        (labels uint32 [V] or None, summary dict, stats): labels[v] = smallest
        caller id reaching v (component minimum on undirected graphs)."""
        lab = np.empty(self.vertices, dtype=np.uint32) if labels else None
        eo = _lib.DualmodeOpts(push_threshold)
        sm = _lib.CcSummary()
        s = _lib.RunStats()
        check(self._lib.plato_connected_components(self.handle, C.byref(eo), _ptr(lab) if labels else None,
                                                   C.byref(sm), C.byref(s)), "plato_connected_components")
        summary = {"components": int(sm.components), "major_label": int(sm.major_label),
                   "major_vertices": int(sm.major_vertices), "major_edges": int(sm.major_edges)}
        return lab, summary, RunStats.from_c(s)

    def hyperanf(self, iteration: int = 20, bits: int = 6, push_threshold: float = 0.05,
                 registers: bool = False):
        """algo::hyperanf (plato/algo/hyperanf/hyperanf.hpp:83-195) ->
        (avg_distance, anfs float64 [n], registers uint8 [V, 2^bits] or None,
        stats)."""
        o = _lib.HyperanfOpts(iteration, bits)
        eo = _lib.DualmodeOpts(push_threshold)
        avg = C.c_double()
        anfs = np.empty(iteration + 1, dtype=np.float64)
        n = C.c_uint32()
        regs = np.empty((self.vertices, 1 << bits), dtype=np.uint8) if registers and 4 <= bits <= 16 else None
        s = _lib.RunStats()
        check(self._lib.plato_hyperanf(self.handle, C.byref(o), C.byref(eo), C.byref(avg), _ptr(anfs),
                                       C.byref(n), _ptr(regs) if regs is not None else None, C.byref(s)),
              "plato_hyperanf")
        return float(avg.value), anfs[: n.value].copy(), regs, RunStats.from_c(s)

    def nstep_degrees(self, step: int = 20, bits: int = 6, kind: str = "both", is_directed=None,
                      targets=None, push_threshold: float = 0.05):
        """nstepdegrees_t::compute (plato/algo/nstepdegrees/nstepdegrees.hpp:380-402)
        -> (in_degrees uint32 [V], out_degrees uint32 [V], stats); step < 0
        means until nothing changes (the CLI's -1); targets: bool [V] by
        caller id or None for every vertex."""
        kinds = {"in": 1, "out": 2, "both": 3}
        if kind not in kinds:
            raise PlatoError(1, "nstep_degrees", f"kind must be in/out/both, got {kind!r}")
        if is_directed is None:
            is_directed = self.info.is_directed_
        o = _lib.NstepOpts(0xFFFFFFFF if step < 0 else step, bits, kinds[kind], int(bool(is_directed)))
        eo = _lib.DualmodeOpts(push_threshold)
        tg = None
        if targets is not None:
            tg = np.ascontiguousarray(np.asarray(targets, dtype=bool).astype(np.uint8))
            if tg.size != self.vertices:
                raise PlatoError(1, "nstep_degrees", "targets must have one entry per vertex")
        din = np.empty(self.vertices, dtype=np.uint32)
        dout = np.empty(self.vertices, dtype=np.uint32)
        s = _lib.RunStats()
        check(self._lib.plato_nstep_degrees(self.handle, C.byref(o), C.byref(eo),
                                            _ptr(tg) if tg is not None else None, _ptr(din), _ptr(dout),
                                            C.byref(s)), "plato_nstep_degrees")
        return din, dout, RunStats.from_c(s)


# ---- reference-shaped entry points -------------------------------------------

def pagerank(graph: Graph, opts: pagerank_opts_t | None = None) -> np.ndarray:
    """algo::pagerank (plato/algo/pagerank/pagerank.hpp:60-149): ranks in the
    reference's units (initial rank 1.0, teleport 1-d), float64 array [V]."""
    opts = opts or pagerank_opts_t()
    r, _ = graph.pagerank(opts.iteration_, opts.damping_, opts.eps_)
    return r.astype(np.float64) * graph.vertices


def personalized_pagerank(graph: Graph, opts: personalized_pagerank_opts_t | None = None,
                          pushpull: bool = False) -> np.ndarray:
    """algo::personalized_pagerank: the pull-only overload
    (personalized_pagerank.hpp:40-134) or, with pushpull=True, the dual-mode
    overload taking in- and out-edges (:137-275)."""
    opts = opts or personalized_pagerank_opts_t()
    r, _ = graph.personalized_pagerank(opts.src_, opts.iteration_, opts.damping_, opts.eps_,
                                       PLATO_PPR_PUSHPULL if pushpull else PLATO_PPR_PULL)
    return r.astype(np.float64)


def breadth_first_search(graph: Graph, opts: bfs_opts_t | None = None,
                         engine_opts: dualmode_engine_opts_t | None = None) -> int:
    """algo::breadth_first_search (plato/algo/bfs/bfs.hpp:55-155): visited count."""
    opts = opts or bfs_opts_t()
    eo = engine_opts or dualmode_engine_opts_t()
    _, _, st = graph.bfs(opts.root_, eo.push_threshold_, parents=False)
    return st.visited


class PPRServer:
    """Continuous-batching personalized PageRank server over a resident Graph.

    submit() queues a seed set; step() admits queued requests into free slots
    (bounded by ``hbm_budget_bytes``), runs one iteration over every live
    query and retires the converged ones with their top-k; poll() returns
    finished results."""

    def __init__(self, graph: Graph, max_slots: int = 256, hbm_budget_bytes: int = 8 << 30,
                 max_iterations: int = 200, damping: float = 0.85, eps: float = 1e-6,
                 topk: int = 100):
        self._lib = load()
        self.graph = graph
        self.topk = topk
        o = _lib.ServerOpts(max_slots, hbm_budget_bytes, max_iterations, damping, eps, topk)
        h = C.c_void_p()
        check(self._lib.plato_server_create(graph.handle, C.byref(o), C.byref(h)),
              "plato_server_create")
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            self._lib.plato_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def submit(self, seeds) -> int:
        s = _u32(seeds)
        rid = C.c_uint64()
        check(self._lib.plato_server_submit(self._h, _ptr(s), s.size, C.byref(rid)),
              "plato_server_submit")
        return int(rid.value)

    def step(self) -> None:
        check(self._lib.plato_server_step(self._h), "plato_server_step")

    def poll(self):
        """-> (request_id, topk_ids, topk_vals, iterations) or None."""
        rid = C.c_uint64()
        ids = np.empty(self.topk, dtype=np.uint32)
        vals = np.empty(self.topk, dtype=np.float32)
        it = C.c_uint32()
        rc = self._lib.plato_server_poll(self._h, C.byref(rid), _ptr(ids), _ptr(vals), C.byref(it))
        if rc == _lib.PLATO_ENOTFOUND:
            return None
        check(rc, "plato_server_poll")
        return int(rid.value), ids, vals, int(it.value)

    def stats(self):
        live, queued = C.c_uint32(), C.c_uint32()
        done = C.c_uint64()
        check(self._lib.plato_server_stats(self._h, C.byref(live), C.byref(queued), C.byref(done)),
              "plato_server_stats")
        return {"live": int(live.value), "queued": int(queued.value), "completed": int(done.value)}
