"""Oracle package — TEST INFRASTRUCTURE ONLY.

``RefGraph`` wraps ``ref_cpu.c`` (liboracle build: ``python -m oracle.build``),
the C/OpenMP restatement of the reference's dual-mode engine path at one
partition in double precision (see the header of ref_cpu.c for the file:line
of every rule it follows).  ``fp64`` is an independent FP64 power iteration /
serial BFS used to cross-check the restatement.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg use
this package, and only as the checker or the timed CPU baseline; the
plato_b200 package never imports it.

Parity status: the reference ships no golden vectors for pagerank / ppr / bfs
results (its algorithm directories have no tests), so algorithm outputs are
unpinned by the reference's own tests; the substrate (DCSC counts,
out-degrees, aggregate-message sums) is pinned against the reference's
substrate tests via tests/golden/.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libref_cpu.so"

_lib = None


def load():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            from .build import build
            build()
        lib = C.CDLL(str(LIB_PATH))
        P = C.c_void_p
        lib.ref_graph_build.restype = P
        lib.ref_graph_build.argtypes = [C.c_uint32, C.c_uint64, P, P, C.c_int]
        lib.ref_graph_free.argtypes = [P]
        lib.ref_graph_dcsc_columns.restype = C.c_uint64
        lib.ref_graph_dcsc_columns.argtypes = [P]
        lib.ref_graph_stored_edges.restype = C.c_uint64
        lib.ref_graph_stored_edges.argtypes = [P]
        lib.ref_out_degrees.argtypes = [P, P]
        lib.ref_in_adjacency.argtypes = [P, P, P, P]
        lib.ref_aggregate_count.restype = C.c_uint64
        lib.ref_aggregate_count.argtypes = [P, P]
        lib.ref_pagerank.argtypes = [P, C.c_uint32, C.c_double, C.c_double, P, P, P]
        lib.ref_ppr.argtypes = [P, C.c_uint32, C.c_uint32, C.c_double, C.c_double, C.c_int, P, P, P,
                                P, P]
        lib.ref_seedset_ppr.argtypes = [P, C.c_uint32, P, C.c_uint32, C.c_double, C.c_double, P,
                                        P, P]
        lib.ref_bfs.argtypes = [P, C.c_uint32, C.c_double, P, P, P, P, P]
        lib.ref_max_threads.restype = C.c_int
        lib.ref_rmat.argtypes = [C.c_uint32, C.c_uint32, C.c_uint64, C.c_double, C.c_double,
                                 C.c_double, C.c_int, C.POINTER(C.c_uint32), C.POINTER(C.c_uint64),
                                 C.POINTER(C.POINTER(C.c_uint32)), C.POINTER(C.POINTER(C.c_uint32))]
        lib.ref_rmat_free.argtypes = [P]
        _lib = lib
    return _lib


def _p(a: np.ndarray) -> C.c_void_p:
    return C.c_void_p(a.ctypes.data)


def max_threads() -> int:
    return int(load().ref_max_threads())


def rmat(scale: int, edgefactor: int, seed: int, symmetrize: bool = False,
         a: float = 0.57, b: float = 0.19, c: float = 0.19):
    """Seeded RMAT edge list (rmat.c, OpenMP) -> (V, src uint32, dst uint32),
    sorted by (src, dst), self-loops and duplicates removed, ids compacted."""
    lib = load()
    V, n = C.c_uint32(), C.c_uint64()
    ps, pd = C.POINTER(C.c_uint32)(), C.POINTER(C.c_uint32)()
    r = lib.ref_rmat(scale, edgefactor, seed, a, b, c, 1 if symmetrize else 0, C.byref(V), C.byref(n),
                     C.byref(ps), C.byref(pd))
    if r != 0:
        raise (ValueError if r == 1 else MemoryError)(f"ref_rmat failed ({r})")
    try:
        src = np.ctypeslib.as_array(ps, shape=(n.value,)).copy() if n.value else np.empty(0, np.uint32)
        dst = np.ctypeslib.as_array(pd, shape=(n.value,)).copy() if n.value else np.empty(0, np.uint32)
    finally:
        lib.ref_rmat_free(C.cast(ps, C.c_void_p))
        lib.ref_rmat_free(C.cast(pd, C.c_void_p))
    return int(V.value), src, dst


class RefGraph:
    """The reference's DCSC + BCSR at one partition (ref_cpu.c)."""

    def __init__(self, vertices: int, src, dst, is_directed: bool = True):
        self._lib = load()
        self.src = np.ascontiguousarray(src, dtype=np.uint32)
        self.dst = np.ascontiguousarray(dst, dtype=np.uint32)
        self.vertices = int(vertices)
        self.is_directed = bool(is_directed)
        self._h = self._lib.ref_graph_build(self.vertices, self.src.size, _p(self.src),
                                            _p(self.dst), 1 if is_directed else 0)
        if not self._h:
            raise MemoryError("ref_graph_build failed")

    def close(self):
        if getattr(self, "_h", None):
            self._lib.ref_graph_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def dcsc_columns(self) -> int:
        return int(self._lib.ref_graph_dcsc_columns(self._h))

    @property
    def stored_edges(self) -> int:
        return int(self._lib.ref_graph_stored_edges(self._h))

    def out_degrees(self) -> np.ndarray:
        out = np.empty(self.vertices, dtype=np.uint32)
        self._lib.ref_out_degrees(self._h, _p(out))
        return out

    def aggregate_count(self):
        values = np.zeros(self.vertices, dtype=np.int32)
        s = self._lib.ref_aggregate_count(self._h, _p(values))
        return int(s), values

    def pagerank(self, iteration: int = 100, damping: float = 0.85, eps: float = 0.0):
        """Reference units (ranks start at 1.0) -> (ranks float64 [V], epochs, delta)."""
        out = np.empty(self.vertices, dtype=np.float64)
        ep = C.c_uint32()
        de = C.c_double()
        self._lib.ref_pagerank(self._h, iteration, damping, eps, _p(out), C.byref(ep), C.byref(de))
        return out, int(ep.value), float(de.value)

    def ppr(self, src: int, iteration: int = 100, damping: float = 0.85, eps: float = 0.0,
            pushpull: bool = False):
        """-> (ranks float64 [V], epochs, push_epochs, mode_trace bits, delta)."""
        out = np.empty(self.vertices, dtype=np.float64)
        ep, pe = C.c_uint32(), C.c_uint32()
        tr = C.c_uint64()
        de = C.c_double()
        r = self._lib.ref_ppr(self._h, src, iteration, damping, eps, 1 if pushpull else 0, _p(out),
                              C.byref(ep), C.byref(pe), C.byref(tr), C.byref(de))
        if r != 0:
            raise ValueError("ref_ppr: bad arguments")
        return out, int(ep.value), int(pe.value), int(tr.value), float(de.value)

    def seedset_ppr(self, seeds, iteration: int = 100, damping: float = 0.85, eps: float = 0.0):
        s = np.ascontiguousarray(seeds, dtype=np.uint32)
        out = np.empty(self.vertices, dtype=np.float64)
        ep = C.c_uint32()
        de = C.c_double()
        r = self._lib.ref_seedset_ppr(self._h, s.size, _p(s), iteration, damping, eps, _p(out),
                                      C.byref(ep), C.byref(de))
        if r != 0:
            raise ValueError("ref_seedset_ppr: bad arguments")
        return out, int(ep.value), float(de.value)

    def bfs(self, root: int, push_threshold: float = 0.05):
        """-> (levels uint32 [V] (0xFFFFFFFF unreached), parents, visited, trace bits, epochs)."""
        lev = np.empty(self.vertices, dtype=np.uint32)
        par = np.empty(self.vertices, dtype=np.uint32)
        vis = C.c_uint64()
        tr = C.c_uint64()
        ep = C.c_uint32()
        r = self._lib.ref_bfs(self._h, root, push_threshold, _p(lev), _p(par), C.byref(vis),
                              C.byref(tr), C.byref(ep))
        if r != 0:
            raise ValueError("ref_bfs: bad arguments")
        return lev, par, int(vis.value), int(tr.value), int(ep.value)


def trustrank_seeds(vertices: int, src, dst, is_directed: bool, seed_num: int, select_method: int,
                    good=None):
    """select_good_seeds (plato/algo/trustrank/trustrank.hpp:88-146) for
    methods 0 (inverse PageRank) and 1 (PageRank) -> (sorted seed ids, the
    ranks used).  Ranks are the reference's default PageRank run
    (pagerank_opts_t: 100 epochs, 0.85, eps 0.001; pagerank.hpp:39-46) on
    the graph, transposed for method 0 (generate_rank_pairs over the
    out-edges, trustrank.hpp:52-71); order: rank descending, id ascending."""
    is_good = (lambda v: True) if good is None else (lambda v: bool(good[v]))
    if vertices <= seed_num:
        return np.array([v for v in range(vertices) if is_good(v)], dtype=np.uint32), None
    s, d = (dst, src) if select_method == 0 else (src, dst)
    g = RefGraph(vertices, s, d, is_directed)
    try:
        ranks, _, _ = g.pagerank(100, 0.85, 0.001)
    finally:
        g.close()
    order = sorted(range(vertices), key=lambda v: (-ranks[v], v))[:seed_num]
    return np.array(sorted(v for v in order if is_good(v)), dtype=np.uint32), ranks
