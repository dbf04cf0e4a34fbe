"""The reference's own engine path, compiled — TEST INFRASTRUCTURE ONLY.

``ReferenceGraph`` wraps ``oracle/_ref/libplato_ref.so``, built by
``oracle.build.build_ref`` from ``oracle/ref_shim/plato_ref_shim.cpp`` and the
reference's own headers (plato/engine/dualmode.hpp, plato/graph/*,
plato/algo/{pagerank,ppr,bfs,trustrank,cgm,hyperanf}/*.hpp, and in a second
library weighted_pagerank.hpp) where they lie in the
reference tree, against one-rank stand-ins for MPI, glog, gflags, libnuma,
libhdfs, boost and yas (oracle/ref_shim/include).  The library is only
present where the reference tree was available at build time (it travels
with the rest of the built files); ``available()`` says whether it loaded.

Uses: tests/golden/make_golden.py writes the reference's outputs on the
fixture graphs to tests/golden/ref_golden.npz (the pins of the oracle and of
the GPU path); CPU tests compare the oracle with it live; bench.py's reference
arm times it.  Nothing in the product imports this module.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "_ref" / "libplato_ref.so"
LIB_W_PATH = Path(__file__).resolve().parent / "_ref" / "libplato_ref_weighted.so"

_lib = None
_lib_w = None


def load():
    """The compiled reference, or None when it was not built here."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            return None
        lib = C.CDLL(str(LIB_PATH))
        P = C.c_void_p
        lib.refp_graph_build.restype = P
        lib.refp_graph_build.argtypes = [C.c_uint32, C.c_uint64, P, P, C.c_int]
        lib.refp_graph_free.argtypes = [P]
        lib.refp_graph_info.argtypes = [P, P, P, P]
        lib.refp_pagerank.argtypes = [P, C.c_uint32, C.c_double, C.c_double, P, P, P, C.c_uint32]
        lib.refp_ppr.argtypes = [P, C.c_uint32, C.c_uint32, C.c_double, C.c_double, C.c_int, P, P]
        lib.refp_trustrank.argtypes = [P, P, C.c_uint32, C.c_uint32, C.c_uint32, C.c_double, C.c_double, P, P]
        lib.refp_threads.restype = C.c_int
        lib.refp_bfs.restype = C.c_uint64
        lib.refp_bfs.argtypes = [P, C.c_uint32, P, C.c_uint32, P, P]
        lib.refp_cc.argtypes = [P, P, P, P, P, P]
        lib.refp_hyperanf.argtypes = [P, C.c_uint32, C.c_uint32, P]
        _lib = lib
    return _lib


def load_weighted():
    """The compiled reference's weighted PageRank, or None."""
    global _lib_w
    if _lib_w is None:
        if not LIB_W_PATH.exists():
            return None
        lib = C.CDLL(str(LIB_W_PATH))
        P = C.c_void_p
        lib.refp_wgraph_build.restype = P
        lib.refp_wgraph_build.argtypes = [C.c_uint32, C.c_uint64, P, P, P, C.c_int]
        lib.refp_wgraph_free.argtypes = [P]
        lib.refp_weighted_pagerank.argtypes = [P, C.c_uint32, C.c_double, C.c_double, P, P]
        _lib_w = lib
    return _lib_w


def available() -> bool:
    return load() is not None


def threads() -> int:
    """OpenMP threads the reference's loops use (cluster_info_t::threads_)."""
    return int(load().refp_threads())


class ReferenceGraph:
    """create_dualmode_seq_from_path's BCSR + DCSC built from an edge list in
    memory (compact caller ids), run through the reference's algorithms."""

    def __init__(self, vertices: int, src, dst, is_directed: bool = True):
        self._lib = load()
        if self._lib is None:
            raise FileNotFoundError(f"{LIB_PATH} was not built (the reference tree was absent at build time)")
        s = np.ascontiguousarray(src, dtype=np.uint32)
        d = np.ascontiguousarray(dst, dtype=np.uint32)
        self._h = self._lib.refp_graph_build(int(vertices), s.size, s.ctypes.data, d.ctypes.data,
                                             1 if is_directed else 0)
        if not self._h:
            raise RuntimeError("the reference's graph build failed")
        v, m, e = C.c_uint32(), C.c_uint32(), C.c_uint64()
        self._lib.refp_graph_info(self._h, C.byref(v), C.byref(m), C.byref(e))
        self.vertices, self.max_v_i, self.edges = int(v.value), int(m.value), int(e.value)

    def close(self):
        if getattr(self, "_h", None):
            self._lib.refp_graph_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def pagerank(self, iteration=100, damping=0.85, eps=0.0):
        """algo::pagerank -> (ranks float64 [max_v_i + 1], epochs, per-epoch deltas)."""
        out = np.empty(self.max_v_i + 1)
        ep = C.c_uint32()
        dl = np.zeros(max(iteration, 1))
        self._lib.refp_pagerank(self._h, iteration, damping, eps, out.ctypes.data, C.byref(ep), dl.ctypes.data,
                                dl.size)
        return out, int(ep.value), dl[:min(int(ep.value), dl.size)].copy()

    def ppr(self, src, iteration=100, damping=0.85, eps=0.0, pushpull=False):
        """algo::personalized_pagerank (pull-only, or dual-mode) -> (ranks, epochs)."""
        out = np.empty(self.max_v_i + 1)
        ep = C.c_uint32()
        self._lib.refp_ppr(self._h, int(src), iteration, damping, eps, 1 if pushpull else 0, out.ctypes.data,
                           C.byref(ep))
        return out, int(ep.value)

    def trustrank(self, good, seed_num=100, select_method=0, iteration=100, damping=0.85, eps=0.001):
        """algo::trustrank with select_good_seeds (methods 0 and 1) -> (ranks, trust epochs)."""
        g = np.ascontiguousarray(good, dtype=np.uint8)
        out = np.empty(self.max_v_i + 1)
        ep = C.c_uint32()
        r = self._lib.refp_trustrank(self._h, g.ctypes.data, seed_num, select_method, iteration, damping, eps,
                                     out.ctypes.data, C.byref(ep))
        if r != 0:
            raise ValueError("select_method must be 0 or 1")
        return out, int(ep.value)

    def connected_components(self):
        """connected_component_t::compute -> (labels uint32 [max_v_i + 1],
        components, major label, major vertices, major edges)."""
        lab = np.empty(self.max_v_i + 1, np.uint32)
        comps, major, mv, me = C.c_uint64(), C.c_uint32(), C.c_uint64(), C.c_uint64()
        self._lib.refp_cc(self._h, lab.ctypes.data, C.byref(comps), C.byref(major), C.byref(mv), C.byref(me))
        return lab, int(comps.value), int(major.value), int(mv.value), int(me.value)

    def hyperanf(self, bits=6, iteration=20):
        """algo::hyperanf<..., bits> -> the average distance (bits 6 or 8)."""
        avg = C.c_double()
        if self._lib.refp_hyperanf(self._h, bits, iteration, C.byref(avg)) != 0:
            raise ValueError("bits must be 6 or 8")
        return float(avg.value)

    def bfs(self, root, cap=256):
        """algo::breadth_first_search -> (visited, vertices activated per epoch,
        push/pull trace bits of the engine's choice per epoch)."""
        act = np.zeros(cap, np.uint64)
        ep = C.c_uint32()
        tr = C.c_uint64()
        vis = self._lib.refp_bfs(self._h, int(root), act.ctypes.data, cap, C.byref(ep), C.byref(tr))
        return int(vis), act[:min(int(ep.value), cap)].copy(), int(tr.value)


class WeightedReferenceGraph:
    """create_dcsc_seqs_from_path<double>'s DCSC built from a weighted edge
    list in memory, run through the reference's algo::weighted_pagerank."""

    def __init__(self, vertices: int, src, dst, weights, is_directed: bool = True):
        self._lib = load_weighted()
        if self._lib is None:
            raise FileNotFoundError(f"{LIB_W_PATH} was not built (the reference tree was absent at build time)")
        s = np.ascontiguousarray(src, dtype=np.uint32)
        d = np.ascontiguousarray(dst, dtype=np.uint32)
        w = np.ascontiguousarray(weights, dtype=np.float64)
        self._h = self._lib.refp_wgraph_build(int(vertices), s.size, s.ctypes.data, d.ctypes.data, w.ctypes.data,
                                              1 if is_directed else 0)
        if not self._h:
            raise RuntimeError("the reference's weighted graph build failed")
        self.vertices = int(vertices)

    def close(self):
        if getattr(self, "_h", None):
            self._lib.refp_wgraph_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def weighted_pagerank(self, iteration=100, damping=0.85, eps=0.001):
        """-> (ranks float64 [V] in the reference's units, epochs)."""
        out = np.empty(self.vertices)
        ep = C.c_uint32()
        self._lib.refp_weighted_pagerank(self._h, iteration, damping, eps, out.ctypes.data, C.byref(ep))
        return out, int(ep.value)
