"""ctypes binding of include/plato_b200.h (libplato_b200.so, built in-tree).

Loading fails loudly when the shared library is missing: there is no CPU
fallback behind this package.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libplato_b200.so"

PLATO_OK, PLATO_EINVAL, PLATO_ENOMEM, PLATO_ECUDA, PLATO_ETIMEDOUT, PLATO_EBUSY, PLATO_ENOTFOUND = range(7)
PLATO_VALUE_F32, PLATO_VALUE_U32 = 0, 1  # plato_write_vertex_csv value types
PLATO_LEVEL_UNREACHED = 0xFFFFFFFF
PLATO_GRAPH_RELABEL, PLATO_GRAPH_NO_RELABEL = 0x1, 0x2
PLATO_PPR_PULL, PLATO_PPR_PUSHPULL = 0, 1

STATUS_NAMES = {0: "PLATO_OK", 1: "PLATO_EINVAL", 2: "PLATO_ENOMEM", 3: "PLATO_ECUDA",
                4: "PLATO_ETIMEDOUT", 5: "PLATO_EBUSY", 6: "PLATO_ENOTFOUND"}


class GraphInfo(C.Structure):
    _fields_ = [("is_directed", C.c_int32), ("vertices", C.c_uint32), ("edges", C.c_uint64),
                ("max_v_i", C.c_uint32)]


class PagerankOpts(C.Structure):
    _fields_ = [("iteration", C.c_uint32), ("damping", C.c_double), ("eps", C.c_double)]


class PprOpts(C.Structure):
    _fields_ = [("iteration", C.c_uint32), ("damping", C.c_double), ("src", C.c_uint32),
                ("eps", C.c_double)]


class BfsOpts(C.Structure):
    _fields_ = [("root", C.c_uint32)]


class DualmodeOpts(C.Structure):
    _fields_ = [("push_threshold", C.c_double)]


class RunStats(C.Structure):
    _fields_ = [("iterations", C.c_uint32), ("push_iterations", C.c_uint32),
                ("pull_iterations", C.c_uint32), ("reserved", C.c_uint32), ("delta", C.c_double),
                ("visited", C.c_uint64), ("mode_trace", C.c_uint64)]


class TrustrankOpts(C.Structure):
    _fields_ = [("iteration", C.c_uint32), ("damping", C.c_double), ("seed_num", C.c_uint32),
                ("select_method", C.c_uint32), ("eps", C.c_double), ("random_seed", C.c_uint64)]


class CcSummary(C.Structure):
    _fields_ = [("components", C.c_uint64), ("major_label", C.c_uint32), ("major_vertices", C.c_uint64),
                ("major_edges", C.c_uint64)]


class HyperanfOpts(C.Structure):
    _fields_ = [("iteration", C.c_uint32), ("bits", C.c_uint32)]


class NstepOpts(C.Structure):
    _fields_ = [("step", C.c_uint32), ("bits", C.c_uint32), ("type", C.c_uint32), ("is_directed", C.c_int32)]


class GraphDeviceView(C.Structure):
    _fields_ = [("vertices", C.c_uint32), ("is_directed", C.c_int32), ("edges", C.c_uint64),
                ("stored_edges", C.c_uint64), ("in_offsets", C.c_void_p), ("in_adj", C.c_void_p),
                ("out_offsets", C.c_void_p), ("out_adj", C.c_void_p), ("out_degree", C.c_void_p),
                ("in_degree", C.c_void_p), ("to_internal", C.c_void_p), ("to_external", C.c_void_p)]


class PprBatchOpts(C.Structure):
    _fields_ = [("max_iterations", C.c_uint32), ("damping", C.c_double), ("eps", C.c_double),
                ("topk", C.c_uint32), ("k_tile", C.c_uint32)]


class ServerOpts(C.Structure):
    _fields_ = [("max_slots", C.c_uint32), ("hbm_budget_bytes", C.c_uint64),
                ("max_iterations", C.c_uint32), ("damping", C.c_double), ("eps", C.c_double),
                ("topk", C.c_uint32)]


class RmatParams(C.Structure):
    _fields_ = [("scale", C.c_uint32), ("edgefactor", C.c_uint32), ("seed", C.c_uint64),
                ("a", C.c_double), ("b", C.c_double), ("c", C.c_double),
                ("symmetrize", C.c_int32), ("permute", C.c_int32)]


P = C.c_void_p
u32p = C.POINTER(C.c_uint32)
u64p = C.POINTER(C.c_uint64)
f32p = C.POINTER(C.c_float)

# name -> (restype, argtypes); every symbol declared in include/plato_b200.h
SIGNATURES = {
    "plato_last_error": (C.c_char_p, []),
    "plato_kernel_launches": (C.c_uint64, []),
    "plato_version": (C.c_char_p, []),
    "plato_profile_enable": (C.c_int, [C.c_int]),
    "plato_profile_reset": (C.c_int, []),
    "plato_profile_read": (C.c_int, [C.c_char_p, C.POINTER(C.c_double), u64p]),
    "plato_graph_create": (C.c_int, [C.POINTER(GraphInfo), P, P, C.c_uint32, C.POINTER(P)]),
    "plato_graph_create_weighted": (C.c_int, [C.POINTER(GraphInfo), P, P, P, C.c_uint32, C.POINTER(P)]),
    "plato_weighted_pagerank": (C.c_int, [P, C.POINTER(PagerankOpts), P, C.POINTER(RunStats)]),
    "plato_graph_destroy": (C.c_int, [P]),
    "plato_graph_get_info": (C.c_int, [P, C.POINTER(GraphInfo)]),
    "plato_graph_get_device_view": (C.c_int, [P, C.POINTER(GraphDeviceView)]),
    "plato_graph_out_degrees": (C.c_int, [P, P]),
    "plato_graph_device_bytes": (C.c_int, [P, u64p]),
    "plato_pagerank": (C.c_int, [P, C.POINTER(PagerankOpts), P, C.POINTER(RunStats)]),
    "plato_personalized_pagerank": (C.c_int, [P, C.POINTER(PprOpts), C.c_int, P, C.POINTER(RunStats)]),
    "plato_connected_components": (C.c_int, [P, C.POINTER(DualmodeOpts), P, C.POINTER(CcSummary),
                                            C.POINTER(RunStats)]),
    "plato_trustrank": (C.c_int, [P, C.POINTER(TrustrankOpts), P, P, P, C.POINTER(C.c_uint32),
                                 C.POINTER(RunStats)]),
    "plato_hyperanf": (C.c_int, [P, C.POINTER(HyperanfOpts), C.POINTER(DualmodeOpts), C.POINTER(C.c_double),
                                P, C.POINTER(C.c_uint32), P, C.POINTER(RunStats)]),
    "plato_nstep_degrees": (C.c_int, [P, C.POINTER(NstepOpts), C.POINTER(DualmodeOpts), P, P, P,
                                     C.POINTER(RunStats)]),
    "plato_bfs": (C.c_int, [P, C.POINTER(BfsOpts), C.POINTER(DualmodeOpts), P, P, C.POINTER(RunStats)]),
    "plato_seedset_ppr": (C.c_int, [P, P, C.c_uint32, C.POINTER(PprOpts), P, C.POINTER(RunStats)]),
    "plato_pagerank_device": (C.c_int, [P, C.POINTER(PagerankOpts), P, P, C.POINTER(RunStats)]),
    "plato_pagerank_csc_noalloc": (C.c_int, [C.c_uint32, C.c_uint64, P, P, P,
                                             C.POINTER(PagerankOpts), P, P, C.POINTER(RunStats)]),
    "plato_partition_layout": (C.c_int, [C.POINTER(GraphInfo), P, P, C.c_uint32, P, C.POINTER(C.c_uint32)]),
    "plato_partition_create": (C.c_int, [C.POINTER(GraphInfo), P, P, C.c_uint32, C.c_uint32,
                                         C.POINTER(C.c_void_p)]),
    "plato_partition_destroy": (C.c_int, [P]),
    "plato_partition_info": (C.c_int, [P, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.POINTER(C.c_uint32),
                                       C.POINTER(C.c_uint64)]),
    "plato_partition_pagerank_init": (C.c_int, [P, P, C.c_double, P]),
    "plato_partition_pagerank_epoch": (C.c_int, [P, P, P, C.c_double, C.c_int, P, P]),
    "plato_partition_ranks": (C.c_int, [P, P, P]),
    "plato_partition_p2p_alloc": (C.c_int, [P, P]),
    "plato_partition_p2p_connect": (C.c_int, [P, P, C.c_uint32]),
    "plato_partition_p2p_connect_local": (C.c_int, [P, C.c_uint32, C.c_uint32]),
    "plato_partition_p2p_reset": (C.c_int, [P]),
    "plato_partition_p2p_init": (C.c_int, [P, C.c_uint32, C.c_double, C.c_double, P]),
    "plato_partition_p2p_epoch": (C.c_int, [P, C.c_uint32, C.c_double, P]),
    "plato_partition_p2p_state": (C.c_int, [P, P, C.POINTER(C.c_void_p), C.POINTER(C.c_uint32)]),
    "plato_partition_p2p_ranks": (C.c_int, [P, P, P, C.POINTER(C.c_uint32)]),
    "plato_diag_pull_ceiling": (C.c_int, [P, C.c_uint32, C.c_uint32, C.POINTER(C.c_double),
                                          C.POINTER(C.c_uint64), C.POINTER(C.c_double)]),
    "plato_diag_batch_ceiling": (C.c_int, [P, C.c_uint32, C.c_uint32, C.c_uint32, C.POINTER(C.c_double),
                                          C.POINTER(C.c_uint64), C.POINTER(C.c_double)]),
    "plato_ppr_batch_k_tile": (C.c_int, [P, C.c_uint32, C.POINTER(C.c_uint32)]),
    "plato_ppr_batch": (C.c_int, [P, C.c_uint32, P, P, C.POINTER(PprBatchOpts), P, P, P, P]),
    "plato_server_create": (C.c_int, [P, C.POINTER(ServerOpts), C.POINTER(P)]),
    "plato_server_submit": (C.c_int, [P, P, C.c_uint32, u64p]),
    "plato_server_step": (C.c_int, [P]),
    "plato_server_poll": (C.c_int, [P, u64p, P, P, u32p]),
    "plato_server_stats": (C.c_int, [P, u32p, u32p, u64p]),
    "plato_server_destroy": (C.c_int, [P]),
    "plato_rmat_generate": (C.c_int, [C.POINTER(RmatParams), C.POINTER(P)]),
    "plato_edge_list_info": (C.c_int, [P, u32p, u64p]),
    "plato_edge_list_data": (C.c_int, [P, C.POINTER(P), C.POINTER(P)]),
    "plato_edge_list_free": (C.c_int, [P]),
    "plato_edge_list_read_csv": (C.c_int, [C.c_char_p, C.POINTER(P)]),
    "plato_edge_list_read_csv_weighted": (C.c_int, [C.c_char_p, C.POINTER(P)]),
    "plato_edge_list_weights": (C.c_int, [P, C.POINTER(P)]),
    "plato_write_vertex_csv": (C.c_int, [C.c_char_p, C.c_char_p, P, C.c_int, C.c_uint32, C.c_uint32,
                                         C.c_int]),
}

_lib = None


class PlatoError(RuntimeError):
    def __init__(self, code: int, where: str, msg: str):
        super().__init__(f"{where}: {STATUS_NAMES.get(code, code)}: {msg}")
        self.code = code


def load(path: str | os.PathLike | None = None):
    """Load libplato_b200.so (once) and declare every C-ABI signature."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise ImportError(f"{p} is missing: build it with `python -m plato_b200.build` "
                          "(the engine has no CPU fallback)")
    lib = C.CDLL(str(p))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name, None)
        if fn is None:
            continue
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


def check(code: int, where: str) -> None:
    if code != PLATO_OK:
        raise PlatoError(code, where, load().plato_last_error().decode(errors="replace"))
