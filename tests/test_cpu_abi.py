"""CPU tests of the C ABI: the library loads, exports every declared symbol,
and rejects bad arguments without touching a GPU."""
import ctypes as C
import re
from pathlib import Path

import pytest

from plato_b200 import _lib

ROOT = Path(__file__).resolve().parent.parent


def declared_symbols():
    text = "\n".join(p.read_text() for p in (ROOT / "include").glob("*.h"))
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(plato_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    for need in ["plato_graph_create", "plato_pagerank", "plato_personalized_pagerank", "plato_bfs",
                 "plato_ppr_batch", "plato_server_create", "plato_last_error"]:
        assert need in syms


def test_library_exports_every_declared_symbol():
    lib = C.CDLL(str(_lib.LIB_PATH))
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, f"not exported: {missing}"


def test_binding_covers_header():
    assert set(declared_symbols()) <= set(_lib.SIGNATURES)


def test_null_arguments_rejected():
    lib = _lib.load()
    h = C.c_void_p()
    assert lib.plato_graph_create(None, None, None, 0, C.byref(h)) == _lib.PLATO_EINVAL
    assert b"null" in lib.plato_last_error()
    assert lib.plato_pagerank(None, None, None, None) == _lib.PLATO_EINVAL
    assert lib.plato_bfs(None, None, None, None, None, None) == _lib.PLATO_EINVAL
    info = _lib.GraphInfo(1, 0, 0, 0)
    assert lib.plato_graph_create(C.byref(info), None, None, 0, C.byref(h)) == _lib.PLATO_EINVAL


def test_rmat_bad_params():
    lib = _lib.load()
    p = _lib.RmatParams(0, 16, 1, 0.57, 0.19, 0.19, 0, 0)
    h = C.c_void_p()
    assert lib.plato_rmat_generate(C.byref(p), C.byref(h)) == _lib.PLATO_EINVAL
    p = _lib.RmatParams(8, 16, 1, 0.9, 0.19, 0.19, 0, 0)
    assert lib.plato_rmat_generate(C.byref(p), C.byref(h)) == _lib.PLATO_EINVAL


def test_version():
    assert b"sm_100a" in _lib.load().plato_version()


def test_missing_library_fails_loudly(tmp_path):
    with pytest.raises(ImportError):
        _lib.load(tmp_path / "nope.so")


def test_graph_flags_checked_before_any_device_work():
    lib = _lib.load()
    info = _lib.GraphInfo(1, 3, 0, 2)
    h = C.c_void_p()
    both = _lib.PLATO_GRAPH_RELABEL | _lib.PLATO_GRAPH_NO_RELABEL
    assert lib.plato_graph_create(C.byref(info), None, None, both, C.byref(h)) == _lib.PLATO_EINVAL
    assert lib.plato_graph_create(C.byref(info), None, None, 0x80, C.byref(h)) == _lib.PLATO_EINVAL


def test_noalloc_rejects_unaligned_buffers_before_any_device_work():
    """The alignment rules of plato_pagerank_csc_noalloc are checked on the
    host before any CUDA call, so a bad pointer gives PLATO_EINVAL (not a
    device fault) even here, with no GPU and pointers that are never touched."""
    lib = _lib.load()
    o = _lib.PagerankOpts(5, 0.85, 0.0)
    good = 1 << 20
    for ranks, off, adj, deg in ((good + 4, good, good, good), (good, good + 4, good, good),
                                 (good, good, good + 2, good), (good, good, good, good + 1)):
        rc = lib.plato_pagerank_csc_noalloc(3, 2, C.c_void_p(off), C.c_void_p(adj), C.c_void_p(deg),
                                            C.byref(o), C.c_void_p(ranks), None, None)
        assert rc == _lib.PLATO_EINVAL
        assert b"aligned" in lib.plato_last_error()
