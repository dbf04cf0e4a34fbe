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
