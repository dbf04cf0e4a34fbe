"""plato_diag_pull_ceiling: the gather-stream diagnostic runs every mode on
a small graph, its checksum equals the number of gathers it made times the
rank it gathered (every rank is 1/V), and it refuses bad modes and graphs
kept in caller order."""
import ctypes as C

import numpy as np
import pytest

import plato_b200 as pb
from plato_b200 import _lib

pytestmark = pytest.mark.gpu


def test_ceiling_modes_run_and_count_their_gathers():
    lib = _lib.load()
    V, s, d = pb.rmat(14, 16, 9)
    with pb.Graph(V, s, d, True) as g:
        indeg = np.bincount(d, minlength=V)
        long_edges = int(indeg[indeg > 64].sum())
        for mode in range(6):
            ms, n, cs = C.c_double(), C.c_uint64(), C.c_double()
            _lib.check(lib.plato_diag_pull_ceiling(g.handle, mode, 4, C.byref(ms), C.byref(n), C.byref(cs)),
                       "plato_diag_pull_ceiling")
            assert n.value == long_edges and ms.value > 0
            if mode >= 1:  # (3 warm-ups + 4 timed) launches x gathers x 1/V
                assert cs.value == pytest.approx(7 * long_edges / V, rel=1e-3)
        ms, n, cs = C.c_double(), C.c_uint64(), C.c_double()
        assert lib.plato_diag_pull_ceiling(g.handle, 6, 4, C.byref(ms), None, None) == _lib.PLATO_EINVAL
    with pb.Graph(V, s, d, True, relabel=False) as g:
        assert lib.plato_diag_pull_ceiling(g.handle, 1, 4, C.byref(ms), None, None) == _lib.PLATO_EINVAL


@pytest.mark.parametrize("kt", [16, 128])
def test_batch_ceiling_modes_run_and_count_their_gathers(kt):
    """plato_diag_batch_ceiling: every row of its state sums to 1, so the
    checksum of modes 0-2 is (3 warm-ups + 4 timed) x the stored edges; mode 3
    runs the real batched iteration and reports its live columns."""
    lib = _lib.load()
    V, s, d = pb.rmat(14, 16, 9)
    for relabel in (True, False):
        with pb.Graph(V, s, d, True, relabel=relabel) as g:
            E = g.device_view().stored_edges
            for mode in range(4):
                ms, n, cs = C.c_double(), C.c_uint64(), C.c_double()
                _lib.check(lib.plato_diag_batch_ceiling(g.handle, kt, mode, 4, C.byref(ms), C.byref(n),
                                                        C.byref(cs)), "plato_diag_batch_ceiling")
                assert n.value == E and ms.value > 0
                if mode < 3:
                    assert cs.value == pytest.approx(7 * E, rel=1e-4)
                else:
                    assert cs.value == kt
            ms = C.c_double()
            assert lib.plato_diag_batch_ceiling(g.handle, kt, 4, 4, C.byref(ms), None, None) == _lib.PLATO_EINVAL
            assert lib.plato_diag_batch_ceiling(g.handle, 8, 0, 4, C.byref(ms), None, None) == _lib.PLATO_EINVAL
