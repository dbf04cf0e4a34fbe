"""GPU tests of the header-only dualmode engine (include/plato_b200/dualmode.cuh)
driven by the reference's own functor bodies (tests/engine/engine_kat.cu)."""
import ctypes as C

import numpy as np
import pytest

import plato_b200 as pb
from oracle import RefGraph

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def kat():
    from tests.engine.build import build
    lib = C.CDLL(str(build()))
    P = C.c_void_p
    lib.kat_error.restype = C.c_char_p
    lib.kat_aggregate.argtypes = [P, C.c_int, P, P]
    lib.kat_pagerank.argtypes = [P, C.c_uint32, C.c_double, C.c_int, C.c_int, P]
    lib.kat_bfs.argtypes = [P, C.c_uint32, P, P, P]
    return lib


def _p(a):
    return C.c_void_p(a.ctypes.data)


@pytest.mark.parametrize("relabel", [True, False])
@pytest.mark.parametrize("combined", [0, 1])
def test_aggregate_message_kat(kat, golden, relabel, combined):
    graphs, kats = golden
    k = kats["aggregate_message"][0]
    g = graphs[k["graph"]]
    with pb.Graph(10, g["src"], g["dst"], True, relabel=relabel) as gr:
        vals = np.zeros(10, np.int32)
        total = C.c_int64()
        assert kat.kat_aggregate(gr.handle, combined, _p(vals), C.byref(total)) == 0, kat.kat_error()
    assert total.value == k["sum"], k["source"]
    assert vals.tolist() == k["values"], k["source"]


@pytest.mark.parametrize("directed", [True, False])
@pytest.mark.parametrize("combined", [0, 1])
@pytest.mark.parametrize("reversed_", [0, 1])
def test_reference_pagerank_functors(kat, directed, combined, reversed_):
    V, s, d = pb.rmat(12, 16, 11, symmetrize=not directed)
    # the transpose's PageRank is the PageRank of the reversed edge list
    ref = RefGraph(V, d, s, directed) if reversed_ else RefGraph(V, s, d, directed)
    want, _, _ = ref.pagerank(15, 0.85, 0.0)
    out = np.empty(V, np.float64)
    with pb.Graph(V, s, d, directed) as g:
        assert kat.kat_pagerank(g.handle, 15, 0.85, combined, reversed_, _p(out)) == 0, kat.kat_error()
    assert np.abs(out - want).max() <= 1e-9 * np.abs(want).max()


def test_combined_pull_at_scale_matches_the_64_edge_pull(kat):
    """The combined pull on a graph with hub columns spread over many warps
    and long runs of short columns: PageRank equal to the 64-edge path's to
    FP64 round-off, in both directions."""
    V, s, d = pb.rmat(16, 16, 13)
    with pb.Graph(V, s, d, True) as g:
        for rev in (0, 1):
            a = np.empty(V, np.float64)
            b = np.empty(V, np.float64)
            assert kat.kat_pagerank(g.handle, 10, 0.85, 0, rev, _p(a)) == 0, kat.kat_error()
            assert kat.kat_pagerank(g.handle, 10, 0.85, 1, rev, _p(b)) == 0, kat.kat_error()
            assert np.abs(a - b).max() <= 1e-12 * np.abs(a).max()


@pytest.mark.parametrize("directed", [True, False])
def test_reference_bfs_functors(kat, directed):
    V, s, d = pb.rmat(13, 16, 12, symmetrize=not directed)
    ref = RefGraph(V, s, d, directed)
    deg = ref.out_degrees()
    with pb.Graph(V, s, d, directed) as g:
        for root in np.flatnonzero(deg > 0)[[0, 40, 400]]:
            lev_ref, _, vis_ref, tr_ref, _ = ref.bfs(int(root))
            lev = np.empty(V, np.uint32)
            vis = C.c_uint64()
            tr = C.c_uint64()
            assert kat.kat_bfs(g.handle, int(root), _p(lev), C.byref(vis), C.byref(tr)) == 0, \
                kat.kat_error()
            np.testing.assert_array_equal(lev, lev_ref)
            assert vis.value == vis_ref
            assert tr.value == tr_ref
