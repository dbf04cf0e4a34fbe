"""GPU parity: CUDA path (through the C ABI) vs the oracle on the same inputs.

Tolerances (written here, per the rank contract): PageRank / PPR in FP32 with
FP32 accumulation must be within L1 <= 1e-6 of the FP64 oracle per vector,
in normalised units (reference PageRank / V); BFS levels bit-exact.
"""
import numpy as np
import pytest

import plato_b200 as pb
from oracle import RefGraph, fp64

pytestmark = pytest.mark.gpu

L1_TOL = 1e-6


def _l1(a, b):
    return float(np.abs(np.asarray(a, np.float64) - np.asarray(b, np.float64)).sum())


@pytest.fixture(scope="module")
def rmat16():
    V, s, d = pb.rmat(16, 16, 1)
    return V, s, d, RefGraph(V, s, d, True)


@pytest.fixture(scope="module")
def rmat14_sym():
    V, s, d = pb.rmat(14, 16, 2, symmetrize=True)
    return V, s, d, RefGraph(V, s, d, False)


def _fixture(golden, name, directed):
    graphs, _ = golden
    g = graphs[name]
    V = int(max(g["src"].max(), g["dst"].max())) + 1
    return V, g["src"], g["dst"]


@pytest.mark.parametrize("relabel", [True, False])
def test_degrees_kat_on_gpu(golden, relabel):
    _, kats = golden
    for k in kats["degrees"]:
        if k["kind"] != "out":
            continue
        V, s, d = _fixture(golden, k["graph"], k["is_directed"])
        with pb.Graph(V, s, d, k["is_directed"], relabel=relabel) as g:
            deg = g.out_degrees()
        for v, want in k["values"].items():
            assert deg[int(v)] == want, k["source"]


@pytest.mark.parametrize("relabel", [True, False])
def test_pagerank_config_s16_100_iterations(rmat16, relabel):
    """RMAT scale 16, ef 16, seed 1, d=0.85, 100 iterations, pull."""
    V, s, d, ref = rmat16
    want, ep, _ = ref.pagerank(100, 0.85, 0.0)
    with pb.Graph(V, s, d, True, relabel=relabel) as g:
        got, st = g.pagerank(100, 0.85, 0.0)
    assert st.iterations == ep == 100
    l1 = _l1(got, want / V)
    assert l1 <= L1_TOL, l1
    r64, _ = fp64.pagerank(V, s, d, True, 100, 0.85, 0.0)
    assert _l1(got, r64 / V) <= L1_TOL


@pytest.mark.parametrize("name,directed", [("graph_10_9.csv", True), ("v100_e2150_ua_c3.csv", False),
                                           ("v100_e4300_da_c3.csv", True)])
def test_pagerank_fixtures(golden, name, directed):
    V, s, d = _fixture(golden, name, directed)
    ref = RefGraph(V, s, d, directed)
    for iters, eps in [(1, 0.0), (2, 0.0), (30, 0.0), (100, 0.001)]:
        want, ep, _ = ref.pagerank(iters, 0.85, eps)
        with pb.Graph(V, s, d, directed) as g:
            got, st = g.pagerank(iters, 0.85, eps)
        assert st.iterations == ep
        assert _l1(got, want / V) <= L1_TOL


def test_pagerank_reference_units_and_early_exit(rmat16):
    V, s, d, ref = rmat16
    want, ep, _ = ref.pagerank(100, 0.85, 0.01)
    with pb.Graph(V, s, d, True) as g:
        got = pb.pagerank(g, pb.pagerank_opts_t(100, 0.85, 0.01))
        _, st = g.pagerank(100, 0.85, 0.01)
    assert st.iterations == ep
    assert _l1(got / V, want / V) <= L1_TOL


def test_pagerank_deterministic(rmat16):
    V, s, d, _ = rmat16
    with pb.Graph(V, s, d, True) as g:
        a, _ = g.pagerank(20)
        b, _ = g.pagerank(20)
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


@pytest.mark.parametrize("pushpull", [False, True])
def test_ppr_single_source(rmat16, pushpull):
    V, s, d, ref = rmat16
    deg = ref.out_degrees()
    cands = np.flatnonzero(deg > 0)
    rng = np.random.default_rng(3)
    mode = pb.PLATO_PPR_PUSHPULL if pushpull else pb.PLATO_PPR_PULL
    with pb.Graph(V, s, d, True) as g:
        for src in rng.choice(cands, 4, replace=False):
            want, ep, pe, tr, _ = ref.ppr(int(src), 400, 0.85, 1e-7, pushpull)
            got, st = g.personalized_pagerank(int(src), 400, 0.85, 1e-7, mode)
            assert abs(st.iterations - ep) <= 1
            assert _l1(got, want) <= L1_TOL
            if pushpull:  # the switch depends on the graph only: same epoch
                assert st.push_iterations == pe >= 1
                n = min(st.iterations, ep, 64)
                assert [m == "push" for m in st.mode_trace[:n]] == [bool((tr >> i) & 1) for i in range(n)]


def test_ppr_fixed_epochs_trace_matches(rmat16):
    V, s, d, ref = rmat16
    src = int(np.flatnonzero(ref.out_degrees() > 0)[10])
    want, ep, pe, tr, _ = ref.ppr(src, 30, 0.85, 0.0, True)
    with pb.Graph(V, s, d, True) as g:
        got, st = g.personalized_pagerank(src, 30, 0.85, 0.0, pb.PLATO_PPR_PUSHPULL)
    assert st.iterations == ep == 30
    assert st.push_iterations == pe
    assert _l1(got, want) <= L1_TOL


@pytest.mark.parametrize("graph", ["sym", "dir"])
def test_bfs_levels_bit_exact(rmat14_sym, rmat16, graph):
    V, s, d, ref = rmat14_sym if graph == "sym" else rmat16
    directed = graph == "dir"
    deg = ref.out_degrees()
    roots = np.random.default_rng(2).choice(np.flatnonzero(deg > 0), 6, replace=False)
    with pb.Graph(V, s, d, directed) as g:
        for root in roots:
            lev_ref, _, vis_ref, tr_ref, ep_ref = ref.bfs(int(root))
            lev, par, st = g.bfs(int(root))
            np.testing.assert_array_equal(lev, lev_ref)
            assert st.visited == vis_ref
            assert st.iterations == ep_ref
            trace = [(tr_ref >> i) & 1 for i in range(min(ep_ref, 64))]
            assert [m == "push" for m in st.mode_trace] == [bool(t) for t in trace]
            reached = np.flatnonzero((lev != pb.PLATO_LEVEL_UNREACHED) & (np.arange(V) != root))
            assert par[root] == root
            assert (lev[par[reached]] == lev[reached] - 1).all()
            # every parent link is an edge of the graph
            key = (par[reached].astype(np.uint64) << np.uint64(32)) | reached.astype(np.uint64)
            ek = (s.astype(np.uint64) << np.uint64(32)) | d.astype(np.uint64)
            if not directed:
                ek = np.concatenate([ek, (d.astype(np.uint64) << np.uint64(32)) | s.astype(np.uint64)])
            assert np.isin(key, ek).all()
            unreached = lev == pb.PLATO_LEVEL_UNREACHED
            assert (par[unreached] == V).all()  # invalid parent = max_v_i + 1


def test_bfs_push_only_and_pull_only(rmat14_sym):
    V, s, d, ref = rmat14_sym
    lev_ref = fp64.bfs_levels(V, s, d, 0, False)
    with pb.Graph(V, s, d, False) as g:
        for thr in (0.0, 1.01):  # always pull / always push
            lev, _, st = g.bfs(0, push_threshold=thr)
            np.testing.assert_array_equal(lev, lev_ref)
            assert st.push_iterations == (st.iterations if thr > 1 else 0)


@pytest.mark.parametrize("relabel", [True, False])
def test_bfs_pull_parent_is_first_frontier_in_neighbour(rmat14_sym, relabel):
    """Pull levels take the first in-neighbour in CSC order that is in the
    frontier (bfs.hpp:119-136).  Without relabelling CSC order is ascending
    caller id, so the parent is the smallest in-neighbour one level up; with
    relabelling the warp, 8-lane and thread rows must still give exact levels
    and valid parents."""
    V, s, d, _ = rmat14_sym
    deg = np.bincount(s, minlength=V) + np.bincount(d, minlength=V)
    roots = np.random.default_rng(5).choice(np.flatnonzero(deg > 0), 3, replace=False)
    u = np.concatenate([s, d]).astype(np.int64)
    v = np.concatenate([d, s]).astype(np.int64)
    with pb.Graph(V, s, d, False, relabel=relabel) as g:
        for root in roots:
            lev_ref = fp64.bfs_levels(V, s, d, int(root), False)
            lev, par, st = g.bfs(int(root), push_threshold=0.0)
            np.testing.assert_array_equal(lev, lev_ref)
            assert st.push_iterations == 0
            reached = np.flatnonzero((lev != pb.PLATO_LEVEL_UNREACHED) & (np.arange(V) != root))
            lv = lev.astype(np.int64)
            ok = (lev[u] != pb.PLATO_LEVEL_UNREACHED) & (lv[u] == lv[v] - 1)
            first = np.full(V, V, np.int64)
            np.minimum.at(first, v[ok], u[ok])
            if relabel:
                assert (lev[par[reached]] == lev[reached] - 1).all()
                key = par[reached].astype(np.int64) * V + reached
                assert np.isin(key, u * V + v).all()
            else:
                np.testing.assert_array_equal(par[reached], first[reached])


def test_bfs_isolated_root_and_edge_cases():
    # vertex 3 has no edges; graph of 5 vertices with a small chain
    s = np.array([0, 1], np.uint32)
    d = np.array([1, 2], np.uint32)
    with pb.Graph(5, s, d, True) as g:
        lev, par, st = g.bfs(3)
        assert st.visited == 1 and lev[3] == 0
        assert (lev[[0, 1, 2, 4]] == pb.PLATO_LEVEL_UNREACHED).all()
        lev, par, st = g.bfs(0)
        assert lev[:3].tolist() == [0, 1, 2] and st.visited == 3
        r, st = g.pagerank(5)
    ref = RefGraph(5, s, d, True)
    want, _, _ = ref.pagerank(5, 0.85, 0.0)
    assert _l1(r, want / 5) <= L1_TOL


def test_bad_ids_rejected():
    with pytest.raises(pb.PlatoError) as e:
        pb.Graph(4, np.array([0, 5], np.uint32), np.array([1, 2], np.uint32))
    assert e.value.code == 1
    with pb.Graph(3, np.array([0], np.uint32), np.array([1], np.uint32)) as g:
        with pytest.raises(pb.PlatoError):
            g.bfs(7)
        with pytest.raises(pb.PlatoError):
            g.personalized_pagerank(9)


def test_kernels_launched_by_native_library(rmat16):
    V, s, d, _ = rmat16
    before = pb.kernel_launches()
    with pb.Graph(V, s, d, True) as g:
        g.pagerank(3)
    assert pb.kernel_launches() - before >= 3 * 2
