"""CPU tests: the oracle against the reference's golden values and against the
independent FP64 oracle; the RMAT generator against its numpy restatement."""
import numpy as np
import pytest

import oracle
from oracle import RefGraph, fp64
from tests import rmat_spec


def _graph(golden, name, directed):
    graphs, _ = golden
    g = graphs[name]
    V = int(max(g["src"].max(), g["dst"].max())) + 1
    return V, g["src"], g["dst"], RefGraph(V, g["src"], g["dst"], directed)


def test_kat_dcsc_counts(golden):
    _, kats = golden
    for k in kats["dcsc_counts"]:
        _, _, _, g = _graph(golden, k["graph"], k["is_directed"])
        assert g.dcsc_columns == k["vertices"], k["source"]
        assert g.stored_edges == k["edges"], k["source"]


def test_kat_degrees(golden):
    _, kats = golden
    for k in kats["degrees"]:
        V, s, d, g = _graph(golden, k["graph"], k["is_directed"])
        if k["kind"] == "out":
            deg = g.out_degrees()
        else:  # in-degree = out-degree of the transposed graph
            deg = RefGraph(V, d, s, k["is_directed"]).out_degrees()
        assert deg.size == 100
        for v, want in k["values"].items():
            assert deg[int(v)] == want, k["source"]


def test_kat_neighbours(golden):
    _, kats = golden
    for k in kats["neighbours"]:
        graphs, _ = golden
        g = graphs[k["graph"]]
        nb = g["dst"][g["src"] == k["vertex"]]
        assert nb.size == k["count"] and np.unique(nb).size == k["count"], k["source"]
        assert nb.min() >= k["lo"] and nb.max() <= k["hi"], k["source"]


def test_kat_aggregate_message(golden):
    _, kats = golden
    for k in kats["aggregate_message"]:
        _, _, _, g = _graph(golden, k["graph"], k["is_directed"])
        total, values = g.aggregate_count()
        assert total == k["sum"], k["source"]
        assert values.tolist() == k["values"], k["source"]


@pytest.mark.parametrize("scale,sym,perm", [(6, False, False), (9, True, False), (10, False, True),
                                            (8, True, True)])
def test_rmat_generator_matches_spec(scale, sym, perm):
    import plato_b200 as pb
    V, s, d = pb.rmat(scale, 16, 7, symmetrize=sym, permute=perm)
    V2, s2, d2 = rmat_spec.rmat(scale, 16, 7, symmetrize=sym, permute=perm)
    assert V == V2
    np.testing.assert_array_equal(s, s2)
    np.testing.assert_array_equal(d, d2)
    assert (s != d).all()
    ids = np.union1d(s, d)
    assert ids.size == V and ids[0] == 0 and ids[-1] == V - 1  # compact


@pytest.mark.parametrize("scale,sym", [(6, False), (11, True), (16, False)])
def test_oracle_rmat_matches_product_and_spec(scale, sym):
    """bench.py's reference arm generates its graph with the oracle's C
    generator (so that its process never loads the product library); the
    lists must equal the product's and the numpy restatement's."""
    import oracle
    import plato_b200 as pb
    V, s, d = oracle.rmat(scale, 16, 3, symmetrize=sym)
    V1, s1, d1 = pb.rmat(scale, 16, 3, symmetrize=sym)
    assert V == V1
    np.testing.assert_array_equal(s, s1)
    np.testing.assert_array_equal(d, d1)
    if scale <= 11:
        V2, s2, d2 = rmat_spec.rmat(scale, 16, 3, symmetrize=sym)
        assert V == V2
        np.testing.assert_array_equal(s, s2)
        np.testing.assert_array_equal(d, d2)


def test_oracle_rank_state_reused_between_calls():
    """The oracle keeps its rank-loop buffers on the graph between calls; a
    second call (and a call of another kind in between) gives the same bits."""
    import oracle
    V, s, d = oracle.rmat(10, 16, 5)
    g = oracle.RefGraph(V, s, d, True)
    try:
        a, ea, _ = g.pagerank(20, 0.85, 0.0)
        src = int(np.flatnonzero(g.out_degrees() > 0)[0])
        g.ppr(src, 30, 0.85, 0.0, True)
        b, eb, _ = g.pagerank(20, 0.85, 0.0)
    finally:
        g.close()
    assert ea == eb == 20
    np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("directed", [True, False])
def test_oracle_pagerank_vs_fp64(directed):
    import plato_b200 as pb
    V, s, d = pb.rmat(11, 16, 1, symmetrize=not directed)
    g = RefGraph(V, s, d, directed)
    for iters, eps in [(1, 0.0), (20, 0.0), (100, 0.001)]:
        r, ep, _ = g.pagerank(iters, 0.85, eps)
        r2, ep2 = fp64.pagerank(V, s, d, directed, iters, 0.85, eps)
        assert ep == ep2
        assert np.abs(r - r2).max() <= 1e-9 * max(1.0, np.abs(r2).max())


@pytest.mark.parametrize("pushpull", [False, True])
def test_oracle_ppr_vs_fp64(pushpull):
    import plato_b200 as pb
    V, s, d = pb.rmat(11, 16, 3)
    g = RefGraph(V, s, d, True)
    deg = g.out_degrees()
    for src in np.flatnonzero(deg > 0)[[0, 7, 50]]:
        r, ep, pe, tr, _ = g.ppr(int(src), 300, 0.85, 1e-7, pushpull)
        r2, ep2 = fp64.ppr(V, s, d, int(src), True, 300, 0.85, 1e-7)
        assert abs(ep - ep2) <= 1
        assert np.abs(r - r2).sum() <= 1e-6
        if pushpull:
            assert pe >= 1 and tr & 1  # starts in push mode from one vertex


def test_oracle_seedset_vs_fp64():
    import plato_b200 as pb
    V, s, d = pb.rmat(10, 16, 4)
    g = RefGraph(V, s, d, True)
    seeds = [0, 3, 3, 17, 40]
    r, ep, _ = g.seedset_ppr(seeds, 60, 0.85, 0.0)
    r2, _ = fp64.seedset_ppr(V, s, d, seeds, True, 60, 0.85, 0.0)
    assert np.abs(r - r2).sum() <= 1e-12


@pytest.mark.parametrize("directed", [True, False])
def test_oracle_bfs_vs_serial(directed):
    import plato_b200 as pb
    V, s, d = pb.rmat(12, 16, 2, symmetrize=not directed)
    g = RefGraph(V, s, d, directed)
    for root in [0, 5, V - 1]:
        lev, par, vis, tr, ep = g.bfs(root)
        lev2 = fp64.bfs_levels(V, s, d, root, directed)
        np.testing.assert_array_equal(lev, lev2)
        assert vis == int((lev2 != 0xFFFFFFFF).sum())
        # parents form a BFS tree
        reached = np.flatnonzero((lev != 0xFFFFFFFF) & (np.arange(V) != root))
        assert (lev[par[reached]] == lev[reached] - 1).all()


def test_oracle_thread_count_reported():
    assert oracle.max_threads() >= 1


def test_cc_oracle_matches_reference_test_labelling(golden):
    """cc_labels (min-propagation fixed point) equals the reference test's
    BFS-from-ascending-ids labelling (test_cgm.cc:81-99) on its fixture."""
    from oracle import fp64
    graphs, _ = golden
    g0 = graphs["v100_e2150_ua_c3.csv"]
    s, d = g0["src"], g0["dst"]
    V = int(max(s.max(), d.max())) + 1
    lab = fp64.cc_labels(V, s, d, False)
    assert (lab == fp64.cc_components_bfs(V, s, d)).all()
    assert (lab <= np.arange(V)).all()


def _switch_epoch(V, s, d, src):
    """Push epochs of dual-mode PPR from `src` when every push epoch walks the
    actives it started with: the actives after k push epochs are the vertices
    within k hops, and the switch comes at the first k whose out-degree sum
    exceeds edges / 20 (personalized_pagerank.hpp:184-205)."""
    deg = np.bincount(s, minlength=V).astype(np.int64)
    order = np.argsort(s, kind="stable")
    off = np.zeros(V + 1, np.int64)
    off[1:] = np.cumsum(deg)
    nbr = d[order]
    act = np.zeros(V, bool)
    act[src] = True
    k = 0
    while int(deg[act].sum()) <= s.size // 20:
        members = np.flatnonzero(act)
        reach = np.concatenate([nbr[off[u]:off[u + 1]] for u in members]) if members.size else []
        act[reach] = True
        k += 1
    return k


def test_oracle_push_epochs_follow_the_epoch_start_actives():
    """A vertex reached in a push epoch is walked from the next epoch on, so
    the switch epoch is a function of the graph alone (the same on every run
    and thread count) and equals the hop-ball recount above."""
    import plato_b200 as pb
    V, s, d = pb.rmat(16, 16, 3)
    g = RefGraph(V, s, d, True)
    deg = g.out_degrees()
    for src in np.flatnonzero(deg > 0)[[3, 100, 2000]]:
        want = _switch_epoch(V, s, d, int(src))
        runs = {g.ppr(int(src), 10, 0.85, 0.0, True)[2] for _ in range(3)}
        assert runs == {min(want, 10)}, (src, runs, want)
