"""GPU parity at the benchmark workloads' full sizes, against the oracle's
C/OpenMP restatement (oracle/ref_cpu.c) on the same inputs:

* BFS, RMAT scale 22 ef 16 seed 2 symmetrised (the 64-root traversal
  workload): levels bit-exact, visited count, epoch count and push/pull trace
  equal, for all 64 of the same roots; parents one level up along real edges
  (checked against the sorted edge set for the first 3 roots).
* PageRank, RMAT scale 24 ef 16 seed 3, 20 pull epochs: L1 <= 1e-6 against
  the reference's ranks / V.
* Single-source PPR on the same graph to delta < 1e-7, pull and push-pull:
  L1 <= 1e-6, epoch counts within one, push epochs and mode trace equal.
* Batched PPR, RMAT scale 22 ef 16 seed 4, a batch of 64 Zipf(1.5) seed sets
  of 1..32 vertices: 4 of its columns against the oracle's seed-set PPR,
  L1 <= 1e-6 and epochs within one; every column sums to its expected mass.
* Connected components on the BFS graph: labels equal the oracle's fixed
  point (the smallest id of each component).

Each graph takes 3-15 s to build in the oracle on 16 host cores; the whole
file runs in about a minute on one B200 host.
"""
import numpy as np
import pytest

import plato_b200 as pb
from oracle import RefGraph

pytestmark = pytest.mark.gpu

L1_TOL = 1e-6


def _l1(a, b):
    return float(np.abs(np.asarray(a, np.float64) - np.asarray(b, np.float64)).sum())


@pytest.fixture(scope="module")
def bfs_graph():
    V, s, d = pb.rmat(22, 16, 2, symmetrize=True)
    ref = RefGraph(V, s, d, False)
    g = pb.Graph(V, s, d, is_directed=False)
    yield V, s, d, ref, g
    g.close()
    ref.close()


@pytest.fixture(scope="module")
def pr_graph():
    V, s, d = pb.rmat(24, 16, 3)
    ref = RefGraph(V, s, d, True)
    g = pb.Graph(V, s, d, is_directed=True)
    yield V, s, d, ref, g
    g.close()
    ref.close()


def test_bfs_s22_levels_bit_exact(bfs_graph):
    V, s, d, ref, g = bfs_graph
    deg = np.bincount(s, minlength=V) + np.bincount(d, minlength=V)
    roots = np.random.default_rng(2).choice(np.flatnonzero(deg > 0), 64, replace=False)
    ek = np.sort(np.concatenate([(s.astype(np.uint64) << np.uint64(32)) | d.astype(np.uint64),
                                 (d.astype(np.uint64) << np.uint64(32)) | s.astype(np.uint64)]))
    for i, root in enumerate(roots):
        lev_ref, _, vis_ref, tr_ref, ep_ref = ref.bfs(int(root), 0.05)
        lev, par, st = g.bfs(int(root))
        np.testing.assert_array_equal(lev, lev_ref)
        assert st.visited == vis_ref
        assert st.iterations == ep_ref
        trace = [bool((tr_ref >> k) & 1) for k in range(min(ep_ref, 64))]
        assert [m == "push" for m in st.mode_trace] == trace
        reached = np.flatnonzero((lev != pb.PLATO_LEVEL_UNREACHED) & (np.arange(V) != root))
        assert par[root] == root
        assert (lev[par[reached]] == lev[reached] - 1).all()
        if i >= 3:
            continue
        key = (par[reached].astype(np.uint64) << np.uint64(32)) | reached.astype(np.uint64)
        pos = np.minimum(np.searchsorted(ek, key), ek.size - 1)
        assert (ek[pos] == key).all()  # every parent link is an edge


def min_id_labels(V, s, d):
    """Smallest id of each vertex's component: the fixed point of the
    oracle's label propagation (oracle/fp64.py cc_labels) on an undirected
    graph, computed by scipy's component search to stay fast at full size."""
    import scipy.sparse as sp
    from scipy.sparse.csgraph import connected_components
    A = sp.csr_matrix((np.ones(s.size, np.int8), (s, d)), shape=(V, V))
    _, comp = connected_components(A, directed=False)
    first = np.full(comp.max() + 1, V, np.int64)
    np.minimum.at(first, comp, np.arange(V))
    return first[comp].astype(np.uint32)


def test_connected_components_s22(bfs_graph):
    V, s, d, _, g = bfs_graph
    lab, _, _ = g.connected_components()
    np.testing.assert_array_equal(lab, min_id_labels(V, s, d))


def test_pagerank_s24_20_epochs(pr_graph):
    V, s, d, ref, g = pr_graph
    want, ep, _ = ref.pagerank(20, 0.85, 0.0)
    got, st = g.pagerank(20, 0.85, 0.0)
    assert st.iterations == ep == 20
    l1 = _l1(got, want / V)
    assert l1 <= L1_TOL, l1


@pytest.mark.parametrize("pushpull", [False, True])
def test_ppr_s24_to_1e7(pr_graph, pushpull):
    V, s, d, ref, g = pr_graph
    deg = np.bincount(s, minlength=V)
    src = int(np.random.default_rng(3).choice(np.flatnonzero(deg > 0)))
    mode = pb.PLATO_PPR_PUSHPULL if pushpull else pb.PLATO_PPR_PULL
    want, ep, pe, tr, _ = ref.ppr(src, 500, 0.85, 1e-7, pushpull)
    got, st = g.personalized_pagerank(src, 500, 0.85, 1e-7, mode)
    assert abs(st.iterations - ep) <= 1
    l1 = _l1(got, want)
    assert l1 <= L1_TOL, l1
    if pushpull:
        assert st.push_iterations == pe >= 1
        n = min(st.iterations, ep, 64)
        assert [m == "push" for m in st.mode_trace[:n]] == [bool((tr >> i) & 1) for i in range(n)]


def test_batched_ppr_s22_k64():
    V, s, d = pb.rmat(22, 16, 4)
    deg = np.bincount(s, minlength=V)
    rng = np.random.default_rng(4)
    cands = np.flatnonzero(deg > 0)
    sizes = np.minimum(rng.zipf(1.5, 64), 32)
    sets = [rng.choice(cands, int(n), replace=False).astype(np.uint32) for n in sizes]
    with pb.Graph(V, s, d, True) as g:
        out = g.ppr_batch(sets, max_iterations=300, eps=1e-6, ranks=True)
    ranks = out["ranks"]
    # a column's mass: every vertex with out-edges passes d of its rank on,
    # so the ranks sum to at most 1 and lose only the dangling share
    sums = ranks.astype(np.float64).sum(axis=1)
    assert (sums <= 1.0 + 1e-5).all() and (sums > 0.1).all()
    ref = RefGraph(V, s, d, True)
    try:
        for q in (0, 1, int(np.argmax(sizes)), 63):
            want, ep, _ = ref.seedset_ppr(sets[q], 300, 0.85, 1e-6)
            assert abs(int(out["iterations"][q]) - ep) <= 1
            l1 = _l1(ranks[q], want)
            assert l1 <= L1_TOL, (q, l1)
    finally:
        ref.close()
