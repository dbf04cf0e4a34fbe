"""GPU parity of weighted PageRank (plato/algo/pagerank/weighted_pagerank.hpp)
against the FP64 oracle (oracle/fp64.weighted_pagerank).

Tolerance: the ranks are in the reference's units (about 1 per vertex), so
the bar is L1 / V <= 1e-6 (the per-vector bar of the other rank algorithms
in normalised units); epochs equal for fixed iterations and within one when
an eps threshold is crossed.  The reference ships no test for this algorithm,
so parity is pinned to the restatement only."""
import numpy as np
import pytest

import plato_b200 as pb
from oracle import fp64

pytestmark = pytest.mark.gpu

L1_PER_VERTEX = 1e-6


def _check(V, s, d, w, directed, iters, eps, relabel=True):
    want, ep, _ = fp64.weighted_pagerank(V, s, d, w, directed, iters, 0.85, eps)
    with pb.Graph(V, s, d, directed, relabel=relabel, weights=w) as g:
        got, st = g.weighted_pagerank(iters, 0.85, eps)
    l1 = float(np.abs(got.astype(np.float64) - want).sum())
    assert l1 / V <= L1_PER_VERTEX, l1
    if eps == 0.0:
        assert st.iterations == ep
    else:
        assert abs(st.iterations - ep) <= 1
    return got, st


@pytest.mark.parametrize("directed", [True, False])
def test_reference_weighted_fixture(golden, tmp_path, directed):
    """The reference's weighted fixture graph, loaded through the weighted CSV reader."""
    graphs, _ = golden
    f = graphs["raw_graph_10_9_weighted.csv"]
    lines = [f"{a},{b},{c!r}" for a, b, c in zip(f["src"].tolist(), f["dst"].tolist(), f["w"].tolist())]
    (tmp_path / "w.csv").write_text("\n".join(lines) + "\n")
    V, s, d, w = pb.read_csv(tmp_path / "w.csv", weighted=True)
    np.testing.assert_array_equal(w, f["w"])
    _check(V, s, d, w, directed, 100, 0.001)
    _check(V, s, d, w, directed, 7, 0.0)


@pytest.mark.parametrize("scale,directed", [(12, True), (12, False), (14, True)])
@pytest.mark.parametrize("relabel", [True, False])
def test_rmat_random_weights(scale, directed, relabel):
    V, s, d = pb.rmat(scale, 16, 11)
    w = np.random.default_rng(scale).uniform(0.1, 10.0, s.size)
    _check(V, s, d, w, directed, 20, 0.0, relabel)
    _check(V, s, d, w, directed, 100, 1e-3, relabel)


def test_duplicate_edges_and_sinks():
    # 0->1 twice with different weights, 2 and 4 have no out-edges, 3 is isolated
    s = np.array([0, 0, 1, 1, 0, 0], np.uint32)
    d = np.array([1, 1, 2, 4, 2, 4], np.uint32)
    w = np.array([1.0, 3.0, 2.0, 0.5, 4.0, 1.0])
    _check(5, s, d, w, True, 30, 0.0)
    _check(5, s, d, w, True, 30, 1e-6)


def test_iteration_zero_and_unweighted_graph():
    V, s, d = pb.rmat(8, 8, 2)
    w = np.ones(s.size)
    with pb.Graph(V, s, d, True, weights=w) as g:
        r, st = g.weighted_pagerank(0, 0.85, 0.0)
        assert st.iterations == 0 and np.all(r == 1.0)
    with pb.Graph(V, s, d, True) as g:
        with pytest.raises(pb.PlatoError):
            g.weighted_pagerank(10)


def test_unit_weights_match_plain_pagerank_shape():
    """With every weight 1 the weighted recurrence is the reference's plain
    PageRank in its own units (rank' = 1 - d + d * sum rank[u] / outdeg[u]):
    V times our normalised PageRank."""
    V, s, d = pb.rmat(12, 16, 5)
    w = np.ones(s.size)
    with pb.Graph(V, s, d, True, weights=w) as g:
        wr, _ = g.weighted_pagerank(20, 0.85, 0.0)
        pr, _ = g.pagerank(20, 0.85, 0.0)
    assert float(np.abs(wr.astype(np.float64) / V - pr).sum()) <= 1e-6
