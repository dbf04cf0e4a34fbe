"""TrustRank (plato_trustrank): good-seed selection by (inverse) PageRank
and the seed-set PPR that follows, against the oracle
(oracle.trustrank_seeds + RefGraph.seedset_ppr, restating
plato/algo/trustrank/trustrank.hpp:88-259)."""
import numpy as np
import pytest

import plato_b200 as pb
from oracle import RefGraph, trustrank_seeds

pytestmark = pytest.mark.gpu

L1_TOL = 1e-6


@pytest.fixture(scope="module")
def g14():
    V, s, d = pb.rmat(14, 16, 8)
    g = pb.Graph(V, s, d, True)
    yield V, s, d, g
    g.close()


def _seed_num_with_gap(ranks, near=100):
    """A seed count near `near` whose cut falls between clearly different
    ranks, so FP64 rounding differences cannot reorder the boundary."""
    r = np.sort(ranks)[::-1]
    for k in list(range(near, near + 50)) + list(range(near - 1, near - 50, -1)):
        if r[k - 1] - r[k] > 1e-9 * r[k - 1]:
            return k
    raise AssertionError("no clear cut near %d" % near)


@pytest.mark.parametrize("method", [0, 1])
def test_trustrank_matches_oracle(g14, method):
    V, s, d, g = g14
    _, ranks = trustrank_seeds(V, s, d, True, 100, method)
    k = _seed_num_with_gap(ranks)
    want_seeds, _ = trustrank_seeds(V, s, d, True, k, method)
    good = np.ones(V, bool)
    good[::3] = False  # a third of the vertices are not good
    want_good, _ = trustrank_seeds(V, s, d, True, k, method, good)
    for gv, want in ((None, want_seeds), (good, want_good)):
        r, seeds, st = g.trustrank(good=gv, seed_num=k, select_method=method, iteration=100,
                                   eps=1e-6)
        np.testing.assert_array_equal(seeds, want)
        ref = RefGraph(V, s, d, True)
        want_r, ep, _ = ref.seedset_ppr(want, 100, 0.85, 1e-6)
        ref.close()
        assert float(np.abs(r.astype(np.float64) - want_r).sum()) <= L1_TOL
        assert abs(st.iterations - ep) <= 1


def test_trustrank_small_graph_takes_all_good_vertices():
    s = np.array([0, 1, 2, 3], np.uint32)
    d = np.array([1, 2, 3, 0], np.uint32)
    with pb.Graph(5, s, d, True) as g:
        r, seeds, _ = g.trustrank(good=np.array([1, 0, 1, 1, 0], bool), seed_num=100)
        assert seeds.tolist() == [0, 2, 3]
        ref = RefGraph(5, s, d, True)
        want, _, _ = ref.seedset_ppr(np.array([0, 2, 3], np.uint32), 100, 0.85, 0.001)
        ref.close()
        assert float(np.abs(r.astype(np.float64) - want).sum()) <= L1_TOL


def test_trustrank_random_selection_is_seeded(g14):
    V, s, d, g = g14
    good = np.zeros(V, bool)
    good[::2] = True
    r1, s1, _ = g.trustrank(good=good, seed_num=64, select_method=2, random_seed=7)
    r2, s2, _ = g.trustrank(good=good, seed_num=64, select_method=2, random_seed=7)
    np.testing.assert_array_equal(s1, s2)
    np.testing.assert_array_equal(r1, r2)
    assert 0 < s1.size <= 64 and good[s1].all()
    _, s3, _ = g.trustrank(good=good, seed_num=64, select_method=2, random_seed=8)
    assert not np.array_equal(s1, s3)


def test_trustrank_errors(g14):
    V, s, d, g = g14
    with pytest.raises(pb.PlatoError):
        g.trustrank(good=np.zeros(V, bool), seed_num=10, select_method=1)  # no good seed
    with pytest.raises(pb.PlatoError):
        g.trustrank(select_method=3)
    with pytest.raises(pb.PlatoError):
        g.trustrank(seed_num=0)
