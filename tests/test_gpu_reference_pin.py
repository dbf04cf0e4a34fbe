"""The CUDA path against the reference's own outputs.

tests/golden/ref_golden.npz holds what the reference's algo::pagerank,
personalized_pagerank, breadth_first_search and trustrank computed on
fixture graphs (its engine path compiled from its own headers, see
tests/golden/make_golden.py).  The GPU results must match them through the C
ABI: PageRank / PPR / TrustRank within L1 <= 1e-6 per vector in normalised
units (FP32 accumulation against the reference's FP64) with the same epoch
counts; BFS with the same visited count, the same number of vertices at
every level and the same push/pull choice per level.
"""
from pathlib import Path

import numpy as np
import pytest

import plato_b200 as pb
from tests.test_cpu_reference_pin import NAMES, graph_edges

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parent.parent
L1_TOL = 1e-6


@pytest.fixture(scope="module")
def gold():
    return np.load(ROOT / "tests" / "golden" / "ref_golden.npz")


def l1(a, b):
    return float(np.abs(np.asarray(a, np.float64) - np.asarray(b, np.float64)).sum())


@pytest.mark.parametrize("name", NAMES)
def test_gpu_matches_reference_outputs(gold, name):
    V, _, _, directed = (int(x) for x in gold[f"{name}__meta"])
    s, d = graph_edges(name)
    with pb.Graph(V, s, d, bool(directed)) as g:
        r, st = g.pagerank(100, 0.85, 0.0)
        assert st.iterations == 100
        assert l1(r, gold[f"{name}__pr100"] / V) <= L1_TOL
        r, st = g.pagerank(100, 0.85, 0.001)
        assert st.iterations == int(gold[f"{name}__preps_epochs"])
        assert l1(r, gold[f"{name}__preps"] / V) <= L1_TOL
        src = int(gold[f"{name}__ppr_src"])
        for mode, m in (("pull", pb.PLATO_PPR_PULL), ("pp", pb.PLATO_PPR_PUSHPULL)):
            r, st = g.personalized_pagerank(src, 200, 0.85, 1e-7, m)
            assert abs(st.iterations - int(gold[f"{name}__ppr_{mode}_epochs"])) <= 1, mode
            assert l1(r, gold[f"{name}__ppr_{mode}"]) <= L1_TOL, mode
        for i, root in enumerate(gold[f"{name}__bfs_roots"]):
            lev, _, st = g.bfs(int(root))
            acts = gold[f"{name}__bfs_actives"][i]
            ep = int(np.count_nonzero(acts)) + 1
            assert st.visited == int(gold[f"{name}__bfs_visited"][i])
            assert st.iterations == ep
            reached = lev[lev != pb.PLATO_LEVEL_UNREACHED]
            hist = np.bincount(reached, minlength=ep + 1)[1:ep + 1]
            np.testing.assert_array_equal(hist, acts[:ep])
            trace = int(gold[f"{name}__bfs_trace"][i])
            assert [m == "push" for m in st.mode_trace] == [bool((trace >> k) & 1) for k in range(ep)]
        good = gold[f"{name}__good"].astype(bool)
        r, st = g.seedset_ppr(np.flatnonzero(good).astype(np.uint32), 100, 0.85, 1e-6)
        assert abs(st.iterations - int(gold[f"{name}__tr_all_epochs"])) <= 1
        assert l1(r, gold[f"{name}__tr_all"]) <= L1_TOL
        for m in (0, 1):
            r, _, st = g.trustrank(good, 100, 0.85, 20, m, 0.001)
            assert abs(st.iterations - int(gold[f"{name}__tr_m{m}_epochs"])) <= 1, m
            assert l1(r, gold[f"{name}__tr_m{m}"]) <= L1_TOL, m


@pytest.mark.parametrize("name", ["v100u", "rmat12u"])
def test_gpu_cc_and_hyperanf_match_reference(gold, name):
    V = int(gold[f"{name}__meta"][0])
    s, d = graph_edges(name)
    with pb.Graph(V, s, d, False) as g:
        lab, summ, _ = g.connected_components()
        np.testing.assert_array_equal(lab, gold[f"{name}__cc_labels"])
        comps, major, mv, me = (int(x) for x in gold[f"{name}__cc_summary"])
        assert summ["components"] == comps and summ["major_label"] == major
        assert summ["major_vertices"] == mv and summ["major_edges"] == me
        for bits, want in zip((6, 8), gold[f"{name}__anf_avg"]):
            avg, _, _, _ = g.hyperanf(20, bits)
            assert avg == pytest.approx(float(want), rel=1e-12), bits


@pytest.mark.parametrize("name", ["w10", "wrmat12"])
def test_gpu_weighted_pagerank_matches_reference(gold, name):
    from tests.test_cpu_reference_pin import weighted_edges
    s, d, w = weighted_edges(gold, name)
    V = int(max(s.max(), d.max())) + 1
    with pb.Graph(V, s, d, True, weights=w) as g:
        for tag, eps in (("100", 0.0), ("eps", 0.001)):
            r, st = g.weighted_pagerank(100, 0.85, eps)
            want = gold[f"{name}__wpr{tag}"]
            assert abs(st.iterations - int(gold[f"{name}__wpr{tag}_epochs"])) <= 1, tag
            # the reference's units (ranks sum to ~V): L1 / V within the PageRank tolerance
            assert l1(r, want) / V <= L1_TOL, tag
