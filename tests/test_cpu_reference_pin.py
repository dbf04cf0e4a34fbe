"""The oracle pinned to the reference's own code.

tests/golden/ref_golden.npz holds what the reference's algo::pagerank,
personalized_pagerank (pull-only and dual-mode), breadth_first_search and
trustrank computed on fixture graphs (its engine path compiled from its own
headers into oracle/_ref/libplato_ref.so, see oracle/refplato.py and
tests/golden/make_golden.py).  The oracle's C restatement must reproduce
them: ranks to FP64 round-off (the two sum the same terms in different
orders), epoch counts exactly, BFS visited counts, vertices per level and the
engine's push/pull choice per level exactly.  Where the compiled reference is
present (it is built wherever the reference tree was at build time), the
same comparison also runs live on a larger RMAT graph.
"""
from pathlib import Path

import numpy as np
import pytest

import oracle
from oracle import refplato

ROOT = Path(__file__).resolve().parent.parent
GOLD = ROOT / "tests" / "golden" / "ref_golden.npz"
FIXTURES = ROOT / "tests" / "golden" / "fixtures.npz"

# ranks are sums of the same terms in another order: FP64 round-off only
RANK_RTOL = 1e-12


def graph_edges(name):
    z = np.load(FIXTURES)
    csv = {"v100u": "v100_e2150_ua_c3", "v100d": "v100_e4300_da_c3"}
    if name in csv:
        return z[csv[name] + "__src"], z[csv[name] + "__dst"]
    scale, seed, sym = {"rmat12d": (12, 1, False), "rmat12u": (12, 2, True), "rmat14d": (14, 3, False)}[name]
    _, s, d = oracle.rmat(scale, 16, seed, symmetrize=sym)
    return s, d


NAMES = ["v100u", "v100d", "rmat12d", "rmat12u", "rmat14d"]


@pytest.fixture(scope="module")
def gold():
    return np.load(GOLD)


def close(a, b, rtol=RANK_RTOL):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.abs(a - b).max()) <= rtol * max(1.0, float(np.abs(b).max()))


def level_histogram(levels, epochs):
    reached = levels[levels != 0xFFFFFFFF]
    return np.bincount(reached, minlength=epochs + 1)[1:epochs + 1].astype(np.uint64)


@pytest.mark.parametrize("name", NAMES)
def test_oracle_matches_reference_outputs(gold, name):
    V, max_v_i, E, directed = (int(x) for x in gold[f"{name}__meta"])
    s, d = graph_edges(name)
    assert V == max_v_i + 1 and E == s.size  # compact ids, same edge list
    g = oracle.RefGraph(V, s, d, bool(directed))
    try:
        r, ep, _ = g.pagerank(100, 0.85, 0.0)
        assert ep == int(gold[f"{name}__pr100_epochs"]) == 100
        assert close(r, gold[f"{name}__pr100"])
        r, ep, _ = g.pagerank(100, 0.85, 0.001)
        assert ep == int(gold[f"{name}__preps_epochs"])
        assert close(r, gold[f"{name}__preps"])
        src = int(gold[f"{name}__ppr_src"])
        for mode, pp in (("pull", False), ("pp", True)):
            r, ep, _, _, _ = g.ppr(src, 200, 0.85, 1e-7, pp)
            assert ep == int(gold[f"{name}__ppr_{mode}_epochs"]), mode
            assert close(r, gold[f"{name}__ppr_{mode}"]), mode
        for i, root in enumerate(gold[f"{name}__bfs_roots"]):
            lev, _, vis, trace, ep = g.bfs(int(root))
            acts = gold[f"{name}__bfs_actives"][i]
            n = int(np.count_nonzero(np.r_[acts, 0] != 0)) + 1  # epochs: the last one activates none
            assert vis == int(gold[f"{name}__bfs_visited"][i])
            assert ep == n
            np.testing.assert_array_equal(level_histogram(lev, ep), acts[:ep])
            assert trace == int(gold[f"{name}__bfs_trace"][i])
        good = gold[f"{name}__good"].astype(bool)
        r, ep, _ = g.seedset_ppr(np.flatnonzero(good).astype(np.uint32), 100, 0.85, 1e-6)
        assert ep == int(gold[f"{name}__tr_all_epochs"])
        assert close(r, gold[f"{name}__tr_all"])
    finally:
        g.close()
    for m in (0, 1):
        seeds, _ = oracle.trustrank_seeds(V, s, d, bool(directed), 20, m, good)
        g = oracle.RefGraph(V, s, d, bool(directed))
        try:
            r, ep, _ = g.seedset_ppr(seeds, 100, 0.85, 0.001)
        finally:
            g.close()
        assert ep == int(gold[f"{name}__tr_m{m}_epochs"]), m
        assert close(r, gold[f"{name}__tr_m{m}"]), m


@pytest.mark.skipif(not refplato.available(), reason="compiled reference not built here")
@pytest.mark.parametrize("directed", [True, False])
def test_oracle_matches_reference_live_rmat16(directed):
    V, s, d = oracle.rmat(16, 16, 5, symmetrize=not directed)
    ref = refplato.ReferenceGraph(V, s, d, directed)
    g = oracle.RefGraph(V, s, d, directed)
    try:
        want, ep_ref, deltas = ref.pagerank(20, 0.85, 0.0)
        got, ep, _ = g.pagerank(20, 0.85, 0.0)
        assert ep == ep_ref == 20 and deltas.size == 20
        assert close(got, want)
        deg = g.out_degrees()
        src = int(np.flatnonzero(deg > 0)[17])
        want, ep_ref = ref.ppr(src, 300, 0.85, 1e-7, True)
        got, ep, _, _, _ = g.ppr(src, 300, 0.85, 1e-7, True)
        assert ep == ep_ref and close(got, want)
        for root in np.flatnonzero(deg > 0)[[0, 1000]]:
            vis_ref, acts, trace_ref = ref.bfs(int(root))
            lev, _, vis, trace, ep = g.bfs(int(root))
            assert vis == vis_ref and trace == trace_ref and ep == acts.size
            np.testing.assert_array_equal(level_histogram(lev, ep), acts)
    finally:
        ref.close()
        g.close()


@pytest.mark.parametrize("name", ["v100u", "rmat12u"])
def test_oracle_cc_and_hyperanf_match_reference(gold, name):
    """connected_component_t labels (the fixed point: each component's
    smallest id) and hyperanf's average distance at register widths 6 and 8."""
    from oracle import fp64, hll
    V = int(gold[f"{name}__meta"][0])
    s, d = graph_edges(name)
    np.testing.assert_array_equal(fp64.cc_labels(V, s, d, False), gold[f"{name}__cc_labels"])
    comps, major, mv, _ = (int(x) for x in gold[f"{name}__cc_summary"])
    lab = gold[f"{name}__cc_labels"]
    vals, counts = np.unique(lab, return_counts=True)
    assert vals.size == comps and (lab == major).sum() == mv == counts.max()
    for bits, want in zip((6, 8), gold[f"{name}__anf_avg"]):
        avg, _, _, _ = hll.hyperanf(V, s, d, False, bits, 20)
        assert avg == pytest.approx(float(want), rel=1e-12), bits


def weighted_edges(gold, name):
    if name == "w10":
        z = np.load(FIXTURES)
        return z["raw_graph_10_9_weighted__src"], z["raw_graph_10_9_weighted__dst"], z["raw_graph_10_9_weighted__w"]
    _, s, d = oracle.rmat(12, 16, 1)
    return s, d, gold["wrmat12__w"].astype(np.float64)


@pytest.mark.parametrize("name", ["w10", "wrmat12"])
def test_oracle_weighted_pagerank_matches_reference(gold, name):
    from oracle import fp64
    s, d, w = weighted_edges(gold, name)
    V = int(max(s.max(), d.max())) + 1
    for tag, eps in (("100", 0.0), ("eps", 0.001)):
        r, ep, _ = fp64.weighted_pagerank(V, s, d, w, True, 100, 0.85, eps)
        assert ep == int(gold[f"{name}__wpr{tag}_epochs"]), tag
        assert close(r, gold[f"{name}__wpr{tag}"]), tag
