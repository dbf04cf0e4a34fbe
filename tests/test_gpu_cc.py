"""Connected components on the dual-mode engine (plato_connected_components)
against the oracle (oracle/fp64.py) and the reference's own test
(plato/algo/cgm/test/test_cgm.cc: labels equal a BFS labelling from
ascending ids on the fixture graph v100_e2150_ua_c3.csv)."""
import numpy as np
import pytest

import plato_b200 as pb
from oracle import fp64

pytestmark = pytest.mark.gpu


def _summary(V, s, d, directed, lab):
    uniq, counts = np.unique(lab, return_counts=True)
    major = int(uniq[counts == counts.max()].min())
    src = np.concatenate([s, d]) if not directed else s
    edges = int((lab[src] == major).sum())
    return {"components": int(uniq.size), "major_label": major,
            "major_vertices": int(counts.max()), "major_edges": edges // 2 if not directed else edges}


@pytest.mark.parametrize("relabel", [True, False])
def test_cc_reference_fixture_matches_reference_test(golden, relabel):
    graphs, _ = golden
    g0 = graphs["v100_e2150_ua_c3.csv"]
    s, d = g0["src"], g0["dst"]
    V = int(max(s.max(), d.max())) + 1
    want = fp64.cc_components_bfs(V, s, d)
    with pb.Graph(V, s, d, False, relabel=relabel) as g:
        lab, summ, st = g.connected_components()
    np.testing.assert_array_equal(lab, want)
    assert summ == _summary(V, s, d, False, want)
    assert st.iterations >= 1


@pytest.mark.parametrize("directed", [False, True])
def test_cc_rmat_labels_and_summary(directed):
    V, s, d = pb.rmat(14, 16, 6, symmetrize=not directed)
    want = fp64.cc_labels(V, s, d, directed)
    if not directed:
        np.testing.assert_array_equal(want, fp64.cc_components_bfs(V, s, d))
    with pb.Graph(V, s, d, directed) as g:
        lab, summ, st = g.connected_components()
        np.testing.assert_array_equal(lab, want)
        assert summ == _summary(V, s, d, directed, want)
        # the switch only changes how labels travel, not the fixed point
        for thr in (0.0, 1.01):
            lab2, summ2, st2 = g.connected_components(push_threshold=thr)
            np.testing.assert_array_equal(lab2, want)
            assert summ2 == summ
            assert st2.push_iterations == (st2.iterations if thr > 1 else 0)


def test_cc_isolated_vertices_and_chains():
    # 0-1-2 chain, 3 isolated, 4->5 directed edge, 6 isolated
    s = np.array([0, 1, 4], np.uint32)
    d = np.array([1, 2, 5], np.uint32)
    with pb.Graph(7, s, d, False) as g:
        lab, summ, _ = g.connected_components()
        assert lab.tolist() == [0, 0, 0, 3, 4, 4, 6]
        assert summ == {"components": 4, "major_label": 0, "major_vertices": 3, "major_edges": 2}
    with pb.Graph(7, s, d, True) as g:
        lab, summ, _ = g.connected_components()
        assert lab.tolist() == [0, 0, 0, 3, 4, 4, 6]  # 0 reaches 1 and 2; 4 reaches 5
    rs = np.array([2, 1], np.uint32)  # directed 2 -> 1 -> 0: everything reached from 2
    rd = np.array([1, 0], np.uint32)
    with pb.Graph(3, rs, rd, True) as g:
        lab, _, _ = g.connected_components()
        assert lab.tolist() == [0, 1, 2]  # labels flow along edges: no smaller id reaches 1 or 2
