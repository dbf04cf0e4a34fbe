"""Empty inputs on the GPU path: graphs with no edges at all (one vertex, and
several isolated vertices), directed and undirected, in the relabelled
(degree-binned) and caller (merge-path) orders.  Every entry point must run
and agree with the oracle: PageRank keeps (1-d)/V on every vertex, PPR keeps
the teleport mass on its seeds, BFS reaches only its root, every vertex is its
own component, and batched and served queries equal their one-at-a-time
answers."""
import numpy as np
import pytest

import plato_b200 as pb
from oracle import RefGraph

pytestmark = pytest.mark.gpu

L1_TOL = 1e-6
NONE = np.array([], np.uint32)


def _l1(a, b):
    return float(np.abs(np.asarray(a, np.float64) - np.asarray(b, np.float64)).sum())


@pytest.fixture(params=[(1, True), (5, True), (5, False)], ids=["V1", "V5-directed", "V5-undirected"])
def edgeless(request):
    V, directed = request.param
    ref = RefGraph(V, NONE, NONE, directed)
    yield V, directed, ref
    ref.close()


@pytest.mark.parametrize("relabel", [True, False])
def test_edgeless_rank_entry_points(edgeless, relabel):
    V, directed, ref = edgeless
    with pb.Graph(V, NONE, NONE, directed, relabel=relabel) as g:
        assert not g.out_degrees().any()
        r, st = g.pagerank(5, 0.85, 0.0)
        want, ep, _ = ref.pagerank(5, 0.85, 0.0)
        assert st.iterations == ep == 5
        assert _l1(r, want / V) <= L1_TOL
        r, st = g.pagerank(100, 0.85, 0.001)  # the eps exit: delta is 0 after the first epoch
        want, ep, _ = ref.pagerank(100, 0.85, 0.001)
        assert st.iterations == ep and _l1(r, want / V) <= L1_TOL
        src = V - 1
        for mode, pushpull in ((pb.PLATO_PPR_PULL, False), (pb.PLATO_PPR_PUSHPULL, True)):
            p, st = g.personalized_pagerank(src, 10, 0.85, 0.0, mode)
            want, ep, pe, _, _ = ref.ppr(src, 10, 0.85, 0.0, pushpull)
            assert st.iterations == ep and _l1(p, want) <= L1_TOL
        seeds = np.array(sorted({0, V - 1}), np.uint32)
        p, st = g.seedset_ppr(seeds, 50, 0.85, 1e-6)
        want, ep, _ = ref.seedset_ppr(seeds, 50, 0.85, 1e-6)
        assert abs(st.iterations - ep) <= 1 and _l1(p, want) <= L1_TOL


@pytest.mark.parametrize("relabel", [True, False])
def test_edgeless_traversals(edgeless, relabel):
    V, directed, ref = edgeless
    with pb.Graph(V, NONE, NONE, directed, relabel=relabel) as g:
        for root in sorted({0, V - 1}):
            lev, par, st = g.bfs(root)
            want, _, visited, _, _ = ref.bfs(root)
            np.testing.assert_array_equal(lev, want)
            assert st.visited == visited == 1 and par[root] == root
        lab, summary, _ = g.connected_components()
        np.testing.assert_array_equal(lab, np.arange(V, dtype=np.uint32))
        assert summary["components"] == V and summary["major_vertices"] == 1 and summary["major_edges"] == 0


def test_edgeless_batched_and_served_queries(edgeless):
    V, directed, ref = edgeless
    sets = [np.array([0], np.uint32), np.array([V - 1], np.uint32), np.arange(V, dtype=np.uint32)]
    with pb.Graph(V, NONE, NONE, directed) as g:
        out = g.ppr_batch(sets, 50, 0.85, 1e-6, topk=min(V, 3), ranks=True)
        for q, s in enumerate(sets):
            want, ep, _ = ref.seedset_ppr(s, 50, 0.85, 1e-6)
            assert abs(int(out["iterations"][q]) - ep) <= 1
            assert _l1(out["ranks"][q], want) <= L1_TOL
        with pb.PPRServer(g, max_slots=2, hbm_budget_bytes=1 << 20, max_iterations=50, eps=1e-6,
                          topk=1) as srv:
            ids = {srv.submit(s): q for q, s in enumerate(sets)}
            got = {}
            for _ in range(1000):
                if len(got) == len(sets):
                    break
                srv.step()
                while (r := srv.poll()) is not None:
                    got[ids[r[0]]] = r
            assert len(got) == len(sets)
            for q in range(len(sets)):
                assert got[q][2][0] == pytest.approx(float(out["topk_vals"][q][0]), abs=1e-7)
