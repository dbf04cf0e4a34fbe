"""BFS searches deeper than the levels the start graph runs in one replay (8):
a long chain on its own and hanging off an RMAT core, directed and
undirected, in both vertex orders.  Levels must equal the oracle's bit for
bit, with the same visited count, epoch count and push/pull trace, through
the continuation launches after the first batch; shallow and deep searches
alternate on one graph (the start graph replayed for each), and a search
with another push threshold captures it again."""
import numpy as np
import pytest

import plato_b200 as pb
from oracle import RefGraph

pytestmark = pytest.mark.gpu


def _chain_on_core(n_chain, core_scale):
    """An RMAT core (or one vertex) whose last vertex starts a chain of
    n_chain new vertices: V0-1 -> V0 -> ... -> V0+n_chain-1."""
    if core_scale:
        V0, s0, d0 = pb.rmat(core_scale, 8, 31)
    else:
        V0, s0, d0 = 1, np.array([], np.uint32), np.array([], np.uint32)
    a = np.arange(V0 - 1, V0 + n_chain - 1, dtype=np.uint32)
    return V0 + n_chain, np.concatenate([s0, a]), np.concatenate([d0, a + 1]), V0


def _check(g, ref, V, root, thr=0.05):
    lev_ref, _, vis_ref, tr_ref, ep_ref = ref.bfs(int(root), thr)
    lev, par, st = g.bfs(int(root), push_threshold=thr)
    np.testing.assert_array_equal(lev, lev_ref)
    assert st.visited == vis_ref
    assert st.iterations == ep_ref
    trace = [(tr_ref >> i) & 1 for i in range(min(ep_ref, 64))]
    assert [m == "push" for m in st.mode_trace] == [bool(t) for t in trace]
    reached = np.flatnonzero((lev != pb.PLATO_LEVEL_UNREACHED) & (np.arange(V) != root))
    assert par[root] == root
    assert (lev[par[reached]] == lev[reached] - 1).all()
    return st


@pytest.mark.parametrize("core_scale", [0, 12])
@pytest.mark.parametrize("directed", [True, False])
@pytest.mark.parametrize("relabel", [True, False])
def test_deep_searches_match_the_oracle(core_scale, directed, relabel):
    V, s, d, V0 = _chain_on_core(300, core_scale)
    ref = RefGraph(V, s, d, directed)
    try:
        with pb.Graph(V, s, d, directed, relabel=relabel) as g:
            deep = []
            # the chain's first vertex, the core's last vertex, a vertex half
            # way along, and (undirected) the chain's far end
            roots = [V0, V0 - 1, V0 + 150] + ([V - 1] if not directed else [])
            for root in roots:
                deep.append(_check(g, ref, V, root).iterations)
            assert max(deep) > 8 + 4 * 10  # many continuation batches ran
            if core_scale:  # a search from the core's hub in between, then the chain again
                deg = np.bincount(s, minlength=V) + np.bincount(d, minlength=V)
                _check(g, ref, V, int(np.argmax(deg[:V0])))
                _check(g, ref, V, V0)
            _check(g, ref, V, V0, thr=0.0)  # always pull: the start graph captured again
            _check(g, ref, V, V0, thr=1.01)  # always push
            _check(g, ref, V, V0)
    finally:
        ref.close()
