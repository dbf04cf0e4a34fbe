"""GPU parity of batched multi-source PPR and the continuous-batching server.

Tolerance: L1 <= 1e-6 per query vector against the FP64 oracle (seed-set PPR
with trustrank semantics); top-k ids must equal the top-k of the engine's own
rank vector (ties by smaller id); a query must give the same result alone and
in a mix, within the same L1 tolerance.
"""
import numpy as np
import pytest

import plato_b200 as pb
from oracle import RefGraph

pytestmark = pytest.mark.gpu

L1_TOL = 1e-6


def _l1(a, b):
    return float(np.abs(np.asarray(a, np.float64) - np.asarray(b, np.float64)).sum())


def zipf_seed_sets(deg, K, max_size, seed):
    """Seed-set sizes Zipf(s=1.5) clipped to [1, max_size], members uniform among deg > 0."""
    rng = np.random.default_rng(seed)
    cands = np.flatnonzero(deg > 0)
    sizes = np.minimum(rng.zipf(1.5, K), max_size)
    return [rng.choice(cands, int(n), replace=False).astype(np.uint32) for n in sizes]


@pytest.fixture(scope="module")
def g14():
    V, s, d = pb.rmat(14, 16, 4)
    ref = RefGraph(V, s, d, True)
    g = pb.Graph(V, s, d, True)
    yield V, s, d, ref, g
    g.close()


def test_batch_matches_oracle_per_query(g14):
    V, s, d, ref, g = g14
    sets = zipf_seed_sets(ref.out_degrees(), 20, 32, 1)
    out = g.ppr_batch(sets, max_iterations=300, eps=1e-6, ranks=True)
    for q, S in enumerate(sets):
        want, ep, _ = ref.seedset_ppr(S, 300, 0.85, 1e-6)
        assert abs(int(out["iterations"][q]) - ep) <= 1
        assert _l1(out["ranks"][q], want) <= L1_TOL, q


@pytest.mark.parametrize("relabel", [True, False])
def test_seedset_ppr_plain_engine(g14, relabel):
    """The plain one-query engine (trustrank with explicit seeds, pull-only)."""
    V, s, d, ref, g = g14
    sets = zipf_seed_sets(ref.out_degrees(), 4, 32, 9)
    with pb.Graph(V, s, d, True, relabel=relabel) as gg:
        for S in sets:
            want, ep, _ = ref.seedset_ppr(S, 300, 0.85, 1e-6)
            got, st = gg.seedset_ppr(S, 300, 0.85, 1e-6)
            assert abs(st.iterations - ep) <= 1
            assert _l1(got, want) <= L1_TOL
            fixed, st2 = gg.seedset_ppr(S, 17, 0.85, 0.0)
            want2, ep2, _ = ref.seedset_ppr(S, 17, 0.85, 0.0)
            assert st2.iterations == ep2 == 17
            assert _l1(fixed, want2) <= L1_TOL


def test_batch_fixed_iterations_exact_count(g14):
    V, s, d, ref, g = g14
    sets = zipf_seed_sets(ref.out_degrees(), 9, 8, 2)
    out = g.ppr_batch(sets, max_iterations=25, eps=0.0, ranks=True)
    assert (out["iterations"] == 25).all()
    for q, S in enumerate(sets):
        want, ep, _ = ref.seedset_ppr(S, 25, 0.85, 0.0)
        assert ep == 25
        assert _l1(out["ranks"][q], want) <= L1_TOL


@pytest.mark.parametrize("kt", [8, 16, 32, 64, 128])
def test_batch_k_tiles_agree(g14, kt):
    V, s, d, ref, g = g14
    sets = zipf_seed_sets(ref.out_degrees(), 13, 16, 3)
    base = g.ppr_batch(sets, max_iterations=200, eps=1e-6, ranks=True, k_tile=32)
    out = g.ppr_batch(sets, max_iterations=200, eps=1e-6, ranks=True, k_tile=kt)
    for q in range(len(sets)):
        assert _l1(out["ranks"][q], base["ranks"][q]) <= L1_TOL


def test_batch_autotuned_k_tile_is_used(g14):
    V, s, d, ref, g = g14
    sets = zipf_seed_sets(ref.out_degrees(), 70, 16, 5)
    kt = g.ppr_batch_k_tile(len(sets))
    assert kt in (8, 16, 32, 64, 128)
    assert g.ppr_batch_k_tile(len(sets)) == kt  # cached per graph and bucket
    auto = g.ppr_batch(sets, max_iterations=200, eps=1e-6, ranks=True)
    fixed = g.ppr_batch(sets, max_iterations=200, eps=1e-6, ranks=True, k_tile=kt)
    assert np.array_equal(auto["ranks"].view(np.uint32), fixed["ranks"].view(np.uint32))
    with pytest.raises(pb.PlatoError):
        g.ppr_batch_k_tile(0)


def test_batch_alone_equals_in_mix(g14):
    V, s, d, ref, g = g14
    sets = zipf_seed_sets(ref.out_degrees(), 40, 32, 4)
    mix = g.ppr_batch(sets, max_iterations=300, eps=1e-6, ranks=True, k_tile=32)
    for q in (0, 17, 39):
        alone = g.ppr_batch([sets[q]], max_iterations=300, eps=1e-6, ranks=True, k_tile=32)
        assert alone["iterations"][0] == mix["iterations"][q]
        # same column arithmetic: identical bits
        assert np.array_equal(alone["ranks"][0].view(np.uint32), mix["ranks"][q].view(np.uint32))


def test_batch_topk_exact(g14):
    V, s, d, ref, g = g14
    sets = zipf_seed_sets(ref.out_degrees(), 12, 32, 5)
    for k in (1, 10, 100):
        out = g.ppr_batch(sets, max_iterations=300, eps=1e-6, ranks=True, topk=k)
        for q in range(len(sets)):
            r = out["ranks"][q]
            order = np.lexsort((np.arange(V), -r.astype(np.float64)))[:k]
            np.testing.assert_array_equal(out["topk_ids"][q], order.astype(np.uint32))
            np.testing.assert_array_equal(out["topk_vals"][q], r[order])


def test_batch_topk_small_graph_pads():
    s = np.array([0, 1, 2], np.uint32)
    d = np.array([1, 2, 0], np.uint32)
    with pb.Graph(3, s, d, True) as g:
        out = g.ppr_batch([[0]], max_iterations=50, eps=1e-9, topk=5, ranks=True)
    assert out["topk_ids"][0, 3] == 0xFFFFFFFF and out["topk_vals"][0, 4] == 0.0
    assert sorted(out["topk_ids"][0, :3].tolist()) == [0, 1, 2]


def test_batch_rejects_bad_input(g14):
    V, s, d, ref, g = g14
    with pytest.raises(pb.PlatoError):
        g.ppr_batch([[V + 5]])
    with pytest.raises(pb.PlatoError):
        g.ppr_batch([[0], []])
    with pytest.raises(pb.PlatoError):
        g.ppr_batch([[0]], topk=2000)


def test_server_results_match_batch_and_alone(g14):
    V, s, d, ref, g = g14
    sets = zipf_seed_sets(ref.out_degrees(), 30, 64, 6)
    k = 50
    with pb.PPRServer(g, max_slots=16, hbm_budget_bytes=1 << 30, max_iterations=300, eps=1e-6,
                      topk=k) as srv:
        ids = {}
        results = {}
        # staggered arrivals: 4 requests per step for the first steps
        pending = list(enumerate(sets))
        steps = 0
        while len(results) < len(sets):
            for _ in range(4):
                if pending:
                    q, S = pending.pop(0)
                    ids[srv.submit(S)] = q
            srv.step()
            steps += 1
            while (r := srv.poll()) is not None:
                rid, tid, tval, it = r
                results[ids[rid]] = (tid.copy(), tval.copy(), it)
            assert steps < 5000
        st = srv.stats()
        assert st["completed"] == len(sets) and st["live"] == 0 and st["queued"] == 0
    for q in (0, 5, 29):
        alone = g.ppr_batch([sets[q]], max_iterations=300, eps=1e-6, topk=k, ranks=True)
        want, ep, _ = ref.seedset_ppr(sets[q], 300, 0.85, 1e-6)
        tid, tval, it = results[q]
        assert abs(it - ep) <= 1
        np.testing.assert_allclose(tval, alone["topk_vals"][0], rtol=0, atol=1e-6)
        # top-k values against the FP64 oracle's vector
        w = np.sort(want)[::-1][:k]
        assert np.abs(tval.astype(np.float64) - w).sum() <= L1_TOL


def test_server_budget_limits_slots(g14):
    V, s, d, ref, g = g14
    per = 8 * V
    with pb.PPRServer(g, max_slots=64, hbm_budget_bytes=3 * per + 10, topk=5) as srv:
        for q in range(6):
            srv.submit([q])
        srv.step()
        st = srv.stats()
        assert st["live"] <= 3 and st["queued"] >= 3
    with pytest.raises(pb.PlatoError) as e:
        pb.PPRServer(g, max_slots=4, hbm_budget_bytes=per // 2, topk=5)
    assert e.value.code == 2  # PLATO_ENOMEM
