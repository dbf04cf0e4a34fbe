"""CPU tests of the HyperLogLog oracle (oracle/hll.py): murmurhash3, add and
estimate against golden vectors made by the reference's own headers
(tests/golden/make_golden.py), the reference's HyperLogLog unit tests, and
the HyperANF / n-step degree answers the reference's tests assert on
raw_graph_7_7.csv."""
import numpy as np
import pytest

from oracle import hll
from tests.conftest import ROOT


@pytest.fixture(scope="module")
def hg():
    return np.load(ROOT / "tests" / "golden" / "hll_golden.npz")


def _graph(golden, name):
    graphs, _ = golden
    g = graphs[name]
    V = int(max(g["src"].max(), g["dst"].max())) + 1
    return V, g["src"], g["dst"]


def test_murmur3_matches_reference(hg):
    np.testing.assert_array_equal(hll.murmur3_u32(hg["hash_ids"]), hg["hash_values"])


@pytest.mark.parametrize("P", range(4, 17))
def test_add_and_estimate_match_reference(hg, P):
    rows, ids, est = hg[f"p{P}_rows"], hg[f"p{P}_ids"], hg[f"p{P}_est"]
    for r, n, e in zip(rows, ids, est):
        if n >= 0:  # ids 0..n-1 added to an empty row by the reference
            mine = np.zeros(1 << P, np.uint8)
            hll.add(mine, np.arange(n, dtype=np.uint32), P)
            np.testing.assert_array_equal(mine, r)
        got = hll.estimate(r[None, :], P)[0]
        if np.isnan(e):
            assert np.isnan(got)
        else:
            assert got == pytest.approx(e, rel=1e-14, abs=0.0), (P, n)


def test_reference_hll_unit_tests(golden):
    _, kats = golden
    add, merge = kats["hyperloglog"]
    r = np.zeros(1 << add["bits"], np.uint8)
    hll.add(r, np.arange(add["ids"], dtype=np.uint32), add["bits"])
    assert abs(hll.estimate(r, add["bits"])[0] - add["ids"]) / add["ids"] <= add["max_rel_error"]
    P = merge["bits"]
    a = np.zeros(1 << P, np.uint8)
    hll.add(a, np.arange(merge["ids"], dtype=np.uint32), P)
    b = a.copy()
    e1 = hll.estimate(a, P)[0]
    merged = np.maximum(a, b)
    assert abs(hll.estimate(merged, P)[0] - e1) <= np.finfo(float).eps
    extra = np.zeros(1 << P, np.uint8)
    hll.add(extra, np.array([merge["ids"]], np.uint32), P)
    assert hll.estimate(np.maximum(merged, extra), P)[0] >= e1


def test_nstep_degrees_kat(golden):
    _, kats = golden
    for k in kats["nstep_degrees"]:
        V, s, d = _graph(golden, k["graph"])
        din, dout, _ = hll.nstep_degrees(V, s, d, k["is_directed"], step=k["step"], bits=k["bits"],
                                         kind=k["type"])
        for v, (want_in, want_out) in k["values"].items():
            assert (din[int(v)], dout[int(v)]) == (want_in, want_out), k["source"]


def test_hyperanf_kat(golden):
    _, kats = golden
    for k in kats["hyperanf"]:
        V, s, d = _graph(golden, k["graph"])
        avg, anfs, regs, _ = hll.hyperanf(V, s, d, k["is_directed"], bits=k["bits"],
                                          iterations=k["iterations"])
        exact = hll.exact_avg_distance(V, s, d)
        assert abs(avg - exact) <= k["tolerance"], (avg, exact, k["source"])
        assert np.all(np.diff(anfs) > 0)


def test_nstep_chain_counts():
    """On a directed chain 0 -> 1 -> ... -> 9 the ball sizes are exact small
    counts: in-degree(v) = min(v, step), out-degree(v) = min(9 - v, step)."""
    s = np.arange(9, dtype=np.uint32)
    d = s + 1
    for step in (1, 2, 4, -1):
        din, dout, _ = hll.nstep_degrees(10, s, d, True, step=step, bits=12)
        lim = 10 if step < 0 else step
        v = np.arange(10)
        np.testing.assert_array_equal(din, np.minimum(v, lim))
        np.testing.assert_array_equal(dout, np.minimum(9 - v, lim))


def test_nstep_undirected_both_copies_in():
    rng = np.random.default_rng(3)
    s = rng.integers(0, 60, 200).astype(np.uint32)
    d = rng.integers(0, 60, 200).astype(np.uint32)
    din, dout, _ = hll.nstep_degrees(60, s, d, False, step=2, bits=8)
    np.testing.assert_array_equal(din, dout)


def test_hyperanf_push_and_pull_agree():
    """The registers after every epoch do not depend on the engine's choice."""
    rng = np.random.default_rng(5)
    s = rng.integers(0, 300, 1500).astype(np.uint32)
    d = rng.integers(0, 300, 1500).astype(np.uint32)
    a = hll.hyperanf(300, s, d, True, bits=6, push_threshold=0.05)
    b = hll.hyperanf(300, s, d, True, bits=6, push_threshold=2.0)  # every epoch push
    np.testing.assert_array_equal(a[2], b[2])
    np.testing.assert_array_equal(a[1], b[1])
    assert all(b[3])
