"""GPU parity of HyperANF and n-step degrees (HyperLogLog propagation) against
the oracle (oracle/hll.py).

Bars: registers bit-exact; n-step degrees bit-exact; ANF series within a
relative 1e-12 of the oracle's (the per-vertex estimates match up to the last
bit of a log, and the two sums run in different orders) with the same
length; the engine's push/pull trace equal to the oracle's.  The reference's
own answers on raw_graph_7_7.csv are checked as well."""
import numpy as np
import pytest

import plato_b200 as pb
from oracle import hll

pytestmark = pytest.mark.gpu

ANF_RTOL = 1e-12


def _graph(golden, name):
    graphs, _ = golden
    g = graphs[name]
    V = int(max(g["src"].max(), g["dst"].max())) + 1
    return V, g["src"], g["dst"]


def _trace(stats):
    return [m == "push" for m in stats.mode_trace]


def test_nstep_degrees_reference_kat(golden):
    _, kats = golden
    for k in kats["nstep_degrees"]:
        V, s, d = _graph(golden, k["graph"])
        with pb.Graph(V, s, d, k["is_directed"]) as g:
            din, dout, _ = g.nstep_degrees(step=k["step"], bits=k["bits"], kind=k["type"])
        for v, (want_in, want_out) in k["values"].items():
            assert (din[int(v)], dout[int(v)]) == (want_in, want_out), k["source"]


def test_hyperanf_reference_kat(golden):
    _, kats = golden
    for k in kats["hyperanf"]:
        V, s, d = _graph(golden, k["graph"])
        with pb.Graph(V, s, d, k["is_directed"]) as g:
            avg, anfs, regs, _ = g.hyperanf(k["iterations"], k["bits"], registers=True)
        want_avg, want_anfs, want_regs, _ = hll.hyperanf(V, s, d, k["is_directed"], bits=k["bits"],
                                                         iterations=k["iterations"])
        assert abs(avg - hll.exact_avg_distance(V, s, d)) <= k["tolerance"], k["source"]
        np.testing.assert_array_equal(regs, want_regs)
        np.testing.assert_allclose(anfs, want_anfs, rtol=ANF_RTOL)
        assert avg == pytest.approx(want_avg, rel=1e-9)


@pytest.mark.parametrize("scale,bits,directed", [(12, 6, True), (12, 6, False), (11, 4, True),
                                                 (11, 8, False), (10, 10, True), (9, 12, False),
                                                 (8, 14, True)])
def test_hyperanf_matches_oracle(scale, bits, directed):
    V, s, d = pb.rmat(scale, 16, 7)
    want_avg, want_anfs, want_regs, want_modes = hll.hyperanf(V, s, d, directed, bits=bits)
    for relabel in (True, False):
        with pb.Graph(V, s, d, directed, relabel=relabel) as g:
            avg, anfs, regs, st = g.hyperanf(20, bits, registers=True)
        np.testing.assert_array_equal(regs, want_regs)
        assert anfs.size == want_anfs.size
        np.testing.assert_allclose(anfs, want_anfs, rtol=ANF_RTOL)
        assert avg == pytest.approx(want_avg, rel=1e-9)
        assert st.iterations == len(want_modes)
        assert _trace(st) == want_modes


def test_hyperanf_iteration_cap_and_push_epochs():
    V, s, d = pb.rmat(12, 8, 3)
    for iters, thr in ((1, 0.05), (3, 0.05), (20, 0.5), (20, 2.0)):
        want_avg, want_anfs, want_regs, want_modes = hll.hyperanf(V, s, d, True, bits=6, iterations=iters,
                                                                  push_threshold=thr)
        with pb.Graph(V, s, d, True) as g:
            avg, anfs, regs, st = g.hyperanf(iters, 6, push_threshold=thr, registers=True)
        np.testing.assert_array_equal(regs, want_regs)
        np.testing.assert_allclose(anfs, want_anfs, rtol=ANF_RTOL)
        assert _trace(st) == want_modes


@pytest.mark.parametrize("step", [1, 2, 3, -1])
@pytest.mark.parametrize("bits", [6, 9])
def test_nstep_all_targets_match_oracle(step, bits):
    V, s, d = pb.rmat(11, 8, 5)
    for directed in (True, False):
        want_in, want_out, want_modes = hll.nstep_degrees(V, s, d, directed, step=step, bits=bits)
        with pb.Graph(V, s, d, directed) as g:
            din, dout, st = g.nstep_degrees(step=step, bits=bits)
        np.testing.assert_array_equal(din, want_in)
        np.testing.assert_array_equal(dout, want_out)
        assert _trace(st) == [p for _, p in want_modes][:64]


@pytest.mark.parametrize("kind", ["in", "out", "both"])
def test_nstep_target_subsets_match_oracle(kind):
    """Few targets put the spread and propagate epochs in push mode, where the
    reference scatters forward even in reversed phases."""
    V, s, d = pb.rmat(12, 8, 9)
    rng = np.random.default_rng(11)
    for n_targets in (1, 5, 200):
        tg = np.zeros(V, dtype=bool)
        tg[rng.choice(V, n_targets, replace=False)] = True
        for directed, opt_dir in ((True, True), (True, False), (False, False)):
            want_in, want_out, want_modes = hll.nstep_degrees(V, s, d, directed, step=3, bits=6, kind=kind,
                                                              is_directed=opt_dir, targets=tg)
            with pb.Graph(V, s, d, directed) as g:
                din, dout, st = g.nstep_degrees(step=3, bits=6, kind=kind, is_directed=opt_dir, targets=tg)
            np.testing.assert_array_equal(din, want_in)
            np.testing.assert_array_equal(dout, want_out)
            assert _trace(st) == [p for _, p in want_modes][:64]
            assert any(p for _, p in want_modes) or n_targets == 200


def test_hll_edge_cases():
    s = np.array([], np.uint32)
    with pb.Graph(5, s, s, True) as g:
        avg, anfs, regs, st = g.hyperanf(20, 6, registers=True)
        assert np.isnan(avg) and anfs.size == 1 and st.iterations == 1
        np.testing.assert_array_equal(regs, hll.single(np.arange(5, dtype=np.uint32), 6))
        din, dout, _ = g.nstep_degrees(step=3, bits=6)
        assert not din.any() and not dout.any()
    with pb.Graph(3, np.array([0, 1], np.uint32), np.array([1, 2], np.uint32), True) as g:
        for bad in (3, 17):
            with pytest.raises(pb.PlatoError):
                g.hyperanf(5, bad)
            with pytest.raises(pb.PlatoError):
                g.nstep_degrees(step=2, bits=bad)
