"""plato_pagerank_csc_noalloc: PageRank that allocates no device memory.

This entry point exists for callers that must not let a library call
cudaMalloc: an application whose own pooling allocator owns the GPU's memory,
a plugin held to a fixed budget, or a latency-critical loop that cannot absorb
an allocation's synchronisation.  It keeps its temporaries in a fixed static
device array inside the library.  These tests call it through the C ABI on a
caller-owned CSC (the resident graph's own device arrays, built without
relabelling so caller ids equal the graph's ids), twice in a row, and check
each result against the regular plato_pagerank entry point and against the
FP64 oracle, within the PageRank tolerance used everywhere else (L1 <= 1e-6
in normalised units).  RMAT s17 has more vertices than the pull kernel's
shared-memory rank tile, so its gathers also read global memory; a small
graph run before and after a large one checks that nothing a call reads is
left over from the previous call.  The file is named to be collected last.
"""
import ctypes as C

import numpy as np
import pytest

import plato_b200 as pb
from plato_b200 import _lib

pytestmark = pytest.mark.gpu

L1_TOL = 1e-6


def _run_noalloc(lib, view, V, iters, eps, d_out, stream=0, stats=True):
    o = _lib.PagerankOpts(iters, 0.85, eps)
    st = _lib.RunStats()
    rc = lib.plato_pagerank_csc_noalloc(V, view.stored_edges, C.c_void_p(view.in_offsets),
                                        C.c_void_p(view.in_adj), C.c_void_p(view.out_degree),
                                        C.byref(o), C.c_void_p(d_out), C.c_void_p(stream),
                                        C.byref(st) if stats else None)
    _lib.check(rc, "plato_pagerank_csc_noalloc")
    return st


def _oracle_pagerank(V, s, d, directed, iters, eps):
    from oracle import RefGraph
    ref = RefGraph(V, s, d, directed)
    try:
        want, ep, _ = ref.pagerank(iters, 0.85, eps)
    finally:
        ref.close()
    return want / V, ep


@pytest.mark.parametrize("scale,directed,iters,eps", [(15, True, 20, 0.0), (15, False, 30, 0.0),
                                                      (15, True, 100, 0.001), (17, True, 20, 0.0),
                                                      (17, False, 100, 0.001)])
def test_noalloc_matches_pagerank_and_oracle_twice(scale, directed, iters, eps):
    import torch

    V, s, d = pb.rmat(scale, 16, 21, symmetrize=not directed)
    lib = _lib.load()
    oracle_ranks, oracle_epochs = _oracle_pagerank(V, s, d, directed, iters, eps)
    with pb.Graph(V, s, d, directed, relabel=False) as g:
        want, st_ref = g.pagerank(iters, 0.85, eps)
        view = g.device_view()
        out = torch.empty(V, dtype=torch.float32, device="cuda")
        results = []
        for _ in range(2):
            out.fill_(float("nan"))
            torch.cuda.synchronize()
            st = _run_noalloc(lib, view, V, iters, eps, out.data_ptr())
            torch.cuda.synchronize()
            got = out.cpu().numpy().astype(np.float64)
            assert st.iterations == st_ref.iterations
            assert abs(st.iterations - oracle_epochs) <= (1 if eps > 0 else 0)
            if eps > 0:
                assert st.delta == pytest.approx(st_ref.delta, rel=1e-4)
            else:
                assert st.delta == st_ref.delta == 0.0
            l1_entry = float(np.abs(got - want.astype(np.float64)).sum())
            l1_oracle = float(np.abs(got - oracle_ranks).sum())
            assert l1_entry <= L1_TOL, l1_entry
            assert l1_oracle <= L1_TOL, l1_oracle
            results.append(got)
        assert np.array_equal(results[0], results[1])


def test_noalloc_small_after_large_is_unchanged():
    """Scratch keeps the previous call's contents: a small graph's result must
    be bit-identical before and after a larger graph used more of it."""
    import torch

    lib = _lib.load()
    Vs, ss, ds = pb.rmat(12, 16, 31)
    Vl, sl, dl = pb.rmat(17, 16, 32)
    with pb.Graph(Vs, ss, ds, True, relabel=False) as gs, pb.Graph(Vl, sl, dl, True, relabel=False) as gl:
        small = torch.empty(Vs, dtype=torch.float32, device="cuda")
        large = torch.empty(Vl, dtype=torch.float32, device="cuda")
        got = []
        for view, V, out in ((gs.device_view(), Vs, small), (gl.device_view(), Vl, large),
                             (gs.device_view(), Vs, small)):
            out.fill_(float("nan"))
            _run_noalloc(lib, view, V, 25, 0.001, out.data_ptr(), stats=False)
            torch.cuda.synchronize()
            if V == Vs:
                got.append(out.cpu().numpy().copy())
        assert np.array_equal(got[0].view(np.uint32), got[1].view(np.uint32))
        want, _ = _oracle_pagerank(Vs, ss, ds, True, 25, 0.001)
        assert float(np.abs(got[1].astype(np.float64) - want).sum()) <= L1_TOL


def test_noalloc_rejects_graphs_over_the_scratch_limit_and_unaligned_ranks():
    import torch

    lib = _lib.load()
    with pb.Graph(3, np.array([0, 1], np.uint32), np.array([1, 2], np.uint32), relabel=False) as g:
        view = g.device_view()
        out = torch.empty(8, dtype=torch.float32, device="cuda")
        o = _lib.PagerankOpts(5, 0.85, 0.0)
        # sizes beyond PLATO_NOALLOC_SCRATCH_BYTES are refused before any launch
        rc = lib.plato_pagerank_csc_noalloc(1 << 30, 1 << 32, C.c_void_p(view.in_offsets),
                                            C.c_void_p(view.in_adj), C.c_void_p(view.out_degree),
                                            C.byref(o), C.c_void_p(out.data_ptr()), None, None)
        assert rc == _lib.PLATO_EINVAL
        assert b"scratch" in lib.plato_last_error()
        # a rank buffer that is not 16-byte aligned is refused before any launch
        rc = lib.plato_pagerank_csc_noalloc(3, view.stored_edges, C.c_void_p(view.in_offsets),
                                            C.c_void_p(view.in_adj), C.c_void_p(view.out_degree),
                                            C.byref(o), C.c_void_p(out.data_ptr() + 4), None, None)
        assert rc == _lib.PLATO_EINVAL
        assert b"aligned" in lib.plato_last_error()
        # the context is still good: a proper call runs
        _run_noalloc(lib, view, 3, 5, 0.0, out.data_ptr())
        torch.cuda.synchronize()
        assert np.isfinite(out[:3].cpu().numpy()).all()
