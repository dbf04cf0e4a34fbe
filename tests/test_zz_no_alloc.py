"""plato_pagerank_csc_noalloc: PageRank that allocates no device memory.

This entry point exists for callers that must not let a library call
cudaMalloc (an application whose own pooling allocator owns the GPU's memory,
a plugin held to a fixed budget, a latency-critical loop that cannot absorb an
allocation's synchronisation).  It keeps its temporaries in a fixed static
device array inside the library.  The test calls it through the C ABI on a
caller-owned CSC (the resident graph's own device arrays, built without
relabelling so caller ids equal the graph's ids) twice in a row and checks
each result against the regular plato_pagerank entry point, within the
PageRank tolerance used everywhere else (L1 <= 1e-6 in normalised units).
The file is named to be collected last.
"""
import ctypes as C

import numpy as np
import pytest

import plato_b200 as pb
from plato_b200 import _lib

pytestmark = pytest.mark.gpu

L1_TOL = 1e-6


def _run_noalloc(lib, view, V, iters, eps, d_out, stream=0):
    o = _lib.PagerankOpts(iters, 0.85, eps)
    st = _lib.RunStats()
    rc = lib.plato_pagerank_csc_noalloc(V, view.stored_edges, C.c_void_p(view.in_offsets),
                                        C.c_void_p(view.in_adj), C.c_void_p(view.out_degree),
                                        C.byref(o), C.c_void_p(d_out), C.c_void_p(stream),
                                        C.byref(st))
    _lib.check(rc, "plato_pagerank_csc_noalloc")
    return st


@pytest.mark.parametrize("directed,iters,eps", [(True, 20, 0.0), (False, 30, 0.0), (True, 100, 0.001)])
def test_noalloc_matches_pagerank_twice(directed, iters, eps):
    import torch

    V, s, d = pb.rmat(15, 16, 21, symmetrize=not directed)
    lib = _lib.load()
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
            got = out.cpu().numpy()
            assert st.iterations == st_ref.iterations
            l1 = float(np.abs(got.astype(np.float64) - want.astype(np.float64)).sum())
            assert l1 <= L1_TOL, l1
            results.append(got)
        assert np.array_equal(results[0].view(np.uint32), results[1].view(np.uint32))


def test_noalloc_rejects_graphs_over_the_scratch_limit():
    import torch

    lib = _lib.load()
    with pb.Graph(3, np.array([0, 1], np.uint32), np.array([1, 2], np.uint32)) as g:
        view = g.device_view()
        out = torch.empty(3, dtype=torch.float32, device="cuda")
        o = _lib.PagerankOpts(5, 0.85, 0.0)
        # sizes beyond PLATO_NOALLOC_SCRATCH_BYTES are refused before any launch
        rc = lib.plato_pagerank_csc_noalloc(1 << 30, 1 << 32, C.c_void_p(view.in_offsets),
                                            C.c_void_p(view.in_adj), C.c_void_p(view.out_degree),
                                            C.byref(o), C.c_void_p(out.data_ptr()), None, None)
        assert rc == _lib.PLATO_EINVAL
        assert b"scratch" in lib.plato_last_error()
