"""1D-partitioned PageRank on the GPU.

* P = 1..4 partitions emulated in one process on one GPU (each writes its
  slice of a shared state, so no exchange is needed): the partition kernels
  and layout give the single-graph plato_pagerank's ranks within the
  PageRank tolerance, with the same epoch count, on directed and undirected
  RMAT graphs, with and without the eps exit.
* The driver with its collectives over NCCL at world size 1 (the process
  group a torchrun job of one GPU has): same ranks.
* The fused exchange over peer memory (plato_partition_p2p_*), P = 1..4
  partitions in one process on one GPU, each epoch run for every partition
  before the next (so every wait is already satisfied): the same ranks as
  the all-gather path bit for bit, and plato_pagerank's within tolerance.
* A wait that nothing satisfies (a partition that never publishes) gives up
  after its timeout and the run reports PLATO_ETIMEDOUT; the GPU stays
  usable.
"""
import os
import socket

import numpy as np
import pytest

import plato_b200 as pb
from plato_b200 import partition

pytestmark = pytest.mark.gpu

L1_TOL = 1e-6


@pytest.mark.parametrize("world", [1, 2, 3, 4])
@pytest.mark.parametrize("directed,eps", [(True, 0.0), (False, 0.0), (True, 0.001)])
def test_emulated_partitions_match_single_graph(world, directed, eps):
    V, s, d = pb.rmat(15, 16, 17, symmetrize=not directed)
    with pb.Graph(V, s, d, directed) as g:
        want, st = g.pagerank(30, 0.85, eps)
    got, ran = partition.emulate_partitions(V, s, d, world, 30, 0.85, eps, directed)
    assert ran == st.iterations
    assert float(np.abs(got.astype(np.float64) - want.astype(np.float64)).sum()) <= L1_TOL


def test_partition_rows_and_edges_add_up():
    V, s, d = pb.rmat(14, 16, 18)
    parts = [partition.Partition(V, s, d, r, 3) for r in range(3)]
    try:
        assert sum(p.real_rows for p in parts) == V
        assert sum(p.edges for p in parts) == s.size
        assert len({p.rows for p in parts}) == 1
    finally:
        for p in parts:
            p.close()


def _free_port():
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        return so.getsockname()[1]


def test_driver_over_nccl_world1():
    import datetime

    import torch.distributed as dist
    V, s, d = pb.rmat(14, 16, 19)
    with pb.Graph(V, s, d, True) as g:
        want, st = g.pagerank(25, 0.85, 0.001)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(_free_port()))
    dist.init_process_group("nccl", rank=0, world_size=1, timeout=datetime.timedelta(seconds=60))
    try:
        got, ran = partition.pagerank_partitioned(V, s, d, 25, 0.85, 0.001)
    finally:
        dist.destroy_process_group()
    assert ran == st.iterations
    assert float(np.abs(got.astype(np.float64) - want.astype(np.float64)).sum()) <= L1_TOL


@pytest.mark.parametrize("world", [1, 2, 3, 4])
@pytest.mark.parametrize("directed,eps", [(True, 0.0), (False, 0.0), (True, 0.001)])
def test_p2p_exchange_equals_allgather_path(world, directed, eps):
    V, s, d = pb.rmat(15, 16, 17, symmetrize=not directed)
    ref, ran_ref = partition.emulate_partitions(V, s, d, world, 30, 0.85, eps, directed)
    got, ran = partition.emulate_partitions_p2p(V, s, d, world, 30, 0.85, eps, directed)
    assert ran == ran_ref
    if eps == 0.0:
        assert ran == 30
    assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))  # the same row sums, bit for bit
    with pb.Graph(V, s, d, directed) as g:
        want, st = g.pagerank(30, 0.85, eps)
    assert ran == st.iterations
    assert float(np.abs(got.astype(np.float64) - want.astype(np.float64)).sum()) <= L1_TOL


def test_p2p_wait_gives_up_and_reports_timeout():
    import ctypes as C

    from plato_b200 import _lib
    V, s, d = pb.rmat(12, 16, 20)
    parts = [partition.Partition(V, s, d, r, 2) for r in range(2)]
    try:
        arr = (C.c_void_p * 2)(*[p._h.value for p in parts])
        _lib.check(_lib.load().plato_partition_p2p_connect_local(arr, 2, 200), "plato_partition_p2p_connect_local")
        for p in parts:
            p.p2p_reset()
        parts[0].p2p_init(1, 0.85)  # partition 1 never publishes its state
        parts[0].p2p_epoch(0, 0.85)
        with pytest.raises(pb.PlatoError) as e:
            parts[0].p2p_state()
        assert e.value.code == _lib.PLATO_ETIMEDOUT
    finally:
        for p in parts:
            p.close()
    with pb.Graph(V, s, d, True) as g:  # the context is still usable
        r, st = g.pagerank(5)
        assert st.iterations == 5 and np.isfinite(r).all()


def test_p2p_driver_world1():
    """pagerank_partitioned_p2p in a one-process group: its IPC handles are
    made and exchanged, its epochs run with no collective."""
    import datetime

    import torch.distributed as dist
    V, s, d = pb.rmat(14, 16, 21)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(_free_port()))
    dist.init_process_group("nccl", rank=0, world_size=1, timeout=datetime.timedelta(seconds=60))
    try:
        got, ran = partition.pagerank_partitioned_p2p(V, s, d, 25, 0.85, 0.001)
    finally:
        dist.destroy_process_group()
    with pb.Graph(V, s, d, True) as g:
        want, st = g.pagerank(25, 0.85, 0.001)
    assert ran == st.iterations
    assert float(np.abs(got.astype(np.float64) - want.astype(np.float64)).sum()) <= L1_TOL
