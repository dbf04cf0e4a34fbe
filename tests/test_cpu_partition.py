"""1D-partitioned PageRank, host side (no GPU).

* plato_partition_layout: every vertex gets one global internal id, the
  partitions hold ceil((V - r) / P) real rows each, rows within a partition
  keep descending in-degree (so each runs the degree-binned kernels), and the
  edges spread evenly.
* The exchange protocol at world size 2 over gloo: each process computes its
  partition's rows of each PageRank epoch from the assembled state (a numpy
  restatement of the partition pull, test infrastructure standing in for the
  GPU kernel), all-gathers the next state in place and all-reduces the delta
  for the eps exit; the ranks equal the oracle's single-graph PageRank.
* The fused-exchange driver (pagerank_partitioned_p2p) at world size 2 over
  gloo, with a stand-in for the partition: every rank receives the IPC
  handles of all ranks in rank order and drives its partition through
  connect, init, the epochs, the ranks and close, on the current stream.
"""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

import oracle
from plato_b200 import partition


@pytest.mark.parametrize("world", [1, 2, 3, 8])
@pytest.mark.parametrize("directed", [True, False])
def test_layout_balances_rows_and_edges(world, directed):
    V, s, d = oracle.rmat(12, 16, 7, symmetrize=not directed)
    gid, n = partition.layout(V, s, d, world, directed)
    assert n == -(-V // world)
    assert np.unique(gid).size == V and gid.max() < world * n
    indeg = np.bincount(d, minlength=V) + (0 if directed else np.bincount(s, minlength=V))
    owner, row = gid // n, gid % n
    for r in range(world):
        mine = owner == r
        assert mine.sum() == (V - r + world - 1) // world
        assert row[mine].max() == mine.sum() - 1  # real rows first, padding last
        by_row = np.empty(mine.sum(), np.int64)
        by_row[row[mine]] = indeg[mine]
        assert (np.diff(by_row) <= 0).all()  # descending in-degree within the partition
    edges = np.bincount(owner[d], minlength=world) + (0 if directed else np.bincount(owner[s], minlength=world))
    assert edges.max() <= 1.1 * edges.mean()


def _free_port():
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        return so.getsockname()[1]


def _partition_epoch(cols, x, lo, n, real, odeg, V, damping, final):
    """Rows [lo, lo + n) of one epoch (pagerank.hpp:104-135, normalised):
    y = sum of the assembled state over in-edges, then the update."""
    y = np.zeros(n)
    for row, srcs in cols.items():
        y[row] = x[srcs].sum()
    r = (1 - damping) / V + damping * y
    old = x[lo:lo + n]
    if final:
        r[real:] = (1 - damping) / V
        return r, 0.0
    out = np.where(odeg > 0, r / np.maximum(odeg, 1), r)
    out[real:] = (1 - damping) / V
    dl = np.where(odeg > 0, np.abs(out - old) * odeg, np.abs(out - old))[:real].sum()
    return out, dl


def _worker(rank, world, port, eps, out):
    import datetime

    import torch
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    V, s, d = oracle.rmat(10, 16, 3)
    damping, iterations = 0.85, 30
    gid, n = partition.layout(V, s, d, world, True)
    lo = rank * n
    odeg_all = np.bincount(s, minlength=V)
    real = (V - rank + world - 1) // world
    odeg = np.zeros(n)
    mine = (gid >= lo) & (gid < lo + n)
    odeg[gid[mine] - lo] = odeg_all[mine]
    cols = {}
    for u, v in zip(gid[s], gid[d]):
        if lo <= v < lo + n:
            cols.setdefault(int(v - lo), []).append(int(u))
    cols = {k: np.array(v) for k, v in cols.items()}
    x = np.zeros(world * n)
    init = np.where(odeg > 0, 1.0 / (V * np.maximum(odeg, 1)), 1.0 / V)
    init[real:] = (1 - damping) / V
    chunks = [torch.zeros(n, dtype=torch.float64) for _ in range(world)]
    dist.all_gather(chunks, torch.from_numpy(init))
    x = torch.cat(chunks).numpy()
    epoch, ran = 0, 0
    while epoch < iterations:
        final = epoch == iterations - 1
        mine_next, dl = _partition_epoch(cols, x, lo, n, real, odeg, V, damping, final)
        dist.all_gather(chunks, torch.from_numpy(mine_next))
        x = torch.cat(chunks).numpy()
        ran += 1
        if not final and eps > 0:
            t = torch.tensor([dl])
            dist.all_reduce(t)
            if t.item() * V < eps:
                epoch = iterations - 2
        epoch += 1
    out[rank] = (x[gid].tolist(), ran)
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("eps", [0.0, 0.01])
def test_partition_protocol_gloo_world2_matches_oracle(eps):
    port = _free_port()
    with mp.get_context("spawn").Manager() as mgr:
        out = mgr.dict()
        mp.start_processes(_worker, args=(2, port, eps, out), nprocs=2, join=True, start_method="spawn")
        res = dict(out)
    V, s, d = oracle.rmat(10, 16, 3)
    g = oracle.RefGraph(V, s, d, True)
    want, ep, _ = g.pagerank(30, 0.85, eps)
    g.close()
    for rank in (0, 1):
        ranks, ran = res[rank]
        assert ran == ep
        assert np.abs(np.asarray(ranks) - want / V).sum() <= 1e-12


def _p2p_driver_worker(rank, world, port, out):
    """pagerank_partitioned_p2p's host side at world size 2 over gloo, with a
    stand-in for the partition (the library calls need a GPU): what each rank
    sends and receives, and in which order it drives its partition."""
    import datetime
    import types

    import torch
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    calls = []

    class StandIn:
        def __init__(self, vertices, src, dst, r, w, is_directed=True):
            calls.append(("new", r, w, is_directed))
            self.r = r

        def p2p_alloc(self):
            return bytes([self.r + 1]) * (3 * partition.IPC_HANDLE_BYTES)

        def p2p_connect(self, all_handles, timeout_ms=0):
            calls.append(("connect", all_handles, timeout_ms))

        def p2p_init(self, iterations, damping, eps=0.0, stream=0):
            calls.append(("init", iterations, damping, eps, stream))

        def p2p_epoch(self, epoch, damping, stream=0):
            calls.append(("epoch", epoch, stream))

        def p2p_ranks(self, stream=0):
            calls.append(("ranks", stream))
            return np.full(4, self.r, np.float32), 3

        def close(self):
            calls.append(("close",))

    partition.Partition = StandIn
    torch.cuda.current_stream = lambda: types.SimpleNamespace(cuda_stream=77)
    s = np.array([0, 1, 2], np.uint32)
    d = np.array([1, 2, 3], np.uint32)
    ranks, ran = partition.pagerank_partitioned_p2p(4, s, d, 5, 0.85, 0.001, False, None, 250)
    out[rank] = (calls, ranks.tolist(), ran)
    dist.barrier()
    dist.destroy_process_group()


def test_p2p_driver_gloo_world2_exchanges_handles_in_rank_order():
    port = _free_port()
    with mp.get_context("spawn").Manager() as mgr:
        out = mgr.dict()
        mp.start_processes(_p2p_driver_worker, args=(2, port, out), nprocs=2, join=True, start_method="spawn")
        res = dict(out)
    hb = 3 * partition.IPC_HANDLE_BYTES
    handles = b"\x01" * hb + b"\x02" * hb
    for rank in (0, 1):
        calls, ranks, ran = res[rank]
        assert calls[0] == ("new", rank, 2, False)
        assert calls[1] == ("connect", handles, 250)
        assert calls[2] == ("init", 5, 0.85, 0.001, 77)
        assert calls[3:8] == [("epoch", e, 77) for e in range(5)]
        assert calls[8:] == [("ranks", 77), ("close",)]
        assert ranks == [float(rank)] * 4 and ran == 3
