"""Multi-process path of bench.py on CPU (gloo, world size 2): replicas run
independently and the job is timed by the slowest rank (max over ranks),
value = whole-job throughput; only the reduction crosses processes."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import datetime
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    import bench
    assert bench.env_rank() == (rank, world, rank)
    ms = 10.0 + 5.0 * rank  # rank 1 is the slow replica
    m = bench.max_over_ranks(ms, dist, "cpu")
    out[rank] = (m, bench.replica_value(1e9, m, world))
    dist.barrier()
    dist.destroy_process_group()


def test_max_over_ranks_gloo_world2():
    port = _free_port()
    with mp.get_context("spawn").Manager() as mgr:  # no fork of a threaded process
        out = mgr.dict()
        mp.start_processes(_worker, args=(2, port, out), nprocs=2, join=True, start_method="spawn")
        res = dict(out)
    assert res[0] == res[1]
    m, v = res[0]
    assert m == pytest.approx(15.0)
    assert v == pytest.approx(2 * 1e9 / 0.015)


def test_single_process_passthrough():
    import bench
    assert bench.max_over_ranks(3.5, None, "cpu") == 3.5
