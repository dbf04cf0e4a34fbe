"""1D-partitioned PageRank over several GPUs (one process per GPU).

The host side of ``plato_partition_*`` (include/plato_b200.h): every process
builds its partition from the whole edge list, and each epoch is one pull
over the partition's rows followed by an in-place all-gather of the next
state over ``torch.distributed`` (NCCL over NVLink on GPUs), mirroring the
reference's per-epoch exchange of pull messages (the reference sends each
message to its owner over MPI, plato/graph/message_passing.hpp:88-144) and
its delta allreduce (plato/graph/state/detail.hpp:77).

    from plato_b200.partition import pagerank_partitioned
    ranks, epochs = pagerank_partitioned(V, src, dst, iterations=20)   # inside torchrun

``emulate_partitions`` runs P partitions in one process on one GPU, one after
the other on a shared state buffer (each writes its own slice, so the
assembled state needs no exchange): the partition kernels and layout with no
collective, for checks on a single GPU.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import check, load

IPC_HANDLE_BYTES = 64  # PLATO_IPC_HANDLE_BYTES


def _u32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.uint32)


def layout(vertices: int, src, dst, world: int, is_directed: bool = True):
    """-> (global internal id of every caller vertex, rows per partition); host only."""
    lib = load()
    s, d = _u32(src), _u32(dst)
    info = _lib.GraphInfo(1 if is_directed else 0, int(vertices), int(s.size), max(int(vertices) - 1, 0))
    gid = np.empty(int(vertices), np.uint32)
    n = C.c_uint32()
    check(lib.plato_partition_layout(C.byref(info), C.c_void_p(s.ctypes.data), C.c_void_p(d.ctypes.data), world,
                                     C.c_void_p(gid.ctypes.data), C.byref(n)), "plato_partition_layout")
    return gid, int(n.value)


class Partition:
    """Partition `rank` of `world` of a graph, resident on the current GPU."""

    def __init__(self, vertices: int, src, dst, rank: int, world: int, is_directed: bool = True):
        self._lib = load()
        s, d = _u32(src), _u32(dst)
        info = _lib.GraphInfo(1 if is_directed else 0, int(vertices), int(s.size), max(int(vertices) - 1, 0))
        h = C.c_void_p()
        check(self._lib.plato_partition_create(C.byref(info), C.c_void_p(s.ctypes.data), C.c_void_p(d.ctypes.data),
                                               rank, world, C.byref(h)), "plato_partition_create")
        self._h = h
        self.rank, self.world = rank, world
        v, n, real, e = C.c_uint32(), C.c_uint32(), C.c_uint32(), C.c_uint64()
        check(self._lib.plato_partition_info(h, C.byref(v), C.byref(n), C.byref(real), C.byref(e)),
              "plato_partition_info")
        self.vertices, self.rows, self.real_rows, self.edges = int(v.value), int(n.value), int(real.value), int(e.value)

    def close(self):
        if getattr(self, "_h", None):
            self._lib.plato_partition_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def init(self, d_state: int, damping: float, stream: int = 0):
        check(self._lib.plato_partition_pagerank_init(self._h, C.c_void_p(d_state), damping, C.c_void_p(stream)),
              "plato_partition_pagerank_init")

    def epoch(self, d_state: int, d_next: int, damping: float, final: bool, d_delta: int | None = None,
              stream: int = 0):
        check(self._lib.plato_partition_pagerank_epoch(self._h, C.c_void_p(d_state), C.c_void_p(d_next), damping,
                                                       1 if final else 0,
                                                       C.c_void_p(d_delta) if d_delta else None,
                                                       C.c_void_p(stream)), "plato_partition_pagerank_epoch")

    # ---- fused exchange over peer memory (plato_partition_p2p_*) ----------------
    def p2p_alloc(self) -> bytes:
        """Allocates the two state replicas and the flags; -> their 3 CUDA IPC handles."""
        h = C.create_string_buffer(3 * IPC_HANDLE_BYTES)
        check(self._lib.plato_partition_p2p_alloc(self._h, h), "plato_partition_p2p_alloc")
        return h.raw

    def p2p_connect(self, all_handles: bytes, timeout_ms: int = 0):
        """Maps the other partitions' replicas and flags (handles of every rank, rank order)."""
        check(self._lib.plato_partition_p2p_connect(self._h, C.c_char_p(all_handles), timeout_ms),
              "plato_partition_p2p_connect")

    def p2p_reset(self):
        check(self._lib.plato_partition_p2p_reset(self._h), "plato_partition_p2p_reset")

    def p2p_init(self, iterations: int, damping: float, eps: float = 0.0, stream: int = 0):
        check(self._lib.plato_partition_p2p_init(self._h, iterations, damping, eps, C.c_void_p(stream)),
              "plato_partition_p2p_init")

    def p2p_epoch(self, epoch: int, damping: float, stream: int = 0):
        check(self._lib.plato_partition_p2p_epoch(self._h, epoch, damping, C.c_void_p(stream)),
              "plato_partition_p2p_epoch")

    def p2p_state(self, stream: int = 0):
        """Waits for every partition's last epoch; -> (device pointer of the
        replica with the ranks (world * rows float32), epochs run)."""
        ptr, ep = C.c_void_p(), C.c_uint32()
        check(self._lib.plato_partition_p2p_state(self._h, C.c_void_p(stream), C.byref(ptr), C.byref(ep)),
              "plato_partition_p2p_state")
        return int(ptr.value), int(ep.value)

    def p2p_ranks(self, stream: int = 0):
        """p2p_state, then -> (ranks in caller ids float32 [V], epochs run)."""
        out = np.empty(self.vertices, np.float32)
        ep = C.c_uint32()
        check(self._lib.plato_partition_p2p_ranks(self._h, C.c_void_p(stream), C.c_void_p(out.ctypes.data),
                                                  C.byref(ep)), "plato_partition_p2p_ranks")
        return out, int(ep.value)

    def ranks(self, h_state: np.ndarray) -> np.ndarray:
        """Caller-id ranks from the assembled state (host float32 [world * rows])."""
        st = np.ascontiguousarray(h_state, dtype=np.float32)
        out = np.empty(self.vertices, np.float32)
        check(self._lib.plato_partition_ranks(self._h, C.c_void_p(st.ctypes.data), C.c_void_p(out.ctypes.data)),
              "plato_partition_ranks")
        return out


def _epochs(step, iterations: int, eps: float, delta_of):
    """The epoch schedule of pagerank.hpp:100-146: `step(final)` runs one
    epoch; with eps > 0 a non-final epoch whose delta (reference units) is
    below eps makes the next epoch the final one."""
    epoch, ran = 0, 0
    while epoch < iterations:
        final = epoch == iterations - 1
        step(final)
        ran += 1
        if not final and eps > 0.0 and delta_of() < eps:
            epoch = iterations - 2
        epoch += 1
    return ran


def pagerank_partitioned(vertices: int, src, dst, iterations: int = 100, damping: float = 0.85,
                         eps: float = 0.0, is_directed: bool = True, group=None):
    """PageRank over the processes of `group` (torch.distributed, default
    group), one partition per process on its current GPU -> (caller-id ranks
    float32 [V], epochs).  Every process passes the same edge list."""
    import torch
    import torch.distributed as dist

    rank, world = dist.get_rank(group), dist.get_world_size(group)
    part = Partition(vertices, src, dst, rank, world, is_directed)
    try:
        n = part.rows
        x = torch.empty(world * n, dtype=torch.float32, device="cuda")
        xn = torch.empty_like(x)
        delta = torch.zeros(1, dtype=torch.float64, device="cuda")
        stream = torch.cuda.current_stream().cuda_stream
        part.init(x.data_ptr(), damping, stream)
        dist.all_gather_into_tensor(x, x[rank * n:(rank + 1) * n], group=group)
        bufs = [x, xn]

        def step(final):
            cur, nxt = bufs
            part.epoch(cur.data_ptr(), nxt.data_ptr(), damping, final, delta.data_ptr() if eps > 0 else None, stream)
            dist.all_gather_into_tensor(nxt, nxt[rank * n:(rank + 1) * n], group=group)
            bufs.reverse()

        def delta_of():
            d = delta.clone()
            dist.all_reduce(d, group=group)
            return float(d.item()) * vertices

        ran = _epochs(step, iterations, eps, delta_of)
        return part.ranks(bufs[0].cpu().numpy()), ran
    finally:
        part.close()


def emulate_partitions(vertices: int, src, dst, world: int, iterations: int = 100, damping: float = 0.85,
                       eps: float = 0.0, is_directed: bool = True):
    """The partitioned PageRank with `world` partitions on the current GPU in
    one process -> (caller-id ranks float32 [V], epochs)."""
    import torch

    parts = [Partition(vertices, src, dst, r, world, is_directed) for r in range(world)]
    try:
        n = parts[0].rows
        x = torch.empty(world * n, dtype=torch.float32, device="cuda")
        xn = torch.empty_like(x)
        deltas = torch.zeros(world, dtype=torch.float64, device="cuda")
        stream = torch.cuda.current_stream().cuda_stream
        for p in parts:
            p.init(x.data_ptr(), damping, stream)
        bufs = [x, xn]

        def step(final):
            cur, nxt = bufs
            for r, p in enumerate(parts):
                p.epoch(cur.data_ptr(), nxt.data_ptr(), damping, final,
                        deltas[r:].data_ptr() if eps > 0 else None, stream)
            bufs.reverse()

        def delta_of():
            return float(deltas.sum().item()) * vertices

        ran = _epochs(step, iterations, eps, delta_of)
        return parts[0].ranks(bufs[0].cpu().numpy()), ran
    finally:
        for p in parts:
            p.close()


def pagerank_partitioned_p2p(vertices: int, src, dst, iterations: int = 100, damping: float = 0.85,
                             eps: float = 0.0, is_directed: bool = True, group=None, timeout_ms: int = 0):
    """The partitioned PageRank with the fused exchange over peer memory: one
    partition per process of `group` on its current GPU, CUDA IPC handles
    exchanged once over torch.distributed, then the epochs with no collective
    (the eps exit, if any, decided on every GPU from the published deltas)
    -> (caller-id ranks float32 [V], epochs)."""
    import torch
    import torch.distributed as dist

    rank, world = dist.get_rank(group), dist.get_world_size(group)
    part = Partition(vertices, src, dst, rank, world, is_directed)
    try:
        handles = [None] * world
        dist.all_gather_object(handles, part.p2p_alloc(), group=group)  # flags are zero before anyone maps them
        part.p2p_connect(b"".join(handles), timeout_ms)
        stream = torch.cuda.current_stream().cuda_stream
        dist.barrier(group=group)  # every partition mapped before any init publishes
        part.p2p_init(iterations, damping, eps, stream)
        for e in range(iterations):
            part.p2p_epoch(e, damping, stream)
        ranks, ran = part.p2p_ranks(stream)
        dist.barrier(group=group)  # no partition frees its replicas while a peer may still store into them
        return ranks, ran
    finally:
        part.close()


def emulate_partitions_p2p(vertices: int, src, dst, world: int, iterations: int = 100, damping: float = 0.85,
                           eps: float = 0.0, is_directed: bool = True, timeout_ms: int = 0):
    """The fused exchange with `world` partitions in one process on the
    current GPU: each epoch runs for every partition before the next epoch,
    so every wait is already satisfied when it runs -> (caller-id ranks
    float32 [V], epochs)."""
    import torch

    parts = [Partition(vertices, src, dst, r, world, is_directed) for r in range(world)]
    try:
        arr = (C.c_void_p * world)(*[p._h.value for p in parts])
        check(load().plato_partition_p2p_connect_local(arr, world, timeout_ms), "plato_partition_p2p_connect_local")
        stream = torch.cuda.current_stream().cuda_stream
        for p in parts:
            p.p2p_reset()
        for p in parts:
            p.p2p_init(iterations, damping, eps, stream)
        for e in range(iterations):
            for p in parts:
                p.p2p_epoch(e, damping, stream)
        return parts[0].p2p_ranks(stream)
    finally:
        for p in parts:
            p.close()
