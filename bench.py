#!/usr/bin/env python
"""Benchmark: PageRank GTEPS on RMAT scale 24 (one B200 per process).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl plato|reference]

Workload (one "step"): PageRank pull, 20 iterations, d = 0.85, on a seeded
RMAT graph, scale 24, edgefactor 16, seed 3 (a,b,c,d = .57,.19,.19,.05),
duplicates and self-loops removed, ids compacted; FP32 ranks with FP32
accumulation.  The graph (CSC+CSR, ~2.2 GB) is resident in HBM and larger
than L2, so no L2 flush is needed between steps.

Metric: GTEPS = stored edges x iterations / step time.  `value` times the
device-output entry point (plato_pagerank_device) with the graph resident;
`e2e` times the host-buffer C-ABI call plato_pagerank (ranks copied back to
pinned host memory every step).  Multi-GPU runs are independent replicas
(weak scaling, no collective on the data path).

--impl reference times the CPU restatement of the reference engine (the
oracle, C/OpenMP on all host threads) on the same graph: each step is one
PageRank epoch (pull + vertex update) in the reference's double precision.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

SCALE, EDGEFACTOR, SEED = 24, 16, 3
ITERATIONS, DAMPING = 20, 0.85
METRIC = "PageRank GTEPS (RMAT s24 ef16, 20 iterations, pull)"
PULL_KERNEL = "k_pull_warp"  # dominant kernel of a PageRank step


def env_rank():
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.rows = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.Q}",
                                      "--format=csv,noheader,nounits"], capture_output=True,
                                     text=True, timeout=5).stdout.strip()
                if out:
                    self.rows.append([c.strip() for c in out.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *exc):
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in self.rows for n, v in zip(names, r[5:9]) if v == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.rows)}


def measured_peak():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def pr_algorithmic_bytes(V: int, E: int) -> int:
    """Bytes one pull epoch must move: column ids 4E + gathered ranks 4E +
    offsets 8(V+1) + x_old 4V + degree 4V + x_new 4V."""
    return 8 * E + 8 * (V + 1) + 12 * V


def cpu_pagerank_sample(V, src, dst, target_s=15.0):
    """Oracle (reference restatement) PageRank epochs on all host threads,
    sized to ~target_s seconds; returns (GTEPS, epochs, seconds, threads, E)."""
    import oracle
    g = oracle.RefGraph(V, src, dst, True)
    E = g.stored_edges
    t0 = time.perf_counter()
    g.pagerank(1, DAMPING, 0.0)
    t1 = time.perf_counter() - t0
    n = int(max(1, min(20, target_s / max(t1, 1e-3))))
    t0 = time.perf_counter()
    g.pagerank(n, DAMPING, 0.0)
    dt = time.perf_counter() - t0
    thr = oracle.max_threads()
    g.close()
    return E * n / dt / 1e9, n, dt, thr, E


def run_reference(args):
    rank, world, _ = env_rank()
    if rank != 0:
        return 0
    import oracle
    import plato_b200 as pb
    V, src, dst = pb.rmat(SCALE, EDGEFACTOR, SEED)
    g = oracle.RefGraph(V, src, dst, True)
    E = g.stored_edges
    for _ in range(args.warmup):
        g.pagerank(1, DAMPING, 0.0)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        g.pagerank(1, DAMPING, 0.0)
        times.append(time.perf_counter() - t0)
    ms = float(np.mean(times)) * 1e3
    val = E / (ms / 1e3) / 1e9
    thr = oracle.max_threads()
    line = {
        "impl": "reference", "metric": METRIC, "value": val, "unit": "GTEPS", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"pagerank_rmat_s{SCALE}_ef{EDGEFACTOR}_seed{SEED}",
                   "vertices": V, "edges": E, "step": "one PageRank epoch (pull + update)"},
        "cpu_baseline": {"value": val, "unit": "GTEPS", "cores": thr, "kind": "port",
                         "sample": f"{args.steps} PageRank epochs of the s{SCALE} graph "
                                   "(oracle ref_cpu.c, reference restatement, OpenMP)"},
        "e2e": {"value": val, "unit": "GTEPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_plato(args):
    import torch

    rank, world, local = env_rank()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as tdist
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        dist = tdist
    import plato_b200 as pb
    from plato_b200 import _lib

    lib = _lib.load()
    t0 = time.perf_counter()
    V, src, dst = pb.rmat(SCALE, EDGEFACTOR, SEED)
    gen_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    g = pb.Graph(V, src, dst, is_directed=True, relabel=True)
    torch.cuda.synchronize()
    build_s = time.perf_counter() - t0
    E = int(g.device_view().stored_edges)
    stream = torch.cuda.current_stream()
    sptr = stream.cuda_stream
    d_out = torch.empty(V, dtype=torch.float32, device="cuda")

    def step():
        g.pagerank_device(d_out.data_ptr(), ITERATIONS, DAMPING, 0.0, stream=sptr)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()

    def barrier():
        if dist:
            dist.barrier()

    # ---- device-resident timed region --------------------------------------
    lib.plato_profile_reset()
    lib.plato_profile_enable(1)
    launches0 = pb.kernel_launches()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        ev0.record(stream)
        for _ in range(args.steps):
            step()
        ev1.record(stream)
        torch.cuda.synchronize()
    barrier()
    launches = pb.kernel_launches() - launches0
    lib.plato_profile_enable(0)
    import ctypes as C
    tot = C.c_double()
    cnt = C.c_uint64()
    lib.plato_profile_read(PULL_KERNEL.encode(), C.byref(tot), C.byref(cnt))
    merge_ms, merge_n = tot.value, int(cnt.value)
    lib.plato_profile_read((PULL_KERNEL + "_fixup").encode(), C.byref(tot), C.byref(cnt))
    fix_ms = tot.value
    ms = ev0.elapsed_time(ev1) / args.steps
    if dist:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    value = world * E * ITERATIONS / (ms / 1e3) / 1e9

    # ---- end to end through the host-buffer C ABI ----------------------------
    host_out = torch.empty(V, dtype=torch.float32, pin_memory=True)
    opts = _lib.PagerankOpts(ITERATIONS, DAMPING, 0.0)
    st = _lib.RunStats()

    def e2e_step():
        _lib.check(lib.plato_pagerank(g.handle, C.byref(opts), C.c_void_p(host_out.data_ptr()),
                                      C.byref(st)), "plato_pagerank")

    for _ in range(2):
        e2e_step()
    barrier()
    t0 = time.perf_counter()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        e2e_step()
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = (time.perf_counter() - t0) * 1e3 / args.steps
    if dist:
        t = torch.tensor([e2e_ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())
    e2e_val = world * E * ITERATIONS / (e2e_ms / 1e3) / 1e9

    # ---- roofline of the dominant kernel -------------------------------------
    peak, peak_kind = measured_peak()
    bytes_per_launch = pr_algorithmic_bytes(V, E)
    per_launch_ms = merge_ms / max(merge_n, 1)
    achieved = bytes_per_launch / (per_launch_ms / 1e3) / 1e9
    roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "traffic": None, "kernel": PULL_KERNEL,
            "peak_source": f"{peak_kind} hbm_gbs (burst copy)",
            "bytes_per_launch": bytes_per_launch, "launch_ms": per_launch_ms,
            "fixup_ms_per_launch": fix_ms / max(merge_n, 1)}
    prof = ROOT / "profiles" / "k_pull_warp_rmat_s24_traffic.json"
    if prof.exists():
        tr = json.loads(prof.read_text())
        roof["traffic"] = tr.get("dram_bytes_per_launch_full")

    line = {
        "metric": METRIC, "value": value, "unit": "GTEPS", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"pagerank_rmat_s{SCALE}_ef{EDGEFACTOR}_seed{SEED}",
                   "vertices": V, "edges": E, "iterations": ITERATIONS, "damping": DAMPING,
                   "parallelism": f"replicas{world}", "l2": "inputs larger than L2 (2.2 GB graph)",
                   "graph_build_s": build_s, "rmat_gen_s": gen_s},
        "e2e": {"value": e2e_val, "unit": "GTEPS", "h2d_bytes_per_step": C.sizeof(opts),
                "d2h_bytes_per_step": 4 * V, "ms_per_step": e2e_ms,
                "note": "host-buffer plato_pagerank; graph resident in HBM"},
        "gpu_launches": launches,
        "roofline": roof,
        "clocks": clk.summary(),
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        gteps, n, dt, thr, _ = cpu_pagerank_sample(V, src, dst)
        line["cpu_baseline"] = {"value": gteps, "unit": "GTEPS", "cores": thr, "kind": "port",
                                "sample": f"{n} PageRank epochs on the same s{SCALE} graph "
                                          f"({dt:.1f} s, oracle ref_cpu.c, FP64, OpenMP)"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    g.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["plato", "reference"], default="plato")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--scale", type=int, default=SCALE,
                    help="RMAT scale (smaller values are for profiling captures only)")
    args = ap.parse_args()
    globals()["SCALE"] = args.scale
    if args.impl == "reference":
        return run_reference(args)
    return run_plato(args)


if __name__ == "__main__":
    sys.exit(main())
