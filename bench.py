#!/usr/bin/env python
"""Benchmark: PageRank GTEPS on RMAT scale 24, plus batched-PPR and serving
queries/s (one B200 per process).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl plato|reference]

Workload (one "step"): PageRank pull, 20 iterations, d = 0.85, on a seeded
RMAT graph, scale 24, edgefactor 16, seed 3 (a,b,c,d = .57,.19,.19,.05),
duplicates and self-loops removed, ids compacted; FP32 ranks with FP32
accumulation.  The graph (CSC+CSR, ~2.2 GB) is resident in HBM and larger
than L2, so no L2 flush is needed between steps.

Metric: GTEPS = stored edges x iterations / step time.  `value` times the
device-output entry point (plato_pagerank_device) with the graph resident
and no instrumentation; per-kernel times for the roofline come from a
separate pass of the same steps.  `e2e` times the host-buffer C-ABI call
plato_pagerank (ranks copied back to pinned host memory every step).  At
N = 1 the same line carries `ppr_batch` (RMAT s22 seed 4, K = 64/256/1024
queries per call against the plain one-query engine) and `serving` (RMAT s24
seed 5, Poisson arrivals, p50/p99 latency).  Multi-GPU runs are independent
replicas (weak scaling, no collective on the data path).

--impl reference times the reference's CPU path on the host cores: its own
engine and algo::pagerank compiled from its headers (oracle/_ref, built
where the reference tree is present; else the oracle's C/OpenMP
restatement), in the reference's double precision, one 20-epoch call per
step on the same graph (built by the oracle's own RMAT generator, so no
product code is loaded).
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
# kernels of one pull epoch: the degree bins (relabelled graphs) or the merge path
PULL_KERNELS = ["k_pull_long", "k_pull_rows16", "k_pull_rows8", "k_pull_rows4", "k_pull_short",
                "k_pull_hubs", "k_pull_warp", "k_pull_warp_fixup"]


def env_rank():
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int, period_ms: int = 50):
        self.gpu = gpu_index
        self.period_ms = period_ms
        self.rows = []
        self._proc = None
        self._t = None

    def _read(self):
        for line in self._proc.stdout:
            line = line.strip()
            if line:
                self.rows.append([c.strip() for c in line.split(",")])

    def __enter__(self):
        # one nvidia-smi in loop mode (a sample every period_ms), stopped by its handle on exit
        try:
            self._proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.Q}",
                                           "--format=csv,noheader,nounits", "-lms", str(self.period_ms)],
                                          stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self._proc = None
            return self
        self._t = threading.Thread(target=self._read, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *exc):
        # no wait on either side: an idle GPU lowers its clocks, and a sample
        # taken then would not describe the timed region
        if self._proc:
            self._proc.terminate()
            try:
                self._proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self._proc.kill()
        if self._t:
            self._t.join(timeout=5)

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


def max_over_ranks(x: float, dist, device: str) -> float:
    """Slowest rank's value (replicas are timed independently; the job is as
    fast as its slowest replica).  `dist` is torch.distributed or None."""
    if dist is None:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_value(units_per_rank: float, ms: float, world: int) -> float:
    """Whole-job throughput of `world` replicas each processing
    `units_per_rank` units in `ms` (the max over ranks)."""
    return world * units_per_rank / (ms / 1e3)


def measured_peak():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def pr_algorithmic_bytes(V: int, E: int) -> int:
    """Bytes one pull epoch must move: column ids 4E + gathered ranks 4E +
    offsets 8(V+1) + x_old 4V + degree 4V + x_new 4V."""
    return 8 * E + 8 * (V + 1) + 12 * V


def pull_bins(V: int, dst) -> dict:
    """Per-kernel algorithmic bytes of one pull epoch on a graph relabelled by
    descending in-degree (the bins of pull_binned.cuh: long > 64, then
    33..64, 17..32 and 5..16 for k_pull_rows16/8/4, short <= 4): each bin
    moves 8 bytes per edge (id + gathered rank) and 20 bytes per row (offset,
    x_old, degree, x_new)."""
    indeg = np.sort(np.bincount(dst, minlength=V))[::-1].astype(np.int64)
    bounds = [("k_pull_long", 64, None), ("k_pull_rows16", 32, 64), ("k_pull_rows8", 16, 32),
              ("k_pull_rows4", 4, 16), ("k_pull_short", -1, 4)]
    out, rows, edges = {"k_pull_hubs": 0}, {}, {}
    for name, lo, hi in bounds:
        m = indeg > lo if hi is None else (indeg > lo) & (indeg <= hi)
        n, e = int(m.sum()), int(indeg[m].sum())
        out[name] = 8 * e + 20 * n
        rows[name], edges[name] = n, e
    out["rows"], out["edges"] = rows, edges
    return out


def cpu_pagerank_sample(V, src, dst, target_s=15.0):
    """Oracle (reference restatement) PageRank epochs on all host threads,
    sized to ~target_s seconds; returns (GTEPS, epochs, seconds, threads, E,
    FP64 ranks after ITERATIONS epochs in reference units)."""
    import oracle
    g = oracle.RefGraph(V, src, dst, True)
    E = g.stored_edges
    t0 = time.perf_counter()
    g.pagerank(1, DAMPING, 0.0)
    t1 = time.perf_counter() - t0
    n = int(max(1, min(ITERATIONS, target_s / max(t1, 1e-3))))
    t0 = time.perf_counter()
    ranks, _, _ = g.pagerank(n, DAMPING, 0.0)
    dt = time.perf_counter() - t0
    if n != ITERATIONS:
        ranks, _, _ = g.pagerank(ITERATIONS, DAMPING, 0.0)
    thr = oracle.max_threads()
    g.close()
    return E * n / dt / 1e9, n, dt, thr, E, ranks


def bench_config(V: int, E: int, world: int) -> dict:
    """The workload's config, identical in both arms."""
    return {"workload": f"pagerank_rmat_s{SCALE}_ef{EDGEFACTOR}_seed{SEED}", "vertices": V, "edges": E,
            "iterations": ITERATIONS, "damping": DAMPING, "parallelism": f"replicas{world}",
            "step": f"one {ITERATIONS}-epoch PageRank call (pull) on the resident graph",
            "l2": "inputs larger than L2 (2.2 GB graph)"}


def run_reference(args):
    """The reference's CPU path on the host cores, on the same graph as the
    GPU arm, one PageRank call per step.

    Where the reference was compiled here (oracle/_ref/libplato_ref.so: its
    own engine, message passing and algo::pagerank, plato/algo/pagerank/
    pagerank.hpp:60-149, with a one-rank in-process MPI), that is what runs
    ("kind": "reference"); each call allocates its states and derives the
    out-degrees as the reference's call does.  Otherwise the oracle's C/OpenMP
    restatement runs ("kind": "port").  A step is a 20-epoch call, fewer epochs
    only when 20 would not let the whole run finish within a few minutes.
    This process loads no product code: the graph comes from the oracle's own
    RMAT generator (oracle/rmat.c), which the CPU tests hold equal to the
    product's."""
    rank, world, _ = env_rank()
    if rank != 0:
        return 0
    import oracle
    from oracle import refplato
    t0 = time.perf_counter()
    V, src, dst = oracle.rmat(SCALE, EDGEFACTOR, SEED)
    gen_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    if refplato.available():
        kind, thr = "reference", refplato.threads()
        g = refplato.ReferenceGraph(V, src, dst, True)
        E = g.edges

        def call(epochs):
            g.pagerank(epochs, DAMPING, 0.0)
        what = ("the reference's own algo::pagerank (pagerank.hpp:60-149) and engine, compiled from its "
                "headers (oracle/_ref/libplato_ref.so, one-rank in-process MPI)")
    else:
        kind, thr = "port", oracle.max_threads()
        g = oracle.RefGraph(V, src, dst, True)
        E = g.stored_edges

        def call(epochs):
            g.pagerank(epochs, DAMPING, 0.0)
        what = "oracle ref_cpu.c, the reference's pull PageRank restated in C/OpenMP"
    build_s = time.perf_counter() - t0
    del src, dst
    # first warm-up call at full length; it sizes the rest of the run
    t0 = time.perf_counter()
    call(ITERATIONS)
    t_full = time.perf_counter() - t0
    budget_s = 150.0
    epochs = ITERATIONS
    if (args.steps + args.warmup) * t_full > budget_s:
        epochs = max(2, int(ITERATIONS * budget_s / ((args.steps + args.warmup) * t_full)))
    for _ in range(max(0, args.warmup - 1)):
        call(epochs)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        call(epochs)
        times.append(time.perf_counter() - t0)
    g.close()
    ms = float(np.mean(times)) * 1e3
    val = E * epochs / (ms / 1e3) / 1e9
    line = {
        "impl": "reference", "metric": METRIC, "value": val, "unit": "GTEPS", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": bench_config(V, E, world),
        "setup": {"rmat_gen_s": gen_s, "graph_build_s": build_s, "first_call_s": t_full,
                  "generator": "oracle/rmat.c (equal to the product's, CPU tests)"},
        "cpu_baseline": {"value": val, "unit": "GTEPS", "cores": thr, "kind": kind,
                         "sample": f"{args.steps} timed calls of {epochs} PageRank epochs each on the whole "
                                   f"s{SCALE} graph ({what}, FP64, host clock)"},
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

    # ---- device-resident timed region (no instrumentation) -------------------
    lib.plato_profile_enable(0)
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
    ms = max_over_ranks(ev0.elapsed_time(ev1) / args.steps, dist, "cuda")
    value = world * E * ITERATIONS / (ms / 1e3) / 1e9

    # ---- per-kernel device times: a separate pass of the same steps ----------
    import ctypes as C
    prof_steps = max(1, min(args.steps, 5))
    lib.plato_profile_reset()
    lib.plato_profile_enable(1)
    for _ in range(prof_steps):
        step()
    torch.cuda.synchronize()
    lib.plato_profile_enable(0)
    kernel_times = {}
    for name in PULL_KERNELS:
        tot = C.c_double()
        cnt = C.c_uint64()
        lib.plato_profile_read(name.encode(), C.byref(tot), C.byref(cnt))
        if cnt.value:
            kernel_times[name] = (tot.value, int(cnt.value))

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
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        e2e_step()
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks((time.perf_counter() - t0) * 1e3 / args.steps, dist, "cuda")
    e2e_val = world * E * ITERATIONS / (e2e_ms / 1e3) / 1e9

    # ---- roofline of the dominant kernel -------------------------------------
    peak, peak_kind = measured_peak()
    epoch_bytes = pr_algorithmic_bytes(V, E)
    bins = pull_bins(V, dst)
    epochs = ITERATIONS * prof_steps
    per = {}
    for name, (tot_ms, n) in kernel_times.items():
        per[name] = {"launches": n, "ms_per_launch": tot_ms / n}
        b = bins.get(name)
        if b:
            per[name]["bytes_per_launch"] = b
            per[name]["achieved_gbs"] = b / (tot_ms / n / 1e3) / 1e9
    epoch_ms = sum(t for t, _ in kernel_times.values()) / max(epochs, 1)
    tot_k = sum(t for t, _ in kernel_times.values()) or 1.0
    for name, (tot_ms, _) in kernel_times.items():
        per[name]["share"] = tot_ms / tot_k
    dom = max(kernel_times, key=lambda k: kernel_times[k][0]) if kernel_times else PULL_KERNELS[0]
    if dom in bins and dom in per:
        dom_bytes = bins[dom]
        dom_ms = per[dom]["ms_per_launch"]
    else:  # merge-path kernel: it is the whole epoch
        dom_bytes = epoch_bytes
        dom_ms = per.get(dom, {"ms_per_launch": epoch_ms})["ms_per_launch"]
    achieved = dom_bytes / (dom_ms / 1e3) / 1e9
    roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "traffic": None, "kernel": dom,
            "peak_source": f"{peak_kind} hbm_gbs (burst copy, of {peak_kind})",
            "bytes_per_launch": dom_bytes, "launch_ms": dom_ms,
            "kernel_timing": f"CUDA events around each pull kernel on its launch stream, in a separate "
                             f"pass of {prof_steps} steps right after the timed region",
            "pull_epoch": {"bytes": epoch_bytes, "ms": epoch_ms,
                           "achieved": epoch_bytes / (epoch_ms / 1e3) / 1e9 if epoch_ms else None,
                           "frac": (epoch_bytes / (epoch_ms / 1e3) / 1e9 / peak) if epoch_ms else None,
                           "step_frac": epoch_bytes * ITERATIONS / (ms / 1e3) / 1e9 / peak},
            "kernels": per, "bins": {"rows": bins["rows"], "edges": bins["edges"]}}
    prof = ROOT / "profiles" / f"{dom}_rmat_s{SCALE}_traffic.json"
    if prof.exists():
        tr = json.loads(prof.read_text())
        roof["traffic"] = tr.get("dram_bytes_per_launch")
        roof["traffic_source"] = (f"profiles/{prof.name}: one ncu capture of this kernel on this workload, "
                                  "not measured in this run")

    line = {
        "metric": METRIC, "value": value, "unit": "GTEPS", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": bench_config(V, E, world),
        "setup": {"graph_build_s": build_s, "rmat_gen_s": gen_s},
        "e2e": {"value": e2e_val, "unit": "GTEPS", "h2d_bytes_per_step": C.sizeof(opts),
                "d2h_bytes_per_step": 4 * V, "ms_per_step": e2e_ms,
                "note": "host-buffer plato_pagerank (ranks copied to pinned host memory every call; "
                        "graph resident in HBM), host clock"},
        "gpu_launches": launches,
        "roofline": roof,
        "clocks": clk.summary(),
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        gteps, n, dt, thr, _, want = cpu_pagerank_sample(V, src, dst)
        line["cpu_baseline"] = {"value": gteps, "unit": "GTEPS", "cores": thr, "kind": "port",
                                "sample": f"{n} PageRank epochs on the same s{SCALE} graph "
                                          f"({dt:.1f} s, oracle ref_cpu.c, FP64, OpenMP)"}
        err = np.abs(host_out.numpy().astype(np.float64) - want / V)
        line["parity"] = {"vs": f"oracle ref_cpu.c FP64, {ITERATIONS} epochs, reference ranks / V",
                          "l1": float(err.sum()), "max_abs": float(err.max()), "tolerance_l1": 1e-6,
                          "ok": bool(err.sum() <= 1e-6)}
    g.close()
    del src, dst
    if world == 1 and not args.no_extras:
        # the metric's second half: batched PPR (s22 seed 4) and serving (s24 seed 5)
        line["ppr_batch"] = bench_ppr_batch(pb)
        line["serving"] = bench_serving(pb)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def bench_ppr_batch(pb, plain_n=16, reps=3):
    """Batched multi-source PPR on RMAT s22 ef16 seed 4: K in 64/256/1024
    queries per call, Zipf(1.5) seed sets of 1..32 vertices, eps 1e-6,
    top-100 per query, against the plain engine (plato_seedset_ppr) answering
    the same queries one at a time.  Host clock around whole calls, seed sets
    from and top-k results to host memory."""
    import oracle
    t_all = time.perf_counter()
    V, s, d = pb.rmat(22, 16, 4)
    g = pb.Graph(V, s, d, is_directed=True)
    deg = np.bincount(s, minlength=V)
    sets = zipf_seed_sets(deg, 1024, 32, 4)
    plain_qps, plain_qps_numpy, plain = plain_engine_qps(g, sets, plain_n, collect=True)
    res = {"workload": "ppr_batch_rmat_s22_ef16_seed4", "vertices": V, "edges": int(s.size),
           "unit": "queries/s", "eps": 1e-6, "topk": 100,
           "plain_qps": plain_qps, "plain_qps_fresh_numpy_output": plain_qps_numpy,
           "plain_sample": f"queries 0..{plain_n - 1}, one plato_seedset_ppr call each, ranks into one "
                           "reused pinned host buffer (the speed-ups are against this rate)",
           "timing": f"host clock around whole plato_ppr_batch calls (seed sets in, top-100 out), median of {reps}"}
    for K in (64, 256, 1024):
        g.ppr_batch(sets[:K], 300, 0.85, 1e-6, topk=100)  # autotune + warm
        dts = []
        for _ in range(reps):
            t0 = time.perf_counter()
            out = g.ppr_batch(sets[:K], 300, 0.85, 1e-6, topk=100)
            dts.append(time.perf_counter() - t0)
        dt = float(np.median(dts))
        res[f"K{K}"] = {"qps": K / dt, "ms_per_batch": dt * 1e3, "speedup_vs_plain": K / dt / plain_qps,
                        "iterations_max": int(out["iterations"].max()), "k_tile": g.ppr_batch_k_tile(K)}
    # sampled columns: batch column vs the plain engine, and column 0 vs the FP64 oracle
    chk = g.ppr_batch(sets[:plain_n], 300, 0.85, 1e-6, ranks=True)
    res["l1_batch_vs_plain_max"] = max(float(np.abs(chk["ranks"][q].astype(np.float64) - plain[q]).sum())
                                       for q in range(plain_n))
    g.close()
    # every sampled column against the FP64 oracle (queries 0..3 of the batch)
    ref = oracle.RefGraph(V, s, d, True)
    cols = []
    for q in range(4):
        want, ep, _ = ref.seedset_ppr(sets[q], 300, 0.85, 1e-6)
        err = np.abs(chk["ranks"][q].astype(np.float64) - want)
        cols.append({"query": q, "l1": float(err.sum()), "max_abs": float(err.max()),
                     "epochs": int(chk["iterations"][q]), "oracle_epochs": ep})
    ref.close()
    res["parity"] = {"vs": "oracle ref_cpu.c FP64", "tolerance_l1": 1e-6, "columns": cols,
                     "l1_max": max(c["l1"] for c in cols), "max_abs": max(c["max_abs"] for c in cols),
                     "ok": all(c["l1"] <= 1e-6 and abs(c["epochs"] - c["oracle_epochs"]) <= 1 for c in cols)}
    res["wall_s"] = time.perf_counter() - t_all
    return res


def bench_serving(pb, rates=(100, 1000, 5000, 20000), slots=256):
    """PPR serving on RMAT s24 ef16 seed 5: Poisson arrivals at each offered
    rate, Zipf(1.5) seed sets of 1..64, eps 1e-6, top-100; latency =
    completion - arrival on the host clock; against the plain engine serving
    one query at a time.  Requests per rate: 5 s of arrivals, at least 300 and
    at most 4 x slots (four generations of the slots when saturated)."""
    t_all = time.perf_counter()
    V, s, d = pb.rmat(24, 16, 5)
    g = pb.Graph(V, s, d, is_directed=True)
    deg = np.bincount(s, minlength=V)
    src_dst = (s, d)
    del s, d

    def n_for(rate):
        return min(4 * slots, max(300, 5 * rate))

    sets = zipf_seed_sets(deg, max(n_for(r) for r in rates), 64, 5)
    plain_n = 16
    plain_qps, plain_qps_numpy, _ = plain_engine_qps(g, sets, plain_n)
    out = {"workload": "ppr_serving_rmat_s24_ef16_seed5", "vertices": V, "unit": "queries/s",
           "slots": slots, "plain_qps": plain_qps, "plain_qps_fresh_numpy_output": plain_qps_numpy,
           "plain_sample": f"queries 0..{plain_n - 1}, one plato_seedset_ppr call each, ranks into one "
                           "reused pinned host buffer (the speed-ups are against this rate)",
           "timing": "host clock: latency = completion - arrival; sustained = requests / wall of the whole "
                     "run; steady = the middle completions (the first and last min(slots, n/4) dropped) over "
                     "the time they took"}
    out.update(_serve(pb, g, sets, rates, n_for, slots))
    out["parity"] = _serving_parity(pb, g, V, src_dst, sets[:2], slots)
    runs = [v for k, v in out.items() if k.startswith("rate")]
    out["best_sustained_qps"] = max(v["sustained_qps"] for v in runs)
    out["speedup_vs_plain_whole_run"] = out["best_sustained_qps"] / plain_qps
    steady = [v["steady"]["qps"] for v in runs if v["steady"]["qps"]]
    out["best_steady_qps"] = max(steady) if steady else None
    out["speedup_vs_plain"] = (out["best_steady_qps"] / plain_qps) if steady else None
    g.close()
    out["wall_s"] = time.perf_counter() - t_all
    return out


def _serving_parity(pb, g, V, src_dst, sets, slots, topk=100):
    """Requests served by a fresh server, their top-k against the FP64 oracle:
    the values at the returned ids, and the k-th value against the oracle's
    k-th largest rank."""
    import oracle
    got = {}
    with pb.PPRServer(g, max_slots=slots, hbm_budget_bytes=64 << 30, max_iterations=300,
                      eps=1e-6, topk=topk) as srv:
        ids = {srv.submit(q): i for i, q in enumerate(sets)}
        while len(got) < len(sets):
            srv.step()
            while (r := srv.poll()) is not None:
                got[ids[r[0]]] = r
    ref = oracle.RefGraph(V, src_dst[0], src_dst[1], True)
    out = []
    for i, q in enumerate(sets):
        want, ep, _ = ref.seedset_ppr(q, 300, 0.85, 1e-6)
        _, t_ids, t_vals, it = got[i]
        err = np.abs(t_vals.astype(np.float64) - want[t_ids])
        kth = float(np.partition(want, V - topk)[V - topk])
        out.append({"request": i, "topk_l1": float(err.sum()), "topk_max_abs": float(err.max()),
                    "kth_value": float(t_vals[-1]), "oracle_kth_value": kth,
                    "iterations": int(it), "oracle_epochs": ep})
    ref.close()
    return {"vs": "oracle ref_cpu.c FP64 (full ranks; compared on the returned top-100)", "requests": out,
            "ok": all(o["topk_max_abs"] <= 1e-6 and abs(o["kth_value"] - o["oracle_kth_value"]) <= 1e-6
                      and abs(o["iterations"] - o["oracle_epochs"]) <= 1 for o in out)}


def plain_engine_qps(g, sets, n, collect=False):
    """The plain engine answering queries 0..n-1 one at a time: plato_seedset_ppr
    (pull-only, eps 1e-6) through the C ABI, the full rank vector copied to one
    pinned host buffer reused by every call (as a serving loop would keep it).
    -> (queries/s, queries/s with a fresh pageable numpy array per call (the
    Python wrapper's default), and with collect the n rank vectors, taken in
    an untimed second pass)."""
    import ctypes as C

    import torch
    from plato_b200 import _lib
    lib = _lib.load()
    V = g.vertices
    pinned = torch.empty(V, dtype=torch.float32, pin_memory=True)
    opts = _lib.PprOpts(300, 0.85, 0, 1e-6)
    st = _lib.RunStats()
    seeds = [np.ascontiguousarray(q, dtype=np.uint32) for q in sets[:n]]

    def one(q):
        _lib.check(lib.plato_seedset_ppr(g.handle, C.c_void_p(q.ctypes.data), q.size, C.byref(opts),
                                         C.c_void_p(pinned.data_ptr()), C.byref(st)), "plato_seedset_ppr")

    one(seeds[0])  # warm
    t0 = time.perf_counter()
    for q in seeds:
        one(q)
    qps = n / (time.perf_counter() - t0)
    ranks = []
    if collect:  # the answers themselves, untimed
        for q in seeds:
            one(q)
            ranks.append(pinned.numpy().copy())
    g.seedset_ppr(sets[0], 300, 0.85, 1e-6)
    t0 = time.perf_counter()
    for q in sets[:n]:
        g.seedset_ppr(q, 300, 0.85, 1e-6)
    qps_numpy = n / (time.perf_counter() - t0)
    return qps, qps_numpy, ranks


def zipf_seed_sets(deg, K, max_size, seed):
    """Seed-set sizes Zipf(s=1.5) clipped to [1, max_size], members uniform among deg > 0."""
    rng = np.random.default_rng(seed)
    cands = np.flatnonzero(deg > 0)
    sizes = np.minimum(rng.zipf(1.5, K), max_size)
    return [rng.choice(cands, int(n), replace=False).astype(np.uint32) for n in sizes]


def suite_bfs(pb, roots_n=64):
    """BFS on RMAT s22 ef16 symmetrised, seed 2: Graph500-style GTEPS (undirected
    edges in the traversed component / time), harmonic mean over the roots."""
    V, s, d = pb.rmat(22, 16, 2, symmetrize=True)
    g = pb.Graph(V, s, d, is_directed=False)
    deg = np.bincount(s, minlength=V) + np.bincount(d, minlength=V)
    rng = np.random.default_rng(2)
    roots = rng.choice(np.flatnonzero(deg > 0), roots_n, replace=False)
    g.bfs(int(roots[0]), parents=False, levels=False)
    teps, times, modes, kept = [], [], [], []
    for r in roots:
        lev, _, st = g.bfs(int(r), parents=False)
        if len(kept) < 4:
            kept.append(lev)
        m = int(deg[lev != pb.PLATO_LEVEL_UNREACHED].sum()) // 2
        t0 = time.perf_counter()
        _, _, st = g.bfs(int(r), parents=False, levels=False)
        dt = time.perf_counter() - t0
        teps.append(m / dt)
        times.append(dt)
        modes.append("".join("P" if x == "push" else "l" for x in st.mode_trace))
    g.close()
    hm = len(teps) / sum(1.0 / t for t in teps)
    return {"workload": "bfs_rmat_s22_ef16_seed2_sym", "vertices": V, "undirected_edges": int(s.size),
            "roots": roots_n, "gteps_harmonic_mean": hm / 1e9,
            "ms_median": float(np.median(times)) * 1e3, "mode_trace_example": modes[0],
            "timing": "host clock around plato_bfs (levels not copied back)",
            "cpu_baseline": cpu_bfs_sample(V, s, d, roots[:len(kept)], deg, kept)}


def cpu_bfs_sample(V, s, d, roots, deg, gpu_levels):
    """The oracle's C/OpenMP BFS (the reference's dual-mode rules) on the host
    cores, for a few of the same roots: harmonic-mean GTEPS, and whether the
    GPU's levels for those roots equal the oracle's bit for bit."""
    import oracle
    ref = oracle.RefGraph(V, s, d, False)
    teps, same = [], []
    for r, mine in zip(roots, gpu_levels):
        t0 = time.perf_counter()
        lev, _, _, _, _ = ref.bfs(int(r), 0.05)
        dt = time.perf_counter() - t0
        teps.append(int(deg[lev != 0xFFFFFFFF].sum()) // 2 / dt)
        same.append(bool(np.array_equal(lev, mine)))
    ref.close()
    return {"gteps_harmonic_mean": len(teps) / sum(1.0 / t for t in teps) / 1e9, "cores": oracle.max_threads(),
            "kind": "port", "sample": f"{len(roots)} of the same roots, oracle ref_cpu.c",
            "levels_bit_exact": all(same)}


def suite_cc(pb):
    """Connected components (label propagation on the dual-mode engine) on the
    BFS graph: RMAT s22 ef16 seed 2 symmetrised."""
    V, s, d = pb.rmat(22, 16, 2, symmetrize=True)
    g = pb.Graph(V, s, d, is_directed=False)
    g.connected_components(labels=False)
    times = []
    for _ in range(5):
        t0 = time.perf_counter()
        _, summ, st = g.connected_components(labels=False)
        times.append(time.perf_counter() - t0)
    g.close()
    ms = float(np.median(times)) * 1e3
    return {"workload": "cc_rmat_s22_ef16_seed2_sym", "vertices": V, "undirected_edges": int(s.size),
            "ms_median": ms, "epochs": st.iterations, "push_epochs": st.push_iterations,
            "gteps": 2 * s.size * st.iterations / (ms / 1e3) / 1e9, "summary": summ,
            "timing": "host clock around plato_connected_components (labels not copied back), median of 5"}


def _profiled(pb, names, fn):
    """Runs fn() with the library's kernel timing on; returns {name: (ms, launches)}."""
    import ctypes as C
    lib = pb.load()
    lib.plato_profile_reset()
    lib.plato_profile_enable(1)
    fn()
    lib.plato_profile_enable(0)
    out = {}
    for name in names:
        tot, cnt = C.c_double(), C.c_uint64()
        lib.plato_profile_read(name.encode(), C.byref(tot), C.byref(cnt))
        out[name] = (tot.value, int(cnt.value))
    return out


HLL_KERNELS = ("k_hll_rows", "k_hll_hubs", "k_hll_spread")


def suite_hll(pb, bits=6):
    """HyperANF and n-step degrees (HyperLogLog propagation) on the BFS graph,
    RMAT s22 ef16 seed 2 symmetrised, P = 6 (the CLIs' default width).

    Roofline of one full epoch (every row active, iteration = 1): algorithmic
    bytes = E*m (a source row per stored edge) + 4E (ids) + 2*V*m (own row
    read, new row written) + 16V (offsets), over the gather kernels' device
    time; E = stored directed edges, m = 2^P."""
    V, s, d = pb.rmat(22, 16, 2, symmetrize=True)
    g = pb.Graph(V, s, d, is_directed=False)
    E = 2 * int(s.size)
    m = 1 << bits
    out = {"workload": "hll_rmat_s22_ef16_seed2_sym", "vertices": V, "stored_edges": E, "bits": bits}
    g.hyperanf(1, bits)
    kt = _profiled(pb, HLL_KERNELS, lambda: g.hyperanf(1, bits))
    dev_ms = kt["k_hll_rows"][0] + kt["k_hll_hubs"][0]
    alg = E * m + 4 * E + 2 * V * m + 16 * V
    peak, peak_kind = measured_peak()
    out["full_epoch"] = {"kernel_ms": dev_ms, "rows_ms": kt["k_hll_rows"][0], "hubs_ms": kt["k_hll_hubs"][0],
                         "algorithmic_bytes": alg, "achieved_gbs": alg / (dev_ms / 1e3) / 1e9,
                         "frac": alg / (dev_ms / 1e3) / 1e9 / peak, "peak_source": f"{peak_kind} hbm_gbs"}
    times = []
    for _ in range(3):
        t0 = time.perf_counter()
        avg, anfs, _, st = g.hyperanf(20, bits)
        times.append(time.perf_counter() - t0)
    kt = _profiled(pb, HLL_KERNELS, lambda: g.hyperanf(20, bits))
    out["hyperanf"] = {"ms_median": float(np.median(times)) * 1e3, "epochs": st.iterations,
                       "push_epochs": st.push_iterations, "avg_distance": avg, "anfs": len(anfs),
                       "gather_kernel_ms": kt["k_hll_rows"][0] + kt["k_hll_hubs"][0],
                       "timing": "host clock around plato_hyperanf (iteration 20), median of 3"}
    rng = np.random.default_rng(2)
    for label, tg in (("all_targets", None),
                      ("64_targets", np.isin(np.arange(V), rng.choice(V, 64, replace=False)))):
        g.nstep_degrees(step=2, bits=bits, targets=tg)
        t0 = time.perf_counter()
        _, _, st = g.nstep_degrees(step=2, bits=bits, targets=tg)
        out[f"nstep_{label}"] = {"ms": (time.perf_counter() - t0) * 1e3, "step": 2, "epochs": st.iterations,
                                 "push_epochs": st.push_iterations}
    g.close()
    return out


def suite_wpr(pb):
    """Weighted PageRank (weighted_pagerank.hpp) on the PageRank graph, RMAT s24
    ef16 seed 3, with seeded uniform(0.1, 10) weights, 20 epochs (eps 0).

    Algorithmic bytes per epoch: 12E (id, weight, gathered state) + 8(V+1)
    offsets + 16V (old rank, weight sum, new rank, new state)."""
    V, s, d = pb.rmat(SCALE, EDGEFACTOR, SEED)
    w = np.random.default_rng(SEED).uniform(0.1, 10.0, s.size)
    g = pb.Graph(V, s, d, is_directed=True, weights=w)
    E = int(s.size)
    g.weighted_pagerank(ITERATIONS, DAMPING, 0.0)
    kt = _profiled(pb, PULL_KERNELS, lambda: g.weighted_pagerank(ITERATIONS, DAMPING, 0.0))
    times = []
    for _ in range(3):
        t0 = time.perf_counter()
        g.weighted_pagerank(ITERATIONS, DAMPING, 0.0)
        times.append(time.perf_counter() - t0)
    g.close()
    epoch_ms = sum(t for t, _ in kt.values()) / ITERATIONS
    alg = 12 * E + 8 * (V + 1) + 16 * V
    peak, peak_kind = measured_peak()
    ms = float(np.median(times)) * 1e3
    return {"workload": f"wpr_rmat_s{SCALE}_ef{EDGEFACTOR}_seed{SEED}_uniform_weights", "vertices": V, "edges": E,
            "ms_median": ms, "gteps": E * ITERATIONS / (ms / 1e3) / 1e9,
            "pull_kernels_ms_per_epoch": epoch_ms, "achieved_gbs": alg / (epoch_ms / 1e3) / 1e9,
            "frac": alg / (epoch_ms / 1e3) / 1e9 / peak, "peak_source": f"{peak_kind} hbm_gbs",
            "timing": "host clock around plato_weighted_pagerank (20 epochs, host output), median of 3"}


def suite_trustrank(pb):
    """TrustRank with seed selection by inverse PageRank (trustrank.hpp) on
    RMAT s22 ef16 seed 4, a seeded 10% of the vertices good, 100 seeds."""
    V, s, d = pb.rmat(22, 16, 4)
    g = pb.Graph(V, s, d, is_directed=True)
    good = np.random.default_rng(4).random(V) < 0.1
    g.trustrank(good, 100, 0.85, 100, 0, 0.001)
    times = []
    for _ in range(3):
        t0 = time.perf_counter()
        _, seeds, st = g.trustrank(good, 100, 0.85, 100, 0, 0.001)
        times.append(time.perf_counter() - t0)
    g.close()
    return {"workload": "trustrank_rmat_s22_ef16_seed4_good10pct", "vertices": V, "edges": int(s.size),
            "ms_median": float(np.median(times)) * 1e3, "seeds": int(seeds.size),
            "trust_epochs": st.iterations,
            "timing": "host clock around plato_trustrank (selection PageRank + trust PPR, ranks to host), median of 3"}


def suite_ppr_single(pb):
    """Single-source PPR on RMAT s24 seed 3 until L1 delta < 1e-7, both engines."""
    V, s, d = pb.rmat(24, 16, 3)
    g = pb.Graph(V, s, d, is_directed=True)
    deg = np.bincount(s, minlength=V)
    src = int(np.random.default_rng(3).choice(np.flatnonzero(deg > 0)))
    out = {"workload": "ppr_rmat_s24_ef16_seed3", "src": src}
    import ctypes as C

    import torch
    from plato_b200 import _lib
    lib = _lib.load()
    pinned = torch.empty(V, dtype=torch.float32, pin_memory=True)  # reused by every call
    got = {}
    for mode, name in ((pb.PLATO_PPR_PULL, "pull"), (pb.PLATO_PPR_PUSHPULL, "pushpull")):
        o = _lib.PprOpts(500, 0.85, src, 1e-7)
        st = _lib.RunStats()

        def call():
            _lib.check(lib.plato_personalized_pagerank(g.handle, C.byref(o), mode, C.c_void_p(pinned.data_ptr()),
                                                       C.byref(st)), "plato_personalized_pagerank")

        call()
        dts = []
        for _ in range(3):
            t0 = time.perf_counter()
            call()
            dts.append(time.perf_counter() - t0)
        got[name] = pinned.numpy().astype(np.float32).copy()
        t0 = time.perf_counter()
        g.personalized_pagerank(src, 500, 0.85, 1e-7, mode)  # the Python wrapper: a fresh pageable array
        fresh = time.perf_counter() - t0
        out[name] = {"ms": float(np.median(dts)) * 1e3, "ms_fresh_numpy_output": fresh * 1e3,
                     "iterations": st.iterations, "push_iterations": st.push_iterations,
                     "timing": "host clock around plato_personalized_pagerank, ranks into a reused pinned "
                               "host buffer, median of 3"}
    g.close()
    import oracle  # CPU baseline: the same query, whole, pull-only and push-pull
    ref = oracle.RefGraph(V, s, d, True)
    for pushpull, name in ((False, "pull"), (True, "pushpull")):
        t0 = time.perf_counter()
        want, ep, pe, _, _ = ref.ppr(src, 500, 0.85, 1e-7, pushpull)
        dt = time.perf_counter() - t0
        err = np.abs(got[name].astype(np.float64) - want)
        out[name]["parity"] = {"vs": "oracle ref_cpu.c FP64", "l1": float(err.sum()),
                               "max_abs": float(err.max()), "oracle_epochs": ep, "tolerance_l1": 1e-6}
        out[name]["cpu_baseline"] = {"ms": dt * 1e3, "epochs": ep, "push_epochs": pe,
                                     "cores": oracle.max_threads(), "kind": "port",
                                     "sample": "the same query, whole, oracle ref_cpu.c (FP64)"}
    ref.close()
    return out


def suite_batch(pb, plain_n=16, quick=False):
    """Batched multi-source PPR on RMAT s22 seed 4 (K in 64/256/1024, Zipf seed
    sets 1..32, eps 1e-6) against the plain engine running the same queries one
    at a time (plato_seedset_ppr, pull-only).  quick: one K=128 batch only (for
    profiler captures)."""
    V, s, d = pb.rmat(22, 16, 4)
    g = pb.Graph(V, s, d, is_directed=True)
    deg = np.bincount(s, minlength=V)
    sets = zipf_seed_sets(deg, 1024, 32, 4)
    if quick:  # one K = 128 batch at k_tile 128, no autotuning: about 3 GB on the device
        out = g.ppr_batch(sets[:128], 300, 0.85, 1e-6, topk=100, k_tile=128)
        g.close()
        return {"workload": "ppr_batch_rmat_s22_ef16_seed4", "K": 128, "k_tile": 128,
                "iterations_max": int(out["iterations"].max())}
    plain_qps, _, plain_ranks = plain_engine_qps(g, sets, plain_n, collect=True)
    res = {"workload": "ppr_batch_rmat_s22_ef16_seed4", "vertices": V, "edges": int(s.size),
           "plain_qps": plain_qps, "plain_sample": plain_n}
    for K in (64, 256, 1024):
        g.ppr_batch(sets[:K], 300, 0.85, 1e-6, topk=100)  # autotune + warm
        dts = []
        for _ in range(5):  # median of five whole batches
            t0 = time.perf_counter()
            out = g.ppr_batch(sets[:K], 300, 0.85, 1e-6, topk=100)
            dts.append(time.perf_counter() - t0)
        dt = float(np.median(dts))
        res[f"K{K}"] = {"qps": K / dt, "s": dt, "speedup_vs_plain": K / dt / plain_qps,
                        "iterations_max": int(out["iterations"].max()), "timing": "median of 5 batches",
                        "batches_s": dts, "k_tile_auto": g.ppr_batch_k_tile(K)}
        per_kt = {}
        for kt in (8, 16, 32, 64):
            if kt > max(8, K):
                continue
            g.ppr_batch(sets[:K], 300, 0.85, 1e-6, topk=100, k_tile=kt)
            t0 = time.perf_counter()
            g.ppr_batch(sets[:K], 300, 0.85, 1e-6, topk=100, k_tile=kt)
            per_kt[kt] = K / (time.perf_counter() - t0)
        res[f"K{K}"]["qps_by_k_tile"] = per_kt
    chk = g.ppr_batch(sets[:plain_n], 300, 0.85, 1e-6, ranks=True)
    l1 = [float(np.abs(chk["ranks"][q].astype(np.float64) - plain_ranks[q]).sum())
          for q in range(plain_n)]
    res["l1_batch_vs_plain_max"] = max(l1)
    g.close()
    import oracle  # CPU baseline: the first query, whole, on the host cores
    ref = oracle.RefGraph(V, s, d, True)
    t0 = time.perf_counter()
    want, ep, _ = ref.seedset_ppr(sets[0], 300, 0.85, 1e-6)
    dt = time.perf_counter() - t0
    ref.close()
    res["cpu_baseline"] = {"qps": 1.0 / dt, "epochs": ep, "cores": oracle.max_threads(), "kind": "port",
                           "sample": "query 0 of the same seed sets, oracle ref_cpu.c (FP64)"}
    err = np.abs(chk["ranks"][0].astype(np.float64) - want)
    res["parity_query0"] = {"vs": "oracle ref_cpu.c FP64", "l1": float(err.sum()), "max_abs": float(err.max()),
                            "epochs": int(chk["iterations"][0]), "oracle_epochs": ep, "tolerance_l1": 1e-6}
    return res


def suite_serving(pb, rates=(100, 1000, 5000, 20000), n_req=400, slot_options=(64, 256)):
    """PPR serving on RMAT s24 seed 5: Poisson arrivals, Zipf seed sets 1..64,
    eps 1e-6, top-100; latency = completion - arrival (host clock)."""
    V, s, d = pb.rmat(24, 16, 5)
    g = pb.Graph(V, s, d, is_directed=True)
    deg = np.bincount(s, minlength=V)
    out = {"workload": "ppr_serving_rmat_s24_ef16_seed5", "vertices": V}
    sets = zipf_seed_sets(deg, n_req, 64, 5)
    # plain engine, one query at a time (reused pinned output buffer)
    out["plain_qps"], _, _ = plain_engine_qps(g, sets, 16)
    for slots in slot_options:
        out[f"slots{slots}"] = _serve(pb, g, sets, rates, n_req, slots)
    g.close()
    return out


def steady_window(t_done, lat_ms, slots):
    """Steady-state rate of a serving run: t_done = completion times in
    completion order, lat_ms = their latencies.  The first and last
    h = min(slots, n / 4) completions are dropped (ramp-up and drain); the
    rate is the n - 2h completions in between over the time they took, with
    their latency percentiles.  A saturated server turns its slots over in
    generations of `slots`, so h = slots spans whole generations."""
    t_done = np.asarray(t_done, dtype=np.float64)
    lat_ms = np.asarray(lat_ms, dtype=np.float64)
    n = t_done.size
    h = max(1, min(slots, n // 4))
    w0, w1 = float(t_done[h - 1]), float(t_done[n - h - 1])
    mid = lat_ms[h:n - h]
    return {"dropped_each_end": h, "completions": n - 2 * h, "window_s": w1 - w0,
            "qps": float((n - 2 * h) / (w1 - w0)) if w1 > w0 else None,
            "p50_ms": float(np.percentile(mid, 50)), "p99_ms": float(np.percentile(mid, 99))}


def _serve(pb, g, sets, rates, n_req, slots):
    """Drives a PPRServer with Poisson arrivals at each offered rate.  n_req:
    requests per rate (an int, or a function of the rate).  Besides the whole
    run (requests / wall, latency percentiles over every request) it reports
    a steady-state window that leaves out the ramp-up and the drain: the
    first and the last h = min(slots, n / 4) completions are dropped, and the
    rate is the n - 2h completions in between over the time they took, with
    the latency percentiles of those requests.  When the server is saturated
    its slots turn over in generations, and h = slots makes the window span
    whole generations."""
    out = {}
    with pb.PPRServer(g, max_slots=slots, hbm_budget_bytes=64 << 30, max_iterations=300,
                      eps=1e-6, topk=100) as srv:
        for rate in rates:
            n = int(n_req(rate)) if callable(n_req) else int(n_req)
            rng = np.random.default_rng(rate)
            arrivals = np.cumsum(rng.exponential(1.0 / rate, n))
            sub, done, lat, t_done = 0, 0, [], []
            ids = {}
            t0 = time.perf_counter()
            while done < n:
                now = time.perf_counter() - t0
                while sub < n and arrivals[sub] <= now:
                    ids[srv.submit(sets[sub])] = arrivals[sub]
                    sub += 1
                st = srv.stats()
                if st["live"] == 0 and st["queued"] == 0 and sub < n:
                    time.sleep(max(0.0, arrivals[sub] - (time.perf_counter() - t0)))
                    continue
                srv.step()
                while (r := srv.poll()) is not None:
                    tc = time.perf_counter() - t0
                    lat.append(tc - ids.pop(r[0]))
                    t_done.append(tc)
                    done += 1
            wall = time.perf_counter() - t0
            lat_ms = np.array(lat) * 1e3
            t_done = np.array(t_done)
            entry = {"offered_qps": rate, "requests": n, "sustained_qps": n / wall,
                     "p50_ms": float(np.percentile(lat_ms, 50)),
                     "p99_ms": float(np.percentile(lat_ms, 99))}
            entry["steady"] = steady_window(t_done, lat_ms, slots)
            out[f"rate{rate}"] = entry
    return out


CEILING_MODES = ["ids", "gather4", "gather8", "gather16", "hot_l1", "coalesced"]


def run_ceiling(args):
    """The long-bin gather stream's ceiling on this GPU (plato_diag_pull_ceiling
    modes 0-5) beside the real k_pull_long, on the benchmark graph: one JSON
    line.  Times are CUDA-event averages per launch."""
    import ctypes as C

    import torch
    import plato_b200 as pb
    from plato_b200 import _lib
    lib = _lib.load()
    V, src, dst = pb.rmat(SCALE, EDGEFACTOR, SEED)
    g = pb.Graph(V, src, dst, is_directed=True)
    bins = pull_bins(V, dst)
    del src, dst
    out = {"ceiling": True, "workload": f"pagerank_rmat_s{SCALE}_ef{EDGEFACTOR}_seed{SEED}", "vertices": V,
           "long_bin": {"rows": bins["rows"]["k_pull_long"], "edges": bins["edges"]["k_pull_long"],
                        "algorithmic_bytes": bins["k_pull_long"]}}
    peak, kind = measured_peak()
    for mode, name in enumerate(CEILING_MODES):
        ms, n, cs = C.c_double(), C.c_uint64(), C.c_double()
        _lib.check(lib.plato_diag_pull_ceiling(g.handle, mode, 20, C.byref(ms), C.byref(n), C.byref(cs)),
                   "plato_diag_pull_ceiling")
        out[name] = {"ms": ms.value, "edges": n.value, "edges_per_ns": n.value / (ms.value * 1e6),
                     "frac_if_long_bin": bins["k_pull_long"] / (ms.value / 1e3) / 1e9 / peak}
    d_out = torch.empty(V, dtype=torch.float32, device="cuda")
    g.pagerank_device(d_out.data_ptr(), ITERATIONS, DAMPING, 0.0)
    kt = _profiled(pb, ["k_pull_long"], lambda: g.pagerank_device(d_out.data_ptr(), ITERATIONS, DAMPING, 0.0))
    torch.cuda.synchronize()
    tot, n = kt["k_pull_long"]
    out["k_pull_long"] = {"ms": tot / n, "edges_per_ns": bins["edges"]["k_pull_long"] / (tot / n * 1e6),
                          "frac": bins["k_pull_long"] / (tot / n / 1e3) / 1e9 / peak}
    out["peak"] = {"hbm_gbs": peak, "source": kind}
    g.close()
    out["batch"] = {"s22": batch_ceiling(pb, 22, 4), "s24": batch_ceiling(pb, 24, 5)}
    print(json.dumps(out), flush=True)
    return 0


BATCH_CEILING_MODES = ["rows", "sequential_rows", "l2_rows", "k_batch_iteration"]


def batch_ceiling(pb, scale, seed, kts=(64, 128), reps=5):
    """The batched pull's row-gather stream on the batched / serving graph
    (plato_diag_batch_ceiling modes 0-2) beside the real batched iteration
    (mode 3) at the same tile widths.  Times are CUDA-event averages."""
    import ctypes as C

    from plato_b200 import _lib
    lib = _lib.load()
    V, s, d = pb.rmat(scale, 16, seed)
    g = pb.Graph(V, s, d, is_directed=True)
    E = int(s.size)
    del s, d
    peak, kind = measured_peak()
    out = {"workload": f"rmat_s{scale}_ef16_seed{seed}", "vertices": V, "edges": E,
           "peak": {"hbm_gbs": peak, "source": kind}}
    for kt in kts:
        row = {}
        for mode, name in enumerate(BATCH_CEILING_MODES):
            ms, n, cs = C.c_double(), C.c_uint64(), C.c_double()
            _lib.check(lib.plato_diag_batch_ceiling(g.handle, kt, mode, reps, C.byref(ms), C.byref(n), C.byref(cs)),
                       "plato_diag_batch_ceiling")
            # bytes the stream needs: ids + one kt-float row per edge
            b = 4 * E + 4 * E * kt
            row[name] = {"ms": ms.value, "row_bytes_gbs": b / (ms.value / 1e3) / 1e9,
                         "frac": b / (ms.value / 1e3) / 1e9 / peak}
        out[f"kt{kt}"] = row
    g.close()
    return out


def run_suite(args):
    import torch  # noqa: F401  (CUDA context for the library)
    import plato_b200 as pb
    res = {"suite": True}
    for name, fn in (("bfs", suite_bfs), ("cc", suite_cc), ("trustrank", suite_trustrank), ("hll", suite_hll),
                     ("wpr", suite_wpr),
                     ("ppr_single", suite_ppr_single),
                     ("ppr_batch", suite_batch), ("serving", suite_serving)):
        if args.only and name not in args.only.split(","):
            continue
        t0 = time.perf_counter()
        res[name] = fn(pb, quick=True) if (args.quick and name == "ppr_batch") else fn(pb)
        res[name]["wall_s"] = time.perf_counter() - t0
        print(json.dumps({name: res[name]}), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["plato", "reference"], default="plato")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the batched-PPR and serving sections of the default line")
    ap.add_argument("--scale", type=int, default=SCALE,
                    help="RMAT scale (smaller values are for profiling captures only)")
    ap.add_argument("--suite", action="store_true",
                    help="also measure BFS, single PPR, batched PPR and serving (one JSON line each)")
    ap.add_argument("--only", default="", help="with --suite: comma list of bfs,cc,trustrank,hll,wpr,ppr_single,ppr_batch,serving")
    ap.add_argument("--quick", action="store_true", help="with --suite: one small batch (profiling)")
    ap.add_argument("--ceiling", action="store_true",
                    help="measure the long-bin gather stream's ceiling beside k_pull_long (one JSON line)")
    args = ap.parse_args()
    globals()["SCALE"] = args.scale
    if args.suite:
        return run_suite(args)
    if args.ceiling:
        return run_ceiling(args)
    if args.impl == "reference":
        return run_reference(args)
    return run_plato(args)


if __name__ == "__main__":
    sys.exit(main())
