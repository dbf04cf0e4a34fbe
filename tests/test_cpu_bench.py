"""bench.py's reference arm: it must time the reference's CPU path without
loading any product code, on the same config as the GPU arm."""
import json
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent

PROBE = r"""
import sys, json, argparse
sys.path.insert(0, {root!r})
import bench
bench.SCALE = 10
args = argparse.Namespace(gpus=1, steps=2, warmup=1)
bench.run_reference(args)
maps = open('/proc/self/maps').read()
print(json.dumps({{"product_module": 'plato_b200' in sys.modules,
                   "product_so": 'libplato_b200' in maps,
                   "oracle_so": 'libref_cpu' in maps or 'libplato_ref' in maps}}))
"""


def test_reference_arm_loads_no_product_code():
    out = subprocess.run([sys.executable, "-c", PROBE.format(root=str(ROOT))], capture_output=True,
                         text=True, timeout=300, cwd=str(ROOT))
    assert out.returncode == 0, out.stderr
    lines = [json.loads(x) for x in out.stdout.strip().splitlines()]
    line, probe = lines[0], lines[1]
    assert line["impl"] == "reference" and line["unit"] == "GTEPS" and line["value"] > 0
    from oracle import refplato
    assert line["e2e"]["h2d_bytes_per_step"] == 0
    assert line["cpu_baseline"]["kind"] == ("reference" if refplato.available() else "port")
    assert not probe["product_module"] and not probe["product_so"]
    assert probe["oracle_so"]


def test_both_arms_share_one_config():
    sys.path.insert(0, str(ROOT))
    import bench
    a = bench.bench_config(100, 1000, 1)
    assert a == bench.bench_config(100, 1000, 1)
    assert set(a) == {"workload", "vertices", "edges", "iterations", "damping", "parallelism", "step", "l2"}


def test_steady_window_spans_whole_generations():
    """A saturated server finishes its slots in generations: 4 generations of
    256 completions clumped 1.6 s apart are 160 q/s, whatever the spread
    inside a generation; the window leaves the ramp-up and the drain out."""
    import numpy as np
    sys.path.insert(0, str(ROOT))
    import bench
    rng = np.random.default_rng(0)
    t = np.sort(np.concatenate([1.6 * (k + 1) + rng.uniform(-0.2, 0.2, 256) for k in range(4)]))
    st = bench.steady_window(t, np.ones(t.size), 256)
    assert st["completions"] == 512 and st["dropped_each_end"] == 256
    assert abs(st["qps"] - 160.0) / 160.0 < 0.15
    # an unsaturated server: Poisson completions at 100/s give about 100/s
    t = np.cumsum(rng.exponential(0.01, 500)) + 0.8
    st = bench.steady_window(t, np.ones(t.size), 256)
    assert st["dropped_each_end"] == 125 and abs(st["qps"] - 100.0) < 15.0


def test_clock_summary_reads_reasons():
    sys.path.insert(0, str(ROOT))
    import bench
    c = bench.ClockSampler(0)
    assert c.summary()["reasons"] == ["unsampled"]
    c.rows = [["0", "1965", "1965", "700", "0x4", "Not Active", "Not Active", "Not Active", "Active"],
              ["0", "1950", "1965", "710", "0x0", "Not Active", "Not Active", "Not Active", "Not Active"]]
    s = c.summary()
    assert s["sm_mhz"] == 1957.5 and s["sm_max_mhz"] == 1965.0 and s["reasons"] == ["sw_power_cap"]
    assert s["samples"] == 2
