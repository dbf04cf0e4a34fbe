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
