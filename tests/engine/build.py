"""Build tests/engine/libengine_kat.so (test infrastructure) against the
header-only engine and libplato_b200.so.

    python -m tests.engine.build
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
SRC = HERE / "engine_kat.cu"
LIB = HERE / "libengine_kat.so"
HDR = ROOT / "include" / "plato_b200" / "dualmode.cuh"


def build(force: bool = False) -> Path:
    newest = max(SRC.stat().st_mtime, HDR.stat().st_mtime)
    if not force and LIB.exists() and LIB.stat().st_mtime >= newest:
        return LIB
    from plato_b200.build import build as build_lib, nvcc, LIB as PLATO_LIB
    build_lib()
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-O2", "-std=c++17",
           "--extended-lambda", "-Xcompiler", "-fPIC", "-shared", f"-I{ROOT / 'include'}",
           str(SRC), "-o", str(tmp), f"-L{PLATO_LIB.parent}", "-lplato_b200",
           f"-Xlinker", f"-rpath,{PLATO_LIB.parent}"]
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
