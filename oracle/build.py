"""Build the oracle (test infrastructure): oracle/libref_cpu.so from ref_cpu.c
and rmat.c, and, where the reference tree is present, oracle/_ref from the
reference's own headers.

    python -m oracle.build [--force]

The reference tree is found at $PLATO_REFERENCE_ROOT, else /root/reference.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
SRCS = [HERE / "ref_cpu.c", HERE / "rmat.c"]
LIB = HERE / "libref_cpu.so"


def build(force: bool = False) -> Path:
    if not force and LIB.exists() and all(LIB.stat().st_mtime >= s.stat().st_mtime for s in SRCS):
        return LIB
    tmp = LIB.with_suffix(".so.tmp")
    cmd = ["gcc", "-O3", "-march=x86-64-v2", "-fopenmp", "-fPIC", "-shared", "-std=c11",
           "-Wall", "-o", str(tmp), *map(str, SRCS), "-lm"]
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


REF_ROOT = Path(os.environ.get("PLATO_REFERENCE_ROOT", "/root/reference"))
REF_SHIM = HERE / "hll_ref_shim.cpp"
REF_LIB = HERE / "_ref" / "libhll_ref.so"


def build_ref(force: bool = False, ref_root: Path = REF_ROOT) -> Path | None:
    """Compile oracle/_ref/libhll_ref.so: hll_ref_shim.cpp over the reference's
    own plato/util/hyperloglog.hpp + hash.hpp, read where they lie in the
    reference tree (header-only, no dependencies).  Returns None when the
    reference tree is absent (the committed golden vectors stand in)."""
    if not (ref_root / "plato" / "util" / "hyperloglog.hpp").exists():
        return None
    if not force and REF_LIB.exists() and REF_LIB.stat().st_mtime >= REF_SHIM.stat().st_mtime:
        return REF_LIB
    REF_LIB.parent.mkdir(exist_ok=True)
    tmp = REF_LIB.with_suffix(".so.tmp")
    cmd = ["g++", "-O2", "-fPIC", "-shared", "-std=c++14", "-I", str(ref_root), "-o", str(tmp),
           str(REF_SHIM)]
    subprocess.run(cmd, check=True)
    os.replace(tmp, REF_LIB)
    return REF_LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
    print(build_ref(force="--force" in sys.argv))
