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
PLATO_SHIM = HERE / "ref_shim" / "plato_ref_shim.cpp"
PLATO_SHIM_W = HERE / "ref_shim" / "plato_ref_shim_weighted.cpp"
PLATO_SHIM_H = HERE / "ref_shim" / "shim_common.hpp"
PLATO_SHIM_INC = HERE / "ref_shim" / "include"
PLATO_LIB = HERE / "_ref" / "libplato_ref.so"
PLATO_LIB_W = HERE / "_ref" / "libplato_ref_weighted.so"


def _newer(lib: Path, *deps: Path) -> bool:
    return lib.exists() and all(lib.stat().st_mtime >= d.stat().st_mtime for d in deps)


def build_ref(force: bool = False, ref_root: Path = REF_ROOT) -> Path | None:
    """Compile the reference's own code into oracle/_ref, from its sources
    where they lie in the reference tree:
      libhll_ref.so    hll_ref_shim.cpp over plato/util/hyperloglog.hpp +
                       hash.hpp (header-only, no dependencies);
      libplato_ref.so, libplato_ref_weighted.so
                       ref_shim/plato_ref_shim*.cpp over the engine, graph and
                       algorithm headers (pagerank, personalized_pagerank, bfs,
                       trustrank, weighted_pagerank, connected_component_t,
                       hyperanf), against the one-rank stand-ins in
                       ref_shim/include for the libraries the reference needs.
    Returns None when the reference tree is absent (the committed golden
    vectors under tests/golden/ stand in)."""
    if not (ref_root / "plato" / "util" / "hyperloglog.hpp").exists():
        return None
    REF_LIB.parent.mkdir(exist_ok=True)
    if force or not _newer(REF_LIB, REF_SHIM):
        tmp = REF_LIB.with_suffix(".so.tmp")
        cmd = ["g++", "-O2", "-fPIC", "-shared", "-std=c++14", "-I", str(ref_root), "-o", str(tmp),
               str(REF_SHIM)]
        subprocess.run(cmd, check=True)
        os.replace(tmp, REF_LIB)
    if (ref_root / "plato" / "engine" / "dualmode.hpp").exists():
        stubs = [p for p in PLATO_SHIM_INC.rglob("*") if p.is_file()]
        # one library per translation unit: the reference's headers define
        # non-inline functions, so each of its programs is a single unit
        for lib, src in ((PLATO_LIB, PLATO_SHIM), (PLATO_LIB_W, PLATO_SHIM_W)):
            if not force and _newer(lib, src, PLATO_SHIM_H, *stubs):
                continue
            tmp = lib.with_suffix(".so.tmp")
            # the stand-ins come first on the include path; __DUALMODE_DEBUG__
            # makes the engine log its push/pull choice (dualmode.hpp:281-293)
            cmd = ["g++", "-O2", "-std=c++17", "-fopenmp", "-fPIC", "-shared", "-w", "-D__DUALMODE_DEBUG__",
                   "-I", str(PLATO_SHIM_INC), "-I", str(ref_root),
                   "-I", str(ref_root / "plato" / "util" / "libcuckoo"), "-I", str(PLATO_SHIM.parent),
                   "-o", str(tmp), str(src), "-Wl,--no-undefined"]
            subprocess.run(cmd, check=True)
            os.replace(tmp, lib)
    return REF_LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
    print(build_ref(force="--force" in sys.argv))
