"""Builds the oracle (the CPU restatement of the Dynamis step) as oracle/_build/liboracle.so.

TEST INFRASTRUCTURE ONLY: the library is loaded by tests/ and by bench.py's cpu_baseline leg.
Compiled without -ffast-math and with -ffp-contract=off so every float operation is one IEEE-754
binary32 operation, as in the CUDA build.
"""
from __future__ import annotations

import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent
OUT = HERE / "_build"
LIBRARY = OUT / "liboracle.so"
SOURCES = [HERE / "oracle.cpp", HERE / "adjoint64.cpp", HERE / "scene.cpp"]
HEADERS = [HERE / "oracle_math.h", HERE / "oracle_geom.h", HERE / "oracle_query.h", ROOT / "include" / "dynamis_abi.h",
           ROOT / "include" / "dynamis_cuda.h"]


def build(verbose: bool = False) -> Path:
    OUT.mkdir(exist_ok=True)
    newest = max(p.stat().st_mtime for p in SOURCES + HEADERS)
    if LIBRARY.exists() and LIBRARY.stat().st_mtime >= newest:
        return LIBRARY
    cmd = ["g++", "-O3", "-std=c++17", "-fPIC", "-shared", "-fopenmp", "-ffp-contract=off", "-fno-fast-math",
           "-I", str(ROOT / "include"), *map(str, SOURCES), "-o", str(LIBRARY)]
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        sys.stderr.write(proc.stderr)
        raise RuntimeError("oracle build failed")
    if verbose:
        print(f"built {LIBRARY}")
    return LIBRARY


if __name__ == "__main__":
    build(verbose=True)
