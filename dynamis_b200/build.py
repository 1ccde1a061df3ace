"""Builds libdynamis_cuda.so (sm_100a) in-tree with nvcc.

The kernels are compiled with IEEE single-precision semantics (-fmad=false -prec-div=true
-prec-sqrt=true): every + - * / sqrt of the step is one correctly rounded binary32 operation, which
is what makes a step reproducible bit for bit. Host code is compiled with -ffp-contract=off for the
same reason.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PACKAGE = Path(__file__).resolve().parent
ROOT = PACKAGE.parent
CSRC = PACKAGE / "csrc"
INCLUDE = ROOT / "include"
BUILD = PACKAGE / "_build"
LIBRARY = PACKAGE / "libdynamis_cuda.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = [
    "-O3", "-lineinfo", "-std=c++17", "-fmad=false", "-prec-div=true", "-prec-sqrt=true",
    "-Xcompiler", "-fPIC,-fvisibility=hidden,-ffp-contract=off", "--expt-relaxed-constexpr",
]
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-fvisibility=hidden", "-ffp-contract=off"]


def _nvcc() -> str:
    for candidate in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if candidate and Path(candidate).exists():
            return candidate
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libdynamis_cuda.so")


def _stale(target: Path, sources: list[Path]) -> bool:
    if not target.exists():
        return True
    mtime = target.stat().st_mtime
    return any(s.stat().st_mtime > mtime for s in sources)


def _run(cmd: list[str]) -> None:
    proc = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True)
    if proc.returncode != 0:
        sys.stderr.write(proc.stdout + proc.stderr)
        raise RuntimeError(f"build step failed: {' '.join(cmd[:3])} ... (exit {proc.returncode})")


def build(verbose: bool = False, ptxas_info: bool = False) -> Path:
    """Compiles the CUDA step library if any source is newer than it; returns its path."""
    BUILD.mkdir(exist_ok=True)
    headers = sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.h")) + sorted(INCLUDE.glob("*.h"))
    world_cu = CSRC / "world.cu"
    scene_cpp = CSRC / "scene.cpp"
    world_o = BUILD / "world.o"
    static_cu = CSRC / "static_sort.cu"
    static_o = BUILD / "static_sort.o"
    scene_o = BUILD / "scene.o"
    nvcc = _nvcc()
    flags = list(NVCC_FLAGS)
    if ptxas_info:
        flags += ["-Xptxas", "-v"]
    if _stale(world_o, [world_cu, *headers]) or ptxas_info:
        _run([nvcc, *ARCH, *flags, "-I", str(INCLUDE), "-c", str(world_cu), "-o", str(world_o)])
    if _stale(static_o, [static_cu, *headers]):
        _run([nvcc, *ARCH, *flags, "-I", str(INCLUDE), "-c", str(static_cu), "-o", str(static_o)])
    if _stale(scene_o, [scene_cpp, *headers]):
        _run(["g++", *CXX_FLAGS, "-I", str(INCLUDE), "-c", str(scene_cpp), "-o", str(scene_o)])
    if _stale(LIBRARY, [world_o, static_o, scene_o]):
        _run([nvcc, *ARCH, "-shared", "-o", str(LIBRARY), str(world_o), str(static_o), str(scene_o)])
    if verbose:
        print(f"built {LIBRARY}")
    return LIBRARY


if __name__ == "__main__":
    build(verbose=True, ptxas_info="--ptxas" in sys.argv)
