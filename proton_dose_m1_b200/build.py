"""Compile libpdm1.so (sm_100a) in-tree with nvcc.

The double-precision march is compiled with --fmad=false so every product
and sum is rounded separately, in the order the reference evaluates them.
"""

from __future__ import annotations

import os
import shutil
import subprocess
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
LIB = PKG / "libpdm1.so"
SOURCES = [PKG / "csrc" / "pdm1_march.cu"]
HEADERS = [PKG / "csrc" / "pdm1_math.cuh", ROOT / "include" / "pdm1.h"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17", "--fmad=false",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off",
    "-shared",
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libpdm1.so")


def stale() -> bool:
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    return any(p.stat().st_mtime > t for p in SOURCES + HEADERS)


def build(force: bool = False, verbose: bool = False) -> Path:
    if force or stale():
        cmd = [nvcc(), *NVCC_FLAGS, "-o", str(LIB), *map(str, SOURCES)]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed:\n{r.stdout}\n{r.stderr}")
        if verbose:
            print(r.stderr)
    return LIB


if __name__ == "__main__":
    build(force=True, verbose=True)
