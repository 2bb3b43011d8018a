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
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
HEADERS = [CSRC / "pdm1_math.cuh", CSRC / "pdm1_device.cuh", CSRC / "pdm1_stage.cuh",
           ROOT / "include" / "pdm1.h"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off"]
# translation unit -> its own precision flags
UNITS = {
    # the FP64 march: every product and sum separately rounded, IEEE div/sqrt
    CSRC / "pdm1_march.cu": ["--fmad=false"],
    # the single-precision stencil: fast math, FMA contraction
    CSRC / "pdm1_stage_fp32.cu": ["--use_fast_math"],
    # dose scoring (gamma index)
    CSRC / "pdm1_gamma.cu": [],
    # learned moving box: proposer network training and BF16 inference, box kernels
    CSRC / "pdm1_box.cu": [],
    # analytical CSDA + straight-streaming reference dose
    CSRC / "pdm1_analytical.cu": [],
    # the plans' caching allocator
    CSRC / "pdm1_pool.cu": [],
}
SOURCES = list(UNITS)

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
        BUILD.mkdir(exist_ok=True)
        objs = []
        log = []
        for src, flags in UNITS.items():
            obj = BUILD / (src.stem + ".o")
            cmd = [nvcc(), *ARCH, *COMMON, *flags, "-c", "-o", str(obj), str(src)]
            if verbose:
                cmd.insert(1, "-Xptxas=-v")
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode != 0:
                raise RuntimeError(f"nvcc failed on {src.name}:\n{r.stdout}\n{r.stderr}")
            log.append(r.stderr)
            objs.append(str(obj))
        r = subprocess.run([nvcc(), *ARCH, "-shared", "-o", str(LIB), *objs], capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc link failed:\n{r.stdout}\n{r.stderr}")
        if verbose:
            print("\n".join(log))
    return LIB


if __name__ == "__main__":
    build(force=True, verbose=True)
