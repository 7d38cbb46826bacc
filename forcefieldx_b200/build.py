"""Build libffxcuda.so (the energy library) and libffxpeak.so (FMA-throughput microkernels
for the benchmark's pipe fractions) in-tree with nvcc for sm_100a (no JIT cache, no torch
extension)."""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SOURCES = ["handle.cu", "nlist.cu", "pme.cu", "real.cu", "vdw.cu", "recip.cu", "pcg.cu", "md.cu", "batch.cu"]
LIB = os.path.join(HERE, "libffxcuda.so")
PEAK_SRC = "peak.cu"
PEAK_LIB = os.path.join(HERE, "libffxpeak.so")
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
              "-Xcompiler", "-fPIC", "-shared", "-diag-suppress", "177"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(HERE, "csrc", s) for s in SOURCES + ["ffx_internal.cuh"]]
    deps.append(os.path.join(os.path.dirname(HERE), "include", "ffxcuda.h"))
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    peak_src = os.path.join(HERE, "csrc", PEAK_SRC)
    if force or not os.path.exists(PEAK_LIB) or os.path.getmtime(PEAK_LIB) < os.path.getmtime(peak_src):
        cmd = [nvcc()] + NVCC_FLAGS + ["-o", PEAK_LIB, peak_src]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
    if not force and not stale():
        return LIB
    cmd = [nvcc()] + NVCC_FLAGS + ["-o", LIB] + [os.path.join(HERE, "csrc", s) for s in SOURCES]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
