"""Build the ibgpu CUDA library in place (sm_100a).

    python immsered-boundary_b200/build_lib.py

Compiles csrc/*.cu with nvcc for sm_100a and links libibgpu.so next to this
file.  kernels_exact.cu is compiled with -fmad=false (the operation-for-
operation FP64 parity build); the other units keep contraction on.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libibgpu.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall"]
UNITS = {
    "ibgpu_api.cu": [],
    "kernels_fp64.cu": [],
    "kernels_exact.cu": ["-fmad=false"],
    "noalloc.cu": [],
    "indicator.cu": [],
    "interfaces.cu": [],
    "wall.cu": ["-fmad=false"],  # IEEE-exact wall distances (no contractions)
}


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _newest_input() -> float:
    t = 0.0
    for d in (CSRC, os.path.join(HERE, "..", "include")):
        for f in os.listdir(d):
            t = max(t, os.path.getmtime(os.path.join(d, f)))
    return t


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= _newest_input():
        return LIB
    os.makedirs(OBJ, exist_ok=True)
    objs = []
    for unit, extra in UNITS.items():
        obj = os.path.join(OBJ, unit.replace(".cu", ".o"))
        cmd = [nvcc(), *ARCH, *COMMON, *extra, "-c", os.path.join(CSRC, unit), "-o", obj]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.check_call(cmd)
        objs.append(obj)
    tmp = LIB + ".tmp"
    subprocess.check_call([nvcc(), *ARCH, "-shared", "-cudart", "static", "-o", tmp, *objs])
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
