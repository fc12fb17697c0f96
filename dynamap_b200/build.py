"""Build libdynamap_b200.so in-tree with nvcc for sm_100a.

The library is plain CUDA/C++ behind the C ABI of include/dynamap.h: no torch
types, cudart linked statically, only the driver (libcuda) needed at run
time.  Objects go to dynamap_b200/_build/, the .so next to this file.

  python -m dynamap_b200.build          # incremental
  python -m dynamap_b200.build --force  # rebuild everything
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libdynamap_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

SOURCES = ["image.cu", "icp.cu", "tsdf.cu", "session.cu", "serving.cu", "noalloc.cu",
           "mesh.cu", "evict.cu", "config.cpp"]
HEADERS = ["common.cuh", "image.cuh", "icp.cuh", "tsdf.cuh", "sessdev.cuh", "session_impl.cuh",
           "dyn_exp.h", "mesh_cell.h", "mc_tables.h", "evict_ops.h", "mesh_kernels.cuh",
           "evict_kernels.cuh"]

# -fmad=false: no FMA contraction, IEEE div/sqrt: every float operation
# rounds once, in source order (the bit-exact parity with the oracle relies
# on it).
NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-fmad=false", "-prec-div=true", "-prec-sqrt=true", "-ftz=false",
    "-Xcompiler", "-fPIC,-ffp-contract=off,-O2",
    "-ccbin", "g++",
]


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(OUT, exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [
        os.path.join(HERE, "..", "include", "dynamap.h")]
    objs = []
    for src in SOURCES:
        sp = os.path.join(CSRC, src)
        obj = os.path.join(OUT, src + ".o")
        objs.append(obj)
        if force or _stale(obj, [sp] + hdrs):
            cmd = [NVCC] + NVCC_FLAGS + ["-c", sp, "-o", obj]
            if src.endswith(".cpp"):
                cmd = ["g++", "-O2", "-std=c++17", "-fPIC", "-ffp-contract=off",
                       "-c", sp, "-o", obj]
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.run(cmd, check=True)
    if force or _stale(LIB, objs):
        cmd = [NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-shared",
               "-cudart", "static", "-ccbin", "g++", "-o", LIB] + objs
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
