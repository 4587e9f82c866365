"""Build libtdgl_b200.so (the CUDA kernels and the C-ABI of include/tdgl_b200.h) for sm_100a, in-tree.

    python -m juliatdgl_b200.build

nvcc cross-compiles here without a GPU.  --fmad=false keeps the stencils' IEEE operation order (no FMA
contraction) so they agree with the reference's CPU arithmetic; kernels that want FMA call fma() explicitly.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libtdgl_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "--fmad=false", "-std=c++17",
         "-Xcompiler", "-fPIC", "-Xcompiler", "-fno-fast-math", "-Xcompiler", "-ffp-contract=off"]


def sources():
    return sorted(glob.glob(os.path.join(SRC, "*.cu")))


def stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = sources() + glob.glob(os.path.join(SRC, "*.cuh")) + [os.path.join(HERE, "..", "include", "tdgl_b200.h")]
    return any(os.path.getmtime(p) > t for p in deps)


def build(verbose: bool = False, extra=()) -> str:
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    for src in sources():
        obj = os.path.join(objdir, os.path.basename(src)[:-3] + ".o")
        cmd = [NVCC, *FLAGS, *extra, "-dc", "-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
        objs.append(obj)
    cmd = [NVCC, *FLAGS, "-shared", *objs, "-o", LIB, "-lcudart"]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(verbose="-v" in sys.argv, extra=[a for a in sys.argv[1:] if a != "-v"])
    print(LIB)
