"""Build the native solver library in-tree for sm_100a.

``python -m briscola_b200.build`` (or ``__graft_entry__.build()``) compiles
``csrc/*.cu`` with nvcc into ``briscola_b200/_lib/libbmg.so``: a plain C ABI
library (include/bmg.h) with the CUDA runtime linked statically.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "_lib", "libbmg.so")
SOURCES = ["bmg_host.cu", "bmg_kernels.cu", "bmg_smooth_fused.cu", "bmg_krylov.cu", "bmg_noalloc.cu"]
HEADERS = ["bmg_internal.h", "bmg_stencil.cuh", "bmg_grid.cuh"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.isabs(c) and os.path.exists(c) or not os.path.isabs(c)):
            return c
    return "nvcc"


def build_native(force: bool = False, verbose: bool = False) -> str:
    srcs = [os.path.join(CSRC, s) for s in SOURCES]
    deps = srcs + [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(HERE, "..", "include", "bmg.h")]
    if not force and os.path.exists(OUT):
        t = os.path.getmtime(OUT)
        if all(os.path.getmtime(d) <= t for d in deps if os.path.exists(d)):
            return OUT
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    cmd = [nvcc(), *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-shared",
           "-o", OUT + ".tmp", *srcs]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    print(build_native(force="--force" in sys.argv, verbose=True))
