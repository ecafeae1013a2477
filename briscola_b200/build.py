"""Build the native libraries in-tree for sm_100a.

``python -m briscola_b200.build`` (or ``__graft_entry__.build()``) compiles
``csrc/*.cu`` with nvcc into two plain C ABI libraries with the CUDA runtime
linked statically: ``briscola_b200/_lib/libbmg.so`` (the multigrid solver,
include/bmg.h), ``briscola_b200/_lib/libbunet.so`` (the U-Net kernels,
include/bunet.h) and ``briscola_b200/_lib/libbfft.so`` (the FFT Poisson
solver, include/bfft.h).
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "_lib", "libbmg.so")
SOURCES = ["bmg_host.cu", "bmg_kernels.cu", "bmg_smooth_fused.cu", "bmg_krylov.cu", "bmg_noalloc.cu",
           "bmg_project.cu"]
HEADERS = ["bmg_internal.h", "bmg_stencil.cuh", "bmg_grid.cuh"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FFT_OUT = os.path.join(HERE, "_lib", "libbfft.so")
FFT_SOURCES = ["bfft.cu"]
UNET_OUT = os.path.join(HERE, "_lib", "libbunet.so")
UNET_SOURCES = ["bun_api.cu", "bun_conv.cu", "bun_elem.cu"]
UNET_HEADERS = ["bun_internal.h", "bun_api_internal.h"]


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.isabs(c) and os.path.exists(c) or not os.path.isabs(c)):
            return c
    return "nvcc"


def _build(out: str, sources, headers, header: str, force: bool, verbose: bool) -> str:
    srcs = [os.path.join(CSRC, s) for s in sources]
    deps = srcs + [os.path.join(CSRC, h) for h in headers] + [os.path.join(HERE, "..", "include", header)]
    if not force and os.path.exists(out):
        t = os.path.getmtime(out)
        if all(os.path.getmtime(d) <= t for d in deps if os.path.exists(d)):
            return out
    os.makedirs(os.path.dirname(out), exist_ok=True)
    cmd = [nvcc(), *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-shared",
           "-o", out + ".tmp", *srcs]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(out + ".tmp", out)
    return out


def build_native(force: bool = False, verbose: bool = False) -> str:
    """libbmg.so (the solver); returns its path."""
    return _build(OUT, SOURCES, HEADERS, "bmg.h", force, verbose)


def build_fft(force: bool = False, verbose: bool = False) -> str:
    """libbfft.so (the FFT Poisson solver, include/bfft.h); returns its path."""
    return _build(FFT_OUT, FFT_SOURCES, [], "bfft.h", force, verbose)


def build_unet(force: bool = False, verbose: bool = False) -> str:
    """libbunet.so (the U-Net kernels); returns its path."""
    return _build(UNET_OUT, UNET_SOURCES, UNET_HEADERS, "bunet.h", force, verbose)


if __name__ == "__main__":
    print(build_native(force="--force" in sys.argv, verbose=True))
    print(build_unet(force="--force" in sys.argv, verbose=True))
    print(build_fft(force="--force" in sys.argv, verbose=True))
