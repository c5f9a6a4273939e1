"""Builds libfdtd_b200.so (the C-ABI library) in-tree with nvcc for sm_100a.

    python -m fdtd_b200.build_lib [--force]

Per-file flags:
  kernels_plain.cu   -fmad=false: the FP64 plain method keeps every product and
                     sum separately rounded, as the reference compiled with
                     -ffp-contract=off.
  fdtd_capi.cu       host code with -ffp-contract=off (CPML / material
                     coefficient set-up in the reference's rounding).
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libfdtd_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off",
          "--expt-relaxed-constexpr", "-Xptxas", "-warn-spills"]
SOURCES = {
    "kernels_plain.cu": ["-fmad=false"],
    "kernels_fused.cu": [],
    "kernels_fused3d.cu": [],
    "kernels_fused3d_tma.cu": [],
    "kernels_fused3d_async.cu": [],
    "kernels_tfsf.cu": [],
    "kernels_batch.cu": [],
    "kernels_common.cu": [],
    "kernels_adjoint.cu": [],
    "fdtd_capi.cu": [],
}
HEADERS = ["internal.h", "fused3d_common.cuh", os.path.join("..", "..", "include", "fdtd_b200.h")]


def _newer(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    objs = []
    hdrs = [os.path.join(CSRC, h) for h in HEADERS]
    for src, extra in SOURCES.items():
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src.replace(".cu", ".o"))
        objs.append(o)
        if force or _newer(o, [s, __file__] + hdrs):
            cmd = [NVCC] + ARCH + COMMON + extra + ["-c", s, "-o", o]
            if verbose:
                print(" ".join(cmd))
            subprocess.run(cmd, check=True)
    if force or _newer(LIB, objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
