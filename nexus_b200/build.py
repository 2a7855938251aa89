"""Builds libnexus_mpm.so (the CUDA library behind include/nexus_mpm.h) in-tree.

Every translation unit is compiled for sm_100a only; the deterministic
transfer kernels are compiled with --fmad=false so each multiply and add is
rounded separately, in the reference's order.  Usage: python -m nexus_b200.build
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libnexus_mpm.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
          "--expt-relaxed-constexpr", f"-I{INCLUDE}", f"-I{CSRC}"]

UNITS = {
    "nxm_state.cu": ["-Xcompiler", "-ffp-contract=off"],  # f32 trimesh sampling, operation by operation
    "nxm_sort.cu": [],
    "nxm_transfer_fast.cu": [],
    "nxm_transfer_det.cu": ["--fmad=false"],
    "nxm_transfer_fast_cpic.cu": [],
    "nxm_noalloc.cu": [],
    "nxm_readback.cu": ["--fmad=false"],
}

HEADERS = ["nxm_device.cuh", "nxm_layout.h", "nxm_kernels.h", "nxm_transfer.inc.cuh"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def _mtime(p: str) -> float:
    return os.path.getmtime(p) if os.path.exists(p) else 0.0


def build(verbose: bool = False, extra: list[str] | None = None) -> str:
    os.makedirs(OBJ, exist_ok=True)
    nvcc = _nvcc()
    dep_time = max(_mtime(os.path.join(CSRC, h)) for h in HEADERS)
    dep_time = max(dep_time, _mtime(os.path.join(INCLUDE, "nexus_mpm.h")), _mtime(__file__))
    objs = []
    relink = not os.path.exists(LIB)
    for src, flags in UNITS.items():
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJ, src.replace(".cu", ".o"))
        objs.append(o)
        if _mtime(o) < max(_mtime(s), dep_time):
            cmd = [nvcc, *ARCH, *COMMON, *flags, *(extra or []), "-c", s, "-o", o]
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.run(cmd, check=True)
            relink = True
    if relink or any(_mtime(o) > _mtime(LIB) for o in objs):
        cmd = [nvcc, *ARCH, "-shared", "-o", LIB, *objs, "-lcudart"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(verbose=True, extra=sys.argv[1:])
