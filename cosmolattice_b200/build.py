"""Build libclb200.so in-tree for sm_100a (``python -m cosmolattice_b200.build``)."""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB_DIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIB_DIR, "libclb200.so")

SOURCES = ["clb_api.cu", "clb_u1.cu", "clb_batch.cu", "clb_noalloc.cu"]
DEPS = ["clb_api.cu", "clb_u1.cu", "clb_batch.cu", "clb_batch.cuh", "clb_vv.h", "clb_adjoint.cuh", "clb_noalloc.cu", "clb_internal.cuh", "clb_handle.cuh", "clb_u1.cuh", "clb_scalar.cuh", "clb_sweep.cuh", "clb_tma.cuh", "clb_spectrum.cuh"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "-Xcompiler", "-fPIC", "-shared",
]


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, d) for d in DEPS] + [os.path.join(ROOT, "include", "clb200.h")]
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not _stale():
        return LIB
    os.makedirs(LIB_DIR, exist_ok=True)
    nvcc = os.environ.get("NVCC", "nvcc")
    cmd = [nvcc, *NVCC_FLAGS, *[os.path.join(CSRC, s) for s in SOURCES], "-o", LIB, "-lcufft"]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
