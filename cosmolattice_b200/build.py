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

SOURCES = ["clb_api.cu", "clb_u1.cu", "clb_su2.cu", "clb_batch.cu", "clb_noalloc.cu", "clb_ic.cu"]
# per-unit flags: the lphi4SU2U1 unit writes the reference's rounding order as plain expressions
UNIT_FLAGS = {"clb_su2.cu": ["-fmad=false"]}
DEPS = ["clb_tangent.cuh", "clb_api.cu", "clb_u1.cu", "clb_batch.cu", "clb_batch.cuh", "clb_vv.h", "clb_adjoint.cuh", "clb_su2.cu", "clb_su2.cuh", "clb_noalloc.cu", "clb_ic.cu", "clb_internal.cuh", "clb_handle.cuh", "clb_u1.cuh", "clb_scalar.cuh", "clb_sweep.cuh", "clb_tma.cuh", "clb_spectrum.cuh"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "-Xcompiler", "-fPIC",
]


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, d) for d in DEPS] + [os.path.join(ROOT, "include", "clb200.h")]
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False, out: str = None, defines=()) -> str:
    """Compile every unit for sm_100a and link ``out`` (default: the package library)."""
    lib = out or LIB
    if not force and out is None and not _stale():
        return LIB
    os.makedirs(os.path.dirname(lib), exist_ok=True)
    nvcc = os.environ.get("NVCC", "nvcc")
    objs = []
    from concurrent.futures import ThreadPoolExecutor

    def one(src):
        obj = os.path.join(os.path.dirname(lib), src.replace(".cu", ".o"))
        cmd = [nvcc, *NVCC_FLAGS, *UNIT_FLAGS.get(src, []), *[f"-D{d}" for d in defines], "-c",
               os.path.join(CSRC, src), "-o", obj]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
        return obj

    with ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        objs = list(ex.map(one, SOURCES))
    cmd = [nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", *objs, "-o", lib, "-lcufft"]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    for o in objs:
        os.remove(o)
    if out is None:
        build_host(verbose)
    return lib


HOST_SRC = os.path.join(os.path.dirname(os.path.abspath(__file__)), "host", "cosmolattice_b200.cpp")
HOST_BIN = os.path.join(os.path.dirname(LIB), "cosmolattice_b200")


def build_host(verbose: bool = False) -> str:
    """The C++20 host program (the reference's main over the C ABI), linked next to the library."""
    cxx = os.environ.get("CXX", "g++")
    cmd = [cxx, "-std=c++20", "-O2", "-Wall", HOST_SRC, "-o", HOST_BIN, "-L", os.path.dirname(LIB), "-lclb200",
           "-Wl,-rpath,$ORIGIN"]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return HOST_BIN


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
