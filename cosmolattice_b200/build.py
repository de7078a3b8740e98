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

SOURCES = ["clb_api.cu", "clb_u1.cu", "clb_su2.cu", "clb_batch.cu", "clb_noalloc.cu", "clb_ic.cu", "clb_gws.cu"]
# per-unit flags: the lphi4SU2U1 unit writes the reference's rounding order as plain expressions
UNIT_FLAGS = {"clb_su2.cu": ["-fmad=false"]}
# every source and header under csrc/: an edit to any of them makes the library stale
DEPS = sorted(f for f in os.listdir(CSRC) if f.endswith((".cu", ".cuh", ".h")))

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


# The scalar-singlet model header is chosen when the library is built (csrc/models/): lphi4 for the
# package library, and each header in SCALAR_VARIANTS into lib/<name>/libclb200.so.  Only the units
# below include it; the others are shared between the builds.
SCALAR_MODEL_UNITS = ["clb_api.cu", "clb_batch.cu", "clb_noalloc.cu"]
SCALAR_VARIANTS = ["tanh2"]


def variant_lib(name: str) -> str:
    return os.path.join(LIB_DIR, name, "libclb200.so")


def _model_defines(name: str):
    return [f'CLB_SCALAR_MODEL_HEADER="models/{name}.h"', f"CLB_SCALAR_MODEL={name}"]


def build(force: bool = False, verbose: bool = False, out: str = None, defines=(), variants=None) -> str:
    """Compile every unit for sm_100a and link ``out`` (default: the package library), then the
    scalar-model variants (default: SCALAR_VARIANTS when building the package library)."""
    lib = out or LIB
    if not force and out is None and not _stale():
        return LIB
    if variants is None:
        variants = SCALAR_VARIANTS if out is None else []
    os.makedirs(os.path.dirname(lib), exist_ok=True)
    nvcc = os.environ.get("NVCC", "nvcc")
    from concurrent.futures import ThreadPoolExecutor

    def one(src, tag="", extra=()):
        obj = os.path.join(os.path.dirname(lib), src.replace(".cu", f"{tag}.o"))
        cmd = [nvcc, *NVCC_FLAGS, *UNIT_FLAGS.get(src, []), *[f"-D{d}" for d in (*defines, *extra)], "-c",
               os.path.join(CSRC, src), "-o", obj]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
        return obj

    jobs = [(src, "", ()) for src in SOURCES]
    jobs += [(src, f".{v}", _model_defines(v)) for v in variants for src in SCALAR_MODEL_UNITS]
    with ThreadPoolExecutor(max_workers=len(jobs)) as ex:
        objs = list(ex.map(lambda j: one(*j), jobs))
    main_objs = objs[:len(SOURCES)]

    def link(objects, target):
        os.makedirs(os.path.dirname(target), exist_ok=True)
        cmd = [nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", *objects, "-o", target, "-lcufft"]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)

    link(main_objs, lib)
    for k, v in enumerate(variants):
        vobjs = objs[len(SOURCES) + k * len(SCALAR_MODEL_UNITS):len(SOURCES) + (k + 1) * len(SCALAR_MODEL_UNITS)]
        shared = [o for src, o in zip(SOURCES, main_objs) if src not in SCALAR_MODEL_UNITS]
        link(vobjs + shared, variant_lib(v))
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
