"""ctypes mirror of include/clb200.h and the loader of the in-tree libclb200.so.

The library is the product path: if it is missing, loading fails loudly (there is no CPU
fallback).  Build it with ``python -m cosmolattice_b200.build`` (or ``__graft_entry__.build()``).
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
# The library built with the scalar-singlet model header named by CLB200_SCALAR_MODEL (lib/<name>/),
# or the package library (lphi4).
_SCALAR_MODEL = os.environ.get("CLB200_SCALAR_MODEL", "lphi4")
LIB_PATH = (os.path.join(_HERE, "lib", "libclb200.so") if _SCALAR_MODEL == "lphi4"
            else os.path.join(_HERE, "lib", _SCALAR_MODEL, "libclb200.so"))

# status codes
CLB_OK = 0
CLB_EINVAL = -1
CLB_ECUDA = -2
CLB_ENOMEM = -3
CLB_ENONFINITE = -4
CLB_ETIMEOUT = -5
CLB_INIT_RESTART = 2
CLB_EUNSUPPORTED = -6
CLB_ESTATE = -7

# evolver ids, numbered as the reference's EvolverType (evolvers/evolvertype.h:37)
EVOLVERS = {"LF": 0, "VV2": 1, "VV4": 2, "VV6": 3, "VV8": 4, "VV10": 5, "VV6_2": 6,
            "PV2": 11, "PV4": 12, "PV6": 13, "PV8": 14, "PV10": 15, "PV6_2": 16}
EVOLVER_NAMES = {v: k for k, v in EVOLVERS.items()}

PREC_FP64 = 0
PREC_FP32_SPLIT = 1
PATH_FUSED = 0
PATH_REFERENCE = 1

MODEL_LPHI4 = 1
MODEL_LPHI4U1 = 2
MODEL_LPHI4SU2U1 = 3

MAX_COUPLINGS = 8
MAX_ENERGIES = 32
MAX_MEANS = 8


class Config(C.Structure):
    _fields_ = [
        ("N", C.c_int32),
        ("dx", C.c_double),
        ("dt", C.c_double),
        ("evolver", C.c_int32),
        ("expansion", C.c_int32),
        ("precision", C.c_int32),
        ("path", C.c_int32),
        ("device", C.c_int32),
        ("fixed_background", C.c_int32),
        ("omega_eos", C.c_double),
        ("H0", C.c_double),
        ("t0", C.c_double),
    ]


class ModelDesc(C.Structure):
    _fields_ = [
        ("kind", C.c_int32),
        ("n_scalars", C.c_int32),
        ("alpha", C.c_double),
        ("fStar", C.c_double),
        ("omegaStar", C.c_double),
        ("MPl", C.c_double),
        ("couplings", C.c_double * MAX_COUPLINGS),
    ]


class ScaleFactor(C.Structure):
    _fields_ = [(n, C.c_double) for n in ("aI", "aSI", "aIM", "aDotI", "aDotSI", "aDotSIM")]


IC_MAX = 8


class ICParams(C.Structure):
    """clb_ic_params."""
    _fields_ = [
        ("seed", C.c_uint64),
        ("amplitude", C.c_double),
        ("k_cutoff", C.c_double),
        ("adot", C.c_double),
        ("mass2", C.c_double * IC_MAX),
        ("fld0", C.c_double * IC_MAX),
        ("pi0", C.c_double * IC_MAX),
        ("charge", C.c_double * 4),
    ]


class Measurement(C.Structure):
    _fields_ = [
        ("aI", C.c_double),
        ("aDotI", C.c_double),
        ("hubble", C.c_double),
        ("n_energies", C.c_int32),
        ("energies", C.c_double * MAX_ENERGIES),
        ("friedmann", C.c_double * 3),
        ("n_means", C.c_int32),
        ("means", (C.c_double * 6) * MAX_MEANS),
        ("gauss_u1", C.c_double * 3),
        ("gauss_su2", C.c_double * 3),
    ]


HIST_COLS = 5


class KernelStat(C.Structure):
    _fields_ = [
        ("name", C.c_char * 40),
        ("launches", C.c_int64),
        ("timed_launches", C.c_int64),
        ("total_ms", C.c_double),
    ]


class ClbError(RuntimeError):
    """A negative status returned through the C ABI."""

    def __init__(self, code: int, message: str):
        super().__init__(f"[{code}] {message}")
        self.code = code


class BatchTuning(C.Structure):
    """clb_batch_tuning."""

    _fields_ = [
        ("tile_z", C.c_int32),
        ("tile_y", C.c_int32),
        ("sites_per_thread", C.c_int32),
        ("planes_x", C.c_int32),
        ("candidates", C.c_int32),
        ("ms_per_sweep", C.c_double),
        ("ms_default", C.c_double),
    ]


class BatchForm(C.Structure):
    """clb_batch_form."""

    _fields_ = [
        ("persistent", C.c_int32),
        ("tile_z", C.c_int32),
        ("tile_y", C.c_int32),
        ("sites_per_thread", C.c_int32),
        ("planes_x", C.c_int32),
        ("clusters", C.c_int32),
        ("cluster_blocks", C.c_int32),
        ("candidates", C.c_int32),
        ("ms_graph", C.c_double),
        ("ms_persistent", C.c_double),
    ]


class AdjointGrad(C.Structure):
    """clb_adjoint_grad."""

    _fields_ = [
        ("observable", C.c_double),
        ("dO_dcouplings", C.c_double * 8),
        ("dO_dscalefactor", C.c_double * 2),
    ]


def _declare(lib: C.CDLL, prefix: str) -> None:
    H = C.c_void_p
    dp = C.POINTER(C.c_double)
    sig = {
        "last_error": (C.c_char_p, [H]),
        "create": (C.c_int, [C.POINTER(Config), C.POINTER(ModelDesc), C.POINTER(H)]),
        "destroy": (None, [H]),
        "set_state": (C.c_int, [H, dp, dp, C.POINTER(ScaleFactor)]),
        "get_state": (C.c_int, [H, dp, dp, C.POINTER(ScaleFactor)]),
        "initialize": (C.c_int, [H, C.c_int32]),
        "evolve": (C.c_int, [H, C.c_int64]),
        "sync": (C.c_int, [H]),
        "measure": (C.c_int, [H, C.c_double, C.POINTER(Measurement)]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, f"{prefix}_{name}")
        fn.restype = res
        fn.argtypes = args
    if prefix == "clb":
        lib.clb_version.restype = C.c_char_p
        lib.clb_version.argtypes = []
        lib.clb_num_components.restype = C.c_int
        lib.clb_num_components.argtypes = [H, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]
        more = {
            "clb_history": (C.c_int, [H, dp, C.c_int64, C.POINTER(C.c_int64)]),
            "clb_set_profiling": (C.c_int, [H, C.c_int32]),
            "clb_reset_stats": (C.c_int, [H]),
            "clb_kernel_stats": (C.c_int, [H, C.POINTER(KernelStat), C.c_int32, C.POINTER(C.c_int32)]),
            "clb_last_evolve_ms": (C.c_int, [H, dp]),
            "clb_cuda_stream": (C.c_void_p, [H]),
            "clb_spectrum": (C.c_int, [H, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_double, C.c_int32,
                                       C.c_int32, dp, dp, C.POINTER(C.c_int64)]),
            "clb_gws_enable": (C.c_int, [H]),
            "clb_gws_set_state": (C.c_int, [H, dp, dp]),
            "clb_gws_get_state": (C.c_int, [H, dp, dp]),
            "clb_gw_spectrum": (C.c_int, [H, C.c_int32, C.c_int32, C.c_int32, C.c_double, C.c_int32, C.c_int32,
                                          dp, dp, C.POINTER(C.c_int64), dp]),
            "clb_forward": (C.c_int, [H, C.c_int64, C.c_int32, dp, C.c_int32, dp]),
            "clb_backward": (C.c_int, [H, C.c_int32, dp, dp, C.POINTER(AdjointGrad)]),
            "clb_generate_state": (C.c_int, [H, C.POINTER(ICParams), C.POINTER(ScaleFactor)]),
            "clb_forward_spectrum": (C.c_int, [H, C.c_int64, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32,
                                               C.c_double, C.c_int32, C.c_int32, dp, dp]),
            "clb_tangent_begin": (C.c_int, [H, dp, C.c_int32, dp, dp, C.POINTER(ScaleFactor)]),
            "clb_tangent_get_state": (C.c_int, [H, dp, dp, C.POINTER(ScaleFactor)]),
            "clb_tangent_observable": (C.c_int, [H, dp, C.c_int32, dp, dp]),
            "clb_tangent_energies": (C.c_int, [H, dp, dp]),
            "clb_tangent_spectrum": (C.c_int, [H, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_double, C.c_int32,
                                               C.c_int32, dp, dp, dp, C.POINTER(C.c_int64)]),
            "clb_tangent_end": (C.c_int, [H]),
            "clb_batch_create": (C.c_int, [C.POINTER(Config), C.POINTER(ModelDesc), C.c_int32, C.POINTER(H)]),
            "clb_batch_destroy": (None, [H]),
            "clb_batch_last_error": (C.c_char_p, [H]),
            "clb_batch_set_state": (C.c_int, [H, C.c_int32, dp, dp, C.POINTER(ScaleFactor)]),
            "clb_batch_get_state": (C.c_int, [H, C.c_int32, dp, dp, C.POINTER(ScaleFactor)]),
            "clb_batch_initialize": (C.c_int, [H, C.c_int32]),
            "clb_batch_evolve": (C.c_int, [H, C.c_int64]),
            "clb_batch_measure": (C.c_int, [H, C.c_int32, C.c_double, C.POINTER(Measurement)]),
            "clb_batch_last_evolve_ms": (C.c_int, [H, dp]),
            "clb_batch_kernel_launches": (C.c_int, [H, C.POINTER(C.c_int64)]),
            "clb_batch_autotune": (C.c_int, [H, C.c_int32, C.POINTER(BatchTuning)]),
            "clb_batch_set_tuning": (C.c_int, [H, C.c_int32, C.c_int32, C.c_int32, C.c_int32]),
            "clb_batch_get_tuning": (C.c_int, [H, C.POINTER(BatchTuning)]),
            "clb_batch_set_persistent": (C.c_int, [H, C.c_int32, C.c_int32, C.c_int32, C.c_int32]),
            "clb_batch_get_form": (C.c_int, [H, C.POINTER(BatchForm)]),
        }
        for name, (res, args) in more.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args


_LIB = None


def load() -> C.CDLL:
    """Load libclb200.so from the package tree; raise if it has not been built."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"libclb200.so not found at {LIB_PATH}: build it with `python -m cosmolattice_b200.build`"
            )
        lib = C.CDLL(LIB_PATH)
        _declare(lib, "clb")
        _LIB = lib
    return _LIB


# Exported symbols the header declares (checked by the CPU test suite).
EXPORTED = [
    "clb_version",
    "clb_last_error",
    "clb_create",
    "clb_destroy",
    "clb_num_components",
    "clb_set_state",
    "clb_get_state",
    "clb_initialize",
    "clb_evolve",
    "clb_sync",
    "clb_measure",
    "clb_spectrum",
    "clb_history",
    "clb_set_profiling",
    "clb_reset_stats",
    "clb_kernel_stats",
    "clb_last_evolve_ms",
    "clb_cuda_stream",
    "clb_forward",
    "clb_backward",
    "clb_forward_spectrum",
    "clb_generate_state",
    "clb_tangent_begin",
    "clb_tangent_get_state",
    "clb_tangent_observable",
    "clb_tangent_energies",
    "clb_tangent_spectrum",
    "clb_tangent_end",
    "clb_batch_create",
    "clb_batch_destroy",
    "clb_batch_last_error",
    "clb_batch_set_state",
    "clb_batch_get_state",
    "clb_batch_initialize",
    "clb_batch_evolve",
    "clb_batch_measure",
    "clb_batch_last_evolve_ms",
    "clb_batch_kernel_launches",
    "clb_batch_autotune",
    "clb_batch_set_tuning",
    "clb_batch_get_tuning",
    "clb_batch_set_persistent",
    "clb_batch_get_form",
    "clb_scalar_averages_noalloc",
    "clb_gws_enable",
    "clb_gws_set_state",
    "clb_gws_get_state",
    "clb_gw_spectrum",
]
