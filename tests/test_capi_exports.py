"""The C-ABI library loads on a CPU-only host and exports every function include/*.h declares."""
import ctypes
import glob
import os
import re

from cosmolattice_b200 import _capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for hdr in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(hdr).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        text = re.sub(r"//[^\n]*", "", text)
        for m in re.finditer(r"\b(clb_[A-Za-z0-9_]+)\s*\(", text):
            names.add(m.group(1))
    return names


def test_header_declares_functions():
    names = declared_functions()
    assert {"clb_create", "clb_evolve", "clb_destroy", "clb_measure"} <= names


def test_library_exports_all_declared_symbols():
    lib = ctypes.CDLL(_capi.LIB_PATH)
    missing = [n for n in sorted(declared_functions()) if not hasattr(lib, n)]
    assert not missing, f"symbols declared in include/*.h but not exported: {missing}"


def test_python_binding_lists_header():
    assert set(_capi.EXPORTED) <= declared_functions()


def test_version_and_error_without_gpu():
    lib = _capi.load()
    assert b"sm_100a" in lib.clb_version()
    # a bad config is rejected before any device call
    cfg = _capi.Config(N=1, dx=1.0, dt=0.1, evolver=1, expansion=0, precision=0, path=0, device=0)
    md = _capi.ModelDesc(kind=_capi.MODEL_LPHI4, n_scalars=1, alpha=1, fStar=1, omegaStar=1, MPl=1)
    h = ctypes.c_void_p()
    rc = lib.clb_create(ctypes.byref(cfg), ctypes.byref(md), ctypes.byref(h))
    assert rc == _capi.CLB_EINVAL
    assert b"N must be" in lib.clb_last_error(None)
    cfg.N = 8
    md.kind = 99
    assert lib.clb_create(ctypes.byref(cfg), ctypes.byref(md), ctypes.byref(h)) == _capi.CLB_EUNSUPPORTED
    md.kind = _capi.MODEL_LPHI4
    cfg.evolver = 9  # RK3_4: not on this library's path
    assert lib.clb_create(ctypes.byref(cfg), ctypes.byref(md), ctypes.byref(h)) == _capi.CLB_EUNSUPPORTED
    cfg.evolver = 1
    cfg.dt = 0.0
    assert lib.clb_create(ctypes.byref(cfg), ctypes.byref(md), ctypes.byref(h)) == _capi.CLB_EINVAL


def test_scalar_model_variants_export_the_same_symbols():
    # each scalar-singlet model header the build compiles besides lphi4 (csrc/models/) gives a
    # complete library of its own
    from cosmolattice_b200.build import SCALAR_VARIANTS, variant_lib

    for name in SCALAR_VARIANTS:
        lib = ctypes.CDLL(variant_lib(name))
        missing = [n for n in sorted(declared_functions()) if not hasattr(lib, n)]
        assert not missing, (name, missing)


def test_model_headers_have_the_reference_shape():
    # every model header defines potentialTerms, potDeriv and potDeriv2 per Tag, like the
    # reference's headers (models/lphi4.h:154-226, models/tanh2.h)
    for name in ("lphi4", "tanh2"):
        text = open(os.path.join(ROOT, "cosmolattice_b200", "csrc", "models", f"{name}.h")).read()
        for fn in ("potentialTerms", "potDeriv", "potDeriv2"):
            assert f"{fn}(Tag<0>" in text and f"{fn}(Tag<1>" in text, (name, fn)
