"""ctypes binding of the CPU parity oracle (oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and bench.py's CPU
baseline, never by the product package.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")

_LIB = None


def build() -> str:
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def load():
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            build()
        import cosmolattice_b200._capi as capi

        lib = C.CDLL(LIB_PATH)
        H = C.c_void_p
        dp = C.POINTER(C.c_double)
        sig = {
            "orc_last_error": (C.c_char_p, [H]),
            "orc_create": (C.c_int, [C.POINTER(capi.Config), C.POINTER(capi.ModelDesc), C.POINTER(H)]),
            "orc_destroy": (None, [H]),
            "orc_set_state": (C.c_int, [H, dp, dp, C.POINTER(capi.ScaleFactor)]),
            "orc_get_state": (C.c_int, [H, dp, dp, C.POINTER(capi.ScaleFactor)]),
            "orc_initialize": (C.c_int, [H, C.c_int32]),
            "orc_evolve": (C.c_int, [H, C.c_int64]),
            "orc_sync": (C.c_int, [H]),
            "orc_measure": (C.c_int, [H, C.c_double, C.POINTER(capi.Measurement)]),
            "orc_num_threads": (C.c_int, []),
            "orc_set_scalar_model": (C.c_int, [H, C.c_int32]),
            "orc_gws_enable": (C.c_int, [H]),
            "orc_gws_set_state": (C.c_int, [H, dp, dp]),
            "orc_gws_get_state": (C.c_int, [H, dp, dp]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = lib
    return _LIB


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class OracleLattice:
    """Same methods as cosmolattice_b200.Lattice, computed by the CPU oracle."""

    def __init__(self, model, rp, precision="fp64", path="reference", device=0):
        import cosmolattice_b200._capi as capi

        self.capi = capi
        self.lib = load()
        self.rp = rp
        cfg = capi.Config()
        cfg.N = rp.N
        cfg.dx = rp.dx
        cfg.dt = rp.dt
        cfg.evolver = rp.eType
        cfg.expansion = 1 if rp.expansion else 0
        cfg.precision = capi.PREC_FP64
        cfg.path = capi.PATH_REFERENCE
        if getattr(rp, "fixedBackground", False):
            cfg.fixed_background = 1
            cfg.omega_eos = rp.omegaEoS
            cfg.H0 = rp.H0 / model.omegaStar
        cfg.t0 = getattr(rp, "t0", 0.0)
        self._desc = model.desc()
        h = C.c_void_p()
        rc = self.lib.orc_create(C.byref(cfg), C.byref(self._desc), C.byref(h))
        if rc != 0:
            raise RuntimeError(self.lib.orc_last_error(None).decode())
        self.h = h
        if getattr(model, "scalar_header", "lphi4") == "tanh2":  # the tanh2 potential restated in oracle.cpp
            self._check(self.lib.orc_set_scalar_model(self.h, 1))
        self.n_components = getattr(model, "n_components", model.Ns)
        self.n_momentum_components = getattr(model, "n_momentum_components", self.n_components)

    def gws_enable(self):
        self._check(self.lib.orc_gws_enable(self.h))

    def gws_set_state(self, u, pi):
        import numpy as np

        u = np.ascontiguousarray(u, dtype=np.float64)
        pi = np.ascontiguousarray(pi, dtype=np.float64)
        self._check(self.lib.orc_gws_set_state(self.h, _dp(u), _dp(pi)))

    def gws_get_state(self):
        import numpy as np

        n = 5 * self.rp.N ** 3
        u, p = np.empty(n), np.empty(n)
        self._check(self.lib.orc_gws_get_state(self.h, _dp(u), _dp(p)))
        return u, p

    def close(self):
        if getattr(self, "h", None):
            self.lib.orc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc):
        if rc != 0:
            raise RuntimeError(self.lib.orc_last_error(self.h).decode())

    def set_state(self, fields, momenta, sf=None):
        f = np.ascontiguousarray(fields, dtype=np.float64)
        p = np.ascontiguousarray(momenta, dtype=np.float64)
        s = None
        if sf is not None:
            s = self.capi.ScaleFactor(**{k: float(sf.get(k, 0.0)) for k in ("aI", "aSI", "aIM", "aDotI", "aDotSI", "aDotSIM")})
        self._check(self.lib.orc_set_state(self.h, _dp(f), _dp(p), C.byref(s) if s is not None else None))

    def get_state(self, fields=True, momenta=True):
        n3 = self.rp.N ** 3
        f = np.empty(self.n_components * n3)
        p = np.empty(self.n_momentum_components * n3)
        sf = self.capi.ScaleFactor()
        self._check(self.lib.orc_get_state(self.h, _dp(f), _dp(p), C.byref(sf)))
        return f, p, {k: getattr(sf, k) for k, _ in self.capi.ScaleFactor._fields_}

    def initialize(self, correct_adot=True, restart=False):
        """orc_initialize; restart: no aDot correction and the GW leapfrog unsynced (mode 2, as
        CLB_INIT_RESTART)."""
        self._check(self.lib.orc_initialize(self.h, 2 if restart else (1 if correct_adot else 0)))

    def evolve(self, n):
        self._check(self.lib.orc_evolve(self.h, int(n)))

    def sync(self):
        self._check(self.lib.orc_sync(self.h))

    def measure(self, e0=1.0):
        from cosmolattice_b200.lattice import measurement_to_dict

        m = self.capi.Measurement()
        self._check(self.lib.orc_measure(self.h, float(e0), C.byref(m)))
        return measurement_to_dict(m)


def num_threads() -> int:
    return load().orc_num_threads()
