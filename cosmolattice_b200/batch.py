"""Batched ensembles of independent one-field lphi4 lattices over the C ABI (clb_batch_*)."""
from __future__ import annotations

import ctypes as C
from typing import Dict, List, Optional, Sequence

import numpy as np

from . import _capi
from .lattice import PRECISIONS, measurement_to_dict
from .models import Model
from .params import RunParameters


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double)) if a is not None else None


class LatticeBatch:
    """Members (model, run parameters) advanced together; they must share dt, evolver and
    expansion.  Methods take the member index where the single-lattice ones take none."""

    def __init__(self, members: Sequence[tuple], precision: str = "fp32", device: int = 0):
        self.lib = _capi.load()
        n = len(members)
        cfgs = (_capi.Config * n)()
        self._descs = (_capi.ModelDesc * n)()
        self.members = list(members)
        for i, (model, rp) in enumerate(members):
            c = cfgs[i]
            c.N, c.dx, c.dt, c.evolver = rp.N, rp.dx, rp.dt, rp.eType
            c.expansion = 1 if rp.expansion else 0
            c.precision = PRECISIONS[precision]
            c.path = _capi.PATH_FUSED
            c.device = device
            self._descs[i] = model.desc()
        h = C.c_void_p()
        rc = self.lib.clb_batch_create(cfgs, self._descs, n, C.byref(h))
        if rc != _capi.CLB_OK:
            raise _capi.ClbError(rc, self.lib.clb_batch_last_error(None).decode())
        self.h = h

    def _check(self, rc):
        if rc != _capi.CLB_OK:
            raise _capi.ClbError(rc, self.lib.clb_batch_last_error(self.h).decode())

    def close(self):
        if getattr(self, "h", None):
            self.lib.clb_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_state(self, i: int, fields, momenta, sf: Optional[Dict[str, float]] = None):
        f = np.ascontiguousarray(fields, dtype=np.float64)
        p = np.ascontiguousarray(momenta, dtype=np.float64)
        N = self.members[i][1].N
        if f.size != N ** 3 or p.size != N ** 3:
            raise ValueError("member arrays must hold N^3 values")
        s = None
        if sf is not None:
            s = _capi.ScaleFactor(**{k: float(sf.get(k, 0.0)) for k in ("aI", "aSI", "aIM", "aDotI", "aDotSI", "aDotSIM")})
        self._check(self.lib.clb_batch_set_state(self.h, i, _dp(f), _dp(p), C.byref(s) if s is not None else None))

    def get_state(self, i: int):
        N = self.members[i][1].N
        f, p = np.empty(N ** 3), np.empty(N ** 3)
        sf = _capi.ScaleFactor()
        self._check(self.lib.clb_batch_get_state(self.h, i, _dp(f), _dp(p), C.byref(sf)))
        return f, p, {k: getattr(sf, k) for k, _ in _capi.ScaleFactor._fields_}

    def initialize(self, correct_adot: bool = True):
        self._check(self.lib.clb_batch_initialize(self.h, 1 if correct_adot else 0))

    def evolve(self, n_steps: int):
        self._check(self.lib.clb_batch_evolve(self.h, int(n_steps)))

    def measure(self, i: int, e0: float = 1.0):
        m = _capi.Measurement()
        self._check(self.lib.clb_batch_measure(self.h, i, float(e0), C.byref(m)))
        return measurement_to_dict(m)

    def last_evolve_ms(self) -> float:
        v = C.c_double()
        self._check(self.lib.clb_batch_last_evolve_ms(self.h, C.byref(v)))
        return v.value

    def kernel_launches(self) -> int:
        v = C.c_int64()
        self._check(self.lib.clb_batch_kernel_launches(self.h, C.byref(v)))
        return v.value

    @staticmethod
    def _tuning_dict(t) -> Dict[str, object]:
        return {k: getattr(t, k) for k, _ in _capi.BatchTuning._fields_}

    def autotune(self, reps: int = 5) -> Dict[str, object]:
        """clb_batch_autotune: time every sweep configuration on this ensemble and keep the fastest."""
        t = _capi.BatchTuning()
        self._check(self.lib.clb_batch_autotune(self.h, int(reps), C.byref(t)))
        return self._tuning_dict(t)

    def set_tuning(self, tile_z: int, tile_y: int, planes_x: int, sites_per_thread: int = 1) -> None:
        """Fix the sweep configuration: tile sites along z and y, x-planes per block, z sites per thread."""
        self._check(self.lib.clb_batch_set_tuning(self.h, int(tile_z), int(tile_y), int(sites_per_thread),
                                                  int(planes_x)))

    def tuning(self) -> Dict[str, object]:
        t = _capi.BatchTuning()
        self._check(self.lib.clb_batch_get_tuning(self.h, C.byref(t)))
        return self._tuning_dict(t)

    def set_persistent(self, tile_z: int, tile_y: int, planes_x: int, sites_per_thread: int = 1) -> None:
        """Run every evolve call as one persistent launch of thread-block clusters with this tile."""
        self._check(self.lib.clb_batch_set_persistent(self.h, int(tile_z), int(tile_y), int(sites_per_thread),
                                                      int(planes_x)))

    def form(self) -> Dict[str, object]:
        """clb_batch_form: persistent or per-stage graph form, the persistent tile and cluster count,
        and the autotuner's per-step times of both forms."""
        f = _capi.BatchForm()
        self._check(self.lib.clb_batch_get_form(self.h, C.byref(f)))
        return {k: getattr(f, k) for k, _ in _capi.BatchForm._fields_}
