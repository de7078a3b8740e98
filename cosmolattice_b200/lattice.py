"""Python handle over the C ABI, and the reference-shaped host API built on it.

``Lattice`` owns one clb_handle (device state of one model on one GPU).  On top of it,
``ModelInitializer``, ``Evolver`` and ``Measurer`` keep the reference's call shapes
(initializers/modelinitializer.h:47-81, evolvers/evolver.h:45-155, measurements/measurer.h:87-178)
so a driver reads like source/cosmolattice.cpp.
"""
from __future__ import annotations

import ctypes as C
import math
import os
from typing import Dict, List, Optional

import numpy as np

from . import _capi
from .initializers import initial_state
from .models import Model
from .params import RunParameters

PRECISIONS = {"fp64": _capi.PREC_FP64, "fp32": _capi.PREC_FP32_SPLIT}
PATHS = {"fused": _capi.PATH_FUSED, "reference": _capi.PATH_REFERENCE}


def _dp(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def c_round(x: float) -> int:
    """C's round(): halves go away from zero (measurer.h:48-53 counts output steps with it);
    Python's round() sends them to the even neighbour instead."""
    return int(np.copysign(np.floor(abs(x) + 0.5), x))


class Lattice:
    """One lattice of one model on one GPU (a clb_handle)."""

    def __init__(self, model: Model, rp: RunParameters, precision: str = "fp64", path: str = "fused",
                 device: int = 0):
        self.lib = _capi.load()
        self.model = model
        self.rp = rp
        cfg = _capi.Config()
        cfg.N = rp.N
        cfg.dx = rp.dx
        cfg.dt = rp.dt
        cfg.evolver = rp.eType
        cfg.expansion = 1 if rp.expansion else 0
        cfg.precision = PRECISIONS[precision]
        cfg.path = PATHS[path]
        cfg.device = device
        if getattr(rp, "fixedBackground", False):
            cfg.fixed_background = 1
            cfg.omega_eos = rp.omegaEoS
            cfg.H0 = rp.H0 / model.omegaStar  # program units (fixedbackgroundexpansion.h:26)
        cfg.t0 = getattr(rp, "t0", 0.0)
        self.cfg = cfg
        self._desc = model.desc()
        h = C.c_void_p()
        rc = self.lib.clb_create(C.byref(cfg), C.byref(self._desc), C.byref(h))
        if rc != _capi.CLB_OK:
            raise _capi.ClbError(rc, self.lib.clb_last_error(None).decode())
        self.h = h
        nf, npm = C.c_int32(), C.c_int32()
        self.lib.clb_num_components(self.h, C.byref(nf), C.byref(npm))
        self.n_field_components, self.n_momentum_components = nf.value, npm.value

    def _check(self, rc: int) -> None:
        if rc != _capi.CLB_OK:
            raise _capi.ClbError(rc, self.lib.clb_last_error(self.h).decode())

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.clb_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_state(self, fields: np.ndarray, momenta: np.ndarray, sf: Optional[Dict[str, float]] = None) -> None:
        f = np.ascontiguousarray(fields, dtype=np.float64)
        p = np.ascontiguousarray(momenta, dtype=np.float64)
        n3 = self.rp.N ** 3
        if f.size != self.n_field_components * n3 or p.size != self.n_momentum_components * n3:
            raise ValueError("state arrays do not match the model's component count")
        s = None
        if sf is not None:
            s = _capi.ScaleFactor(**{k: float(sf.get(k, 0.0)) for k in ("aI", "aSI", "aIM", "aDotI", "aDotSI", "aDotSIM")})
        self._check(self.lib.clb_set_state(self.h, _dp(f), _dp(p), C.byref(s) if s is not None else None))

    def generate_state(self, params: Dict[str, object], sf: Optional[Dict[str, float]] = None) -> None:
        """clb_generate_state: the initial state drawn and transformed on the device.  params: seed,
        amplitude, k_cutoff, adot, and per matter component mass2, fld0, pi0; charge."""
        p = _capi.ICParams()
        p.seed = int(params["seed"]) & ((1 << 64) - 1)
        for k in ("amplitude", "k_cutoff", "adot"):
            setattr(p, k, float(params[k]))
        for k, n in (("mass2", _capi.IC_MAX), ("fld0", _capi.IC_MAX), ("pi0", _capi.IC_MAX), ("charge", 4)):
            v = list(params.get(k, ()))
            if len(v) > n:
                raise ValueError(f"{k}: at most {n} values")
            getattr(p, k)[:] = [float(x) for x in v] + [0.0] * (n - len(v))
        s = None
        if sf is not None:
            s = _capi.ScaleFactor(**{k: float(sf.get(k, 0.0)) for k in ("aI", "aSI", "aIM", "aDotI", "aDotSI", "aDotSIM")})
        self._check(self.lib.clb_generate_state(self.h, C.byref(p), C.byref(s) if s is not None else None))

    def get_state(self, fields: bool = True, momenta: bool = True):
        n3 = self.rp.N ** 3
        f = np.empty(self.n_field_components * n3) if fields else None
        p = np.empty(self.n_momentum_components * n3) if momenta else None
        sf = _capi.ScaleFactor()
        self._check(self.lib.clb_get_state(self.h, _dp(f) if fields else None, _dp(p) if momenta else None, C.byref(sf)))
        sfd = {k: getattr(sf, k) for k, _ in _capi.ScaleFactor._fields_}
        return f, p, sfd

    def initialize(self, correct_adot: bool = True, restart: bool = False) -> None:
        """clb_initialize; restart: the state is a restarted one (CLB_INIT_RESTART)."""
        mode = _capi.CLB_INIT_RESTART if restart else (1 if correct_adot else 0)
        self._check(self.lib.clb_initialize(self.h, mode))

    def evolve(self, n_steps: int) -> None:
        self._check(self.lib.clb_evolve(self.h, int(n_steps)))

    def sync(self) -> None:
        self._check(self.lib.clb_sync(self.h))

    def measure(self, e0: float = 1.0) -> Dict[str, object]:
        m = _capi.Measurement()
        self._check(self.lib.clb_measure(self.h, float(e0), C.byref(m)))
        return measurement_to_dict(m)

    def spectrum(self, which: int = 0, comp: int = 0, ps_type: int = 1, ps_version: int = 1, dk: float = 1.0,
                 nbins: Optional[int] = None, fold: bool = True):
        """(k, spectrum, mode counts) of scalar `comp`: which = 0 field, 1 momentum."""
        if nbins is None:
            nbins = int(np.floor(np.sqrt(3.0) / 2.0 * self.rp.N / dk))
        k = np.empty(nbins)
        v = np.empty(nbins)
        c = np.empty(nbins, dtype=np.int64)
        self._check(self.lib.clb_spectrum(self.h, which, comp, ps_type, ps_version, float(dk), nbins, 1 if fold else 0,
                                          _dp(k), _dp(v), c.ctypes.data_as(C.POINTER(C.c_int64))))
        return k, v, c

    def forward(self, n_steps: int, checkpoint_every: int, weights) -> float:
        """clb_forward: n_steps VV steps with checkpoints; returns O = sum_k w_k E_k / E_tot."""
        w = np.ascontiguousarray(weights, dtype=np.float64)
        o = C.c_double()
        self._check(self.lib.clb_forward(self.h, int(n_steps), int(checkpoint_every), _dp(w), int(w.size), C.byref(o)))
        return o.value

    def forward_spectrum(self, n_steps: int, checkpoint_every: int, which: int, comp: int, bin_weights,
                         ps_type: int = 1, ps_version: int = 1, dk: float = 1.0, fold: bool = False) -> float:
        """clb_forward_spectrum: the forward pass with O = sum_b w_b P_b, P the spectrum() of one
        component at the end state (same arguments); backward() then returns dO."""
        w = np.ascontiguousarray(bin_weights, dtype=np.float64)
        o = C.c_double()
        self._check(self.lib.clb_forward_spectrum(self.h, int(n_steps), int(checkpoint_every), int(which), int(comp),
                                                  int(ps_type), int(ps_version), float(dk), int(w.size),
                                                  1 if fold else 0, _dp(w), C.byref(o)))
        return o.value

    def backward(self, through_init: bool = True):
        """clb_backward: (fields_bar, momenta_bar, grad dict) of the last forward's observable."""
        n3 = self.rp.N ** 3
        fb, pb = np.empty(self.n_field_components * n3), np.empty(self.n_momentum_components * n3)
        g = _capi.AdjointGrad()
        self._check(self.lib.clb_backward(self.h, 1 if through_init else 0, _dp(fb), _dp(pb), C.byref(g)))
        return fb, pb, {
            "observable": g.observable,
            "dO_dcouplings": [g.dO_dcouplings[i] for i in range(8)],
            "dO_daI": g.dO_dscalefactor[0],
            "dO_daDotI": g.dO_dscalefactor[1],
        }

    def tangent_begin(self, couplings_dot, fields_dot=None, momenta_dot=None,
                      sf_dot: Optional[Dict[str, float]] = None) -> None:
        """clb_tangent_begin: from now on evolve the derivative of the state along the coupling
        direction couplings_dot (model.couplings() order) alongside the state."""
        n3 = self.rp.N ** 3
        cd = np.ascontiguousarray(couplings_dot, dtype=np.float64)
        f = p = None
        if fields_dot is not None:
            f = np.ascontiguousarray(fields_dot, dtype=np.float64)
            if f.size != self.n_field_components * n3:
                raise ValueError("fields_dot does not match the model's component count")
        if momenta_dot is not None:
            p = np.ascontiguousarray(momenta_dot, dtype=np.float64)
            if p.size != self.n_momentum_components * n3:
                raise ValueError("momenta_dot does not match the model's component count")
        s = None
        if sf_dot is not None:
            s = _capi.ScaleFactor(**{k: float(sf_dot.get(k, 0.0)) for k in ("aI", "aSI", "aIM", "aDotI", "aDotSI", "aDotSIM")})
        self._check(self.lib.clb_tangent_begin(self.h, _dp(cd), int(cd.size), _dp(f) if f is not None else None,
                                               _dp(p) if p is not None else None, C.byref(s) if s is not None else None))

    def tangent_get_state(self):
        """(fields_dot, momenta_dot, scale-factor tangents) of the tangent-linear form."""
        n3 = self.rp.N ** 3
        f = np.empty(self.n_field_components * n3)
        p = np.empty(self.n_momentum_components * n3)
        sf = _capi.ScaleFactor()
        self._check(self.lib.clb_tangent_get_state(self.h, _dp(f), _dp(p), C.byref(sf)))
        return f, p, {k: getattr(sf, k) for k, _ in _capi.ScaleFactor._fields_}

    def tangent_observable(self, weights):
        """(O, dO/dcoupling) for O = sum_k w_k E_k / E_tot at the current state."""
        w = np.ascontiguousarray(weights, dtype=np.float64)
        o, do = C.c_double(), C.c_double()
        self._check(self.lib.clb_tangent_observable(self.h, _dp(w), int(w.size), C.byref(o), C.byref(do)))
        return o.value, do.value

    def tangent_energies(self):
        """(E, dE): the 11 energies of tangent_observable and their derivatives."""
        e, de = np.empty(11), np.empty(11)
        self._check(self.lib.clb_tangent_energies(self.h, _dp(e), _dp(de)))
        return e, de

    def tangent_spectrum(self, which: int = 0, comp: int = 0, ps_type: int = 1, ps_version: int = 1, dk: float = 1.0,
                         nbins: Optional[int] = None, fold: bool = True):
        """(k, spectrum, d spectrum, mode counts): spectrum() and its derivative along the tangent."""
        if nbins is None:
            nbins = int(np.floor(np.sqrt(3.0) / 2.0 * self.rp.N / dk))
        k, v, dv = np.empty(nbins), np.empty(nbins), np.empty(nbins)
        c = np.empty(nbins, dtype=np.int64)
        self._check(self.lib.clb_tangent_spectrum(self.h, which, comp, ps_type, ps_version, float(dk), nbins,
                                                  1 if fold else 0, _dp(k), _dp(v), _dp(dv),
                                                  c.ctypes.data_as(C.POINTER(C.c_int64))))
        return k, v, dv, c

    def tangent_end(self) -> None:
        self._check(self.lib.clb_tangent_end(self.h))

    # ---- gravitational waves (clb_gws_*; the reference's GW sector with doLFforGWs) ----
    def gws_enable(self) -> None:
        self._check(self.lib.clb_gws_enable(self.h))
        self.gws_on = True

    gws_on = False  # the GW sector is enabled on this lattice

    def gws_set_state(self, u=None, pi=None) -> None:
        n = 5 * self.rp.N ** 3
        args = []
        for a in (u, pi):
            if a is None:
                args.append(None)
            else:
                a = np.ascontiguousarray(a, dtype=np.float64)
                if a.size != n:
                    raise ValueError("GW arrays hold 5 x N^3 values")
                args.append(a)
        self._check(self.lib.clb_gws_set_state(self.h, *[_dp(a) if a is not None else None for a in args]))

    def gws_get_state(self):
        n = 5 * self.rp.N ** 3
        u, p = np.empty(n), np.empty(n)
        self._check(self.lib.clb_gws_get_state(self.h, _dp(u), _dp(p)))
        return u, p

    def gw_spectrum(self, prj_type: int = 2, ps_type: int = 1, ps_version: int = 1, dk: float = 1.0,
                    nbins: Optional[int] = None, fold: bool = True):
        """(k, d(rho_GW/rho)/dlog k per bin, mode counts, rho_GW/rho) of clb_gw_spectrum."""
        if nbins is None:
            nbins = int(math.floor(math.sqrt(3.0) / 2.0 * self.rp.N / dk))
        k, v = np.empty(nbins), np.empty(nbins)
        c = np.empty(nbins, dtype=np.int64)
        frac = C.c_double()
        self._check(self.lib.clb_gw_spectrum(self.h, int(prj_type), int(ps_type), int(ps_version), float(dk), nbins,
                                             1 if fold else 0, _dp(k), _dp(v),
                                             c.ctypes.data_as(C.POINTER(C.c_int64)), C.byref(frac)))
        return k, v, c, frac.value

    def history(self) -> np.ndarray:
        """Per-step rows (a, aDot, <pi^2>, <grad^2>, <V>) of the last evolve call."""
        n = C.c_int64()
        self._check(self.lib.clb_history(self.h, None, 0, C.byref(n)))
        out = np.empty((n.value, _capi.HIST_COLS))
        if n.value:
            self._check(self.lib.clb_history(self.h, _dp(out), n.value, C.byref(n)))
        return out

    def set_profiling(self, on: bool) -> None:
        self._check(self.lib.clb_set_profiling(self.h, 1 if on else 0))

    def reset_stats(self) -> None:
        self._check(self.lib.clb_reset_stats(self.h))

    def kernel_stats(self) -> Dict[str, Dict[str, float]]:
        arr = (_capi.KernelStat * 16)()
        n = C.c_int32()
        self._check(self.lib.clb_kernel_stats(self.h, arr, 16, C.byref(n)))
        return {arr[i].name.decode(): {"launches": arr[i].launches, "timed_launches": arr[i].timed_launches,
                                       "total_ms": arr[i].total_ms} for i in range(min(n.value, 16))}

    def last_evolve_ms(self) -> float:
        v = C.c_double()
        self._check(self.lib.clb_last_evolve_ms(self.h, C.byref(v)))
        return v.value

    def cuda_stream(self) -> int:
        return self.lib.clb_cuda_stream(self.h) or 0


def measurement_to_dict(m: _capi.Measurement) -> Dict[str, object]:
    return {
        "aI": m.aI,
        "aDotI": m.aDotI,
        "hubble": m.hubble,
        "energies": [m.energies[i] for i in range(m.n_energies)],
        "friedmann": [m.friedmann[i] for i in range(3)],
        "means": [[m.means[f][j] for j in range(6)] for f in range(m.n_means)],
        "gauss_u1": [m.gauss_u1[i] for i in range(3)],
        "gauss_su2": [m.gauss_su2[i] for i in range(3)],
    }


class ModelInitializer:
    """ModelInitializer::initialize (modelinitializer.h:47-81) for scalar-singlet models."""

    def __init__(self, model: Model, lSide: float, seed: str):
        self.model = model

    def initialize(self, model: Model, rp: RunParameters, lattice: Lattice) -> None:
        fields, momenta, aI, aDot = initial_state(model, rp)
        lattice.set_state(fields, momenta, {"aI": aI, "aSI": aI, "aIM": aI, "aDotI": aDot, "aDotSI": aDot})
        lattice.initialize(correct_adot=True)


class Evolver:
    """Evolver<Model> (evolver.h:45-155): LF and VV2-VV10 over a Lattice."""

    def __init__(self, model: Model, rp: RunParameters, lattice: Lattice):
        self.lattice = lattice

    def evolve(self, model: Model, t_minus_t0: float) -> None:
        self.lattice.evolve(1)

    def evolve_n(self, n: int) -> None:
        self.lattice.evolve(n)

    def sync(self, model: Model, t_minus_t0: float) -> None:
        self.lattice.sync()


class Measurer:
    """Frequent output of Measurer::measure (measurer.h:87-121) as reference text files:
    average_energies.txt, average_energy_conservation.txt, average_scale_factor.txt and one
    average_scalar_<i>.txt per singlet, numbers formatted with 15 significant digits
    (measurementssaverstd.h:61-69)."""

    def __init__(self, model: Model, rp: RunParameters, outdir: Optional[str] = None):
        self.model = model
        self.rp = rp
        self.outdir = outdir if outdir is not None else rp.outFn
        self.outputFreq = max(1, c_round(rp.tOutFreq / rp.dt))
        self.spectraFreq = max(1, c_round(rp.tOutInfreq / rp.dt))  # measurer.h:48-53
        self.e0 = None
        self.files: Dict[str, object] = {}
        self.history: List[Dict[str, object]] = []
        if self.outdir:
            os.makedirs(self.outdir, exist_ok=True)

    def _mean_files(self):
        """Names of the per-field means files, in the order of the measurement's means rows
        (scalarsingletmeasurer.h, complexscalarmeasurer.h:40-52, u1measurer.h:45-55)."""
        m = self.model
        if getattr(m, "NSU2", 0):  # + su2doubletmeasurer.h:42, su2measurer.h:39
            return ["scalar_0", "cmplx_scalar_0_0", "cmplx_scalar_0_1", "norm_cmplx_scalar_0", "norm_SU2Doublet_0",
                    "norm_U1_0", "norm_SU2_0"]
        if getattr(m, "NU1", 0):
            return ["cmplx_scalar_0_0", "cmplx_scalar_0_1", "norm_cmplx_scalar_0", "norm_U1_0"]
        return [f"scalar_{i}" for i in range(m.Ns)]

    def _headers(self):
        # energiesmeasurer.h:127-150: singlets, complex scalars, SU(2) doublets, U(1), SU(2), the
        # potential terms, E_tot
        m = self.model
        en = ["t"]
        for i in range(m.Ns):
            en += [f"E^kin_scal{i}", f"E^grad_scal{i}"]
        for i in range(getattr(m, "NCs", 0)):
            en += [f"E^kin_cmplxscal{i}", f"E^grad_cmplxscal{i}"]
        for i in range(getattr(m, "NSU2Doublet", 0)):
            en += ["E^kin_SU2matter", "E^grad_SU2matter"]
        for i in range(getattr(m, "NU1", 0)):
            en += [f"E^kin_U1{i}", f"E^grad_U1{i}"]
        for i in range(getattr(m, "NSU2", 0)):
            en += ["E^kin_SU2", "E^grad_SU2"]
        en += [f"Vpot_term_{k}" for k in range(m.NPotTerms)] + ["E_tot"]
        cons = ["t"] + (["rel_diff_friedmann", "LHS_friedmann", "RHS_friedmann"] if self.rp.expansion else ["energy_cons"])
        means = ["t", "<phi>", "<pi>", "<phi^2>", "<pi^2>", "rms(phi)", "rms(pi)"]
        means_eb = ["t", "<|E|>", "<|B|>", "<|E|^2>", "<|B|^2>", "rms(|E|)", "rms(|B|)"]
        h = {
            "energies": en,
            "energy_conservation": cons,
            "scale_factor": ["t", "a", "aDot", "H"],
            **{name: (means_eb if name.startswith(("norm_U1", "norm_SU2_")) else means) for name in self._mean_files()},
        }
        gauss = ["t", "av|LHS-RHS|_over_av|LHS+RHS|", "av|LHS|", "av|RHS|"]
        if getattr(m, "NU1", 0):
            h["gauss_U1_0"] = gauss
        if getattr(m, "NSU2", 0):
            h["gauss_SU2_0"] = gauss
        return h

    def _write(self, name: str, values: List[float]) -> None:
        if not self.outdir:
            return
        if name not in self.files:
            path = os.path.join(self.outdir, f"average_{name}.txt")
            if os.path.exists(path) and not self.rp.appendMode and not self.rp.overwriteMode:
                raise FileExistsError(f'Refusing to overwrite existing output file "{path}". Set '
                                      "'appendToFiles = true' to append, or 'overwriteFiles = true' to delete.")
            fh = open(path, "a" if self.rp.appendMode else "w")
            if self.rp.printHeaders and not self.rp.appendMode:
                fh.write("#" + "    ".join(self._headers()[name]) + "\n")
            self.files[name] = fh
        fh = self.files[name]
        fh.write("    ".join(f"{v:.15g}" for v in values) + "\n")
        fh.flush()

    def are_we_measuring(self, n: int) -> bool:
        return n % self.outputFreq == 0

    def are_we_measuring_spectra(self, n: int) -> bool:
        return n % self.spectraFreq == 0

    def _spectra_sets(self):
        """(file name, [(which, comp, gauge-electric)...] summed into column 1, same for column 2) per
        measured field (scalarsingletmeasurer.h:74-83, complexscalarmeasurer.h:75-90,
        su2doubletmeasurer.h, u1measurer.h:91-104)."""
        m = self.model
        if getattr(m, "NSU2", 0):
            return [("scalar_0", [(0, 0)], [(1, 0)]),
                    ("norm_cmplx_scalar_0", [(0, 1), (0, 2)], [(1, 1), (1, 2)]),
                    ("norm_SU2Doublet_scalar_0", [(0, c) for c in range(3, 7)], [(1, c) for c in range(3, 7)]),
                    ("norm_U1_0", [(1, 7), (1, 8), (1, 9)], None)]
        if getattr(m, "NU1", 0):
            return [("norm_cmplx_scalar_0", [(0, 0), (0, 1)], [(1, 0), (1, 1)]),
                    ("norm_U1_0", [(1, 2), (1, 3), (1, 4)], None)]
        return [(f"scalar_{i}", [(0, i)], [(1, i)]) for i in range(m.Ns)]

    def measure_spectra(self, t: float, lattice: Lattice) -> None:
        """SpectrumSaverStd::save (spectrumsaverstd.h:54-96), verbosity 0: one line per bin with the
        bin centre times kIR and the spectra of the measured quantity, a blank line per time."""
        if not self.outdir:
            return
        rp = self.rp
        for name, cols1, cols2 in self._spectra_sets():
            cols = []
            k = None
            for group in (cols1, cols2):
                if group is None:
                    continue
                acc = None
                for which, comp in group:
                    kk, v, _ = lattice.spectrum(which=which, comp=comp, ps_type=rp.powerSpectrumType,
                                                ps_version=rp.powerSpectrumVersion, dk=rp.deltaKBin,
                                                nbins=rp.nBinsSpectra)
                    acc = v if acc is None else acc + v
                    k = kk
                cols.append(acc)
            key = "spectra_" + name
            if key not in self.files:
                path = os.path.join(self.outdir, key + ".txt")
                if os.path.exists(path) and not rp.appendMode and not rp.overwriteMode:
                    raise FileExistsError(f'Refusing to overwrite existing output file "{path}".')
                fh = open(path, "a" if rp.appendMode else "w")
                if rp.printHeaders and not rp.appendMode:
                    fh.write("1:binCentralValue " + " ".join(f"{i + 2}:PS" for i in range(len(cols))) + "\n")
                self.files[key] = fh
            fh = self.files[key]
            centres = (np.arange(rp.nBinsSpectra) + 0.5) * rp.deltaKBin * rp.kIR
            for b in range(rp.nBinsSpectra):
                fh.write(" ".join(f"{x:.15g}" for x in [centres[b]] + [c[b] for c in cols]) + "\n")
            fh.write("\n")
            fh.flush()

    def measure_gws(self, t: float, lattice: Lattice) -> None:
        """GWsMeasurer::measureSpectra (gwsmeasurer.h:41-53): spectra_energy_gws.txt (the bin
        centre times kIR and d(rho_GW/rho)/dlog k) and average_energies_gws.txt (t, rhoGW/rho,
        rhoGW)."""
        if not self.outdir:
            return
        rp = self.rp
        k, v, c, frac = lattice.gw_spectrum(prj_type=rp.GWprojectorType, ps_type=rp.powerSpectrumType,
                                            ps_version=rp.powerSpectrumVersion, dk=rp.deltaKBin, nbins=rp.nBinsSpectra)
        key = "spectra_energy_gws"
        if key not in self.files:
            fh = open(os.path.join(self.outdir, key + ".txt"), "a" if rp.appendMode else "w")
            if rp.printHeaders and not rp.appendMode:
                fh.write("1:binCentralValue 2:PS\n")
            self.files[key] = fh
        fh = self.files[key]
        centres = (np.arange(rp.nBinsSpectra) + 0.5) * rp.deltaKBin * rp.kIR
        for b in range(rp.nBinsSpectra):
            fh.write(f"{centres[b]:.15g} {v[b]:.15g}\n")
        fh.write("\n")
        fh.flush()
        rho = lattice.measure(self.e0 if self.e0 is not None else 1.0)["energies"][-1]
        if "energies_gws" not in self.files:
            path = os.path.join(self.outdir, "average_energies_gws.txt")
            fh = open(path, "a" if rp.appendMode else "w")
            if rp.printHeaders and not rp.appendMode:
                fh.write("#t    rhoGW_over_rho    rhoGW\n")
            self.files["energies_gws"] = fh
        self.files["energies_gws"].write(f"{t:.15g}    {frac:.15g}    {frac * rho:.15g}\n")
        self.files["energies_gws"].flush()

    def measure(self, n: int, t: float, lattice: Lattice) -> Dict[str, object]:
        first = self.e0 is None
        m = lattice.measure(self.e0 if self.e0 is not None else 1.0)
        etot = m["energies"][-1]
        if first:
            self.e0 = etot
            if not self.rp.expansion:
                m["friedmann"][0] = 0.0
        m["t"] = t
        self.history.append(m)
        self._write("energies", [t] + m["energies"])
        self._write("energy_conservation", [t] + (m["friedmann"] if self.rp.expansion else m["friedmann"][:1]))
        if self.rp.expansion:
            self._write("scale_factor", [t, m["aI"], m["aDotI"], m["hubble"]])
        for name, row in zip(self._mean_files(), m["means"]):
            self._write(name, [t] + row)
        if getattr(self.model, "NU1", 0):
            self._write("gauss_U1_0", [t] + m["gauss_u1"])
        if getattr(self.model, "NSU2", 0):
            self._write("gauss_SU2_0", [t] + m["gauss_su2"])
        return m

    def close(self) -> None:
        for fh in self.files.values():
            fh.close()
        self.files = {}


def run(par, model_name: str = "lphi4", precision: str = "fp64", path: str = "fused", outdir: Optional[str] = None,
        lattice_factory=None):
    """The reference main loop (source/cosmolattice.cpp:168-201) over the GPU library.
    lattice_factory(model, rp), if given, makes the lattice the loop drives instead (an object with
    Lattice's set_state / initialize / evolve / sync / measure / spectrum)."""
    from .models import MODELS
    from .params import RunParameters

    rp = RunParameters(par)
    model = MODELS[model_name](par, rp)
    lattice = (lattice_factory(model, rp) if lattice_factory is not None
               else Lattice(model, rp, precision=precision, path=path))
    if rp.withGWs:
        lattice.gws_enable()
    measurer = Measurer(model, rp, outdir)
    ModelInitializer(model, rp.lSide, rp.baseSeed).initialize(model, rp, lattice)
    evolver = Evolver(model, rp, lattice)
    t = rp.t0
    i = 0
    while t < rp.tMax - rp.dt / 2.0:
        freq = measurer.are_we_measuring(i)
        infreq = measurer.are_we_measuring_spectra(i)
        if freq or infreq:
            evolver.sync(model, t - rp.t0)
        if freq:
            measurer.measure(i, t, lattice)
        if infreq:
            measurer.measure_spectra(t, lattice)
            if rp.withGWs:
                measurer.measure_gws(t, lattice)
        # advance to the next measurement in one device call
        n = min(measurer.outputFreq - (i % measurer.outputFreq), measurer.spectraFreq - (i % measurer.spectraFreq))
        n_left = c_round((rp.tMax - t) / rp.dt)
        n = max(1, min(n, n_left))
        evolver.evolve_n(n)
        t += n * rp.dt
        i += n
    measurer.close()
    return measurer.history, lattice
