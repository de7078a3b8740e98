import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the product kernels")


def make_scalar_case(N=16, evolver="VV2", expansion=True, model="lphi4_1f", dt=0.01, seed="t", amp=1e-3,
                     kcut=None, extra=None):
    """Parameter set, run parameters, model and initial state of a small lphi4 lattice."""
    from cosmolattice_b200 import MODELS, ParameterParser, RunParameters
    from cosmolattice_b200.initializers import scalar_initial_state

    params = {
        "N": N, "kIR": 1.0, "dt": dt, "evolver": evolver, "expansion": "true" if expansion else "false",
        "lambda": 1.0, "initial_amplitudes": "5.6964e18" if model == "lphi4_1f" else "5.6964e18 0",
        "initial_momenta": "0" if model == "lphi4_1f" else "0 0",
        "fluct_amplitude": amp, "kCutOff": kcut if kcut is not None else N / 4.0, "baseSeed": seed,
    }
    if model == "lphi4":
        params["q"] = 1.5
        params["initial_amplitudes"] = "5.6964e18 1e17"
    if extra:
        params.update(extra)
    par = ParameterParser(params=params)
    rp = RunParameters(par)
    m = MODELS[model](par, rp)
    f, p, aI, aD = scalar_initial_state(m, rp)
    sf = {"aI": aI, "aSI": aI, "aIM": aI, "aDotI": aD, "aDotSI": aD}
    return par, rp, m, f, p, sf


def make_u1_case(N=12, evolver="VV2", expansion=True, dt=0.01, seed="u", amp=1e-2, gU1=0.5, kcut=None,
                 extra=None):
    """Parameter set, run parameters, lphi4U1 model and RandomWithMatter initial state."""
    from cosmolattice_b200 import MODELS, ParameterParser, RunParameters
    from cosmolattice_b200.initializers import u1_initial_state

    params = {
        "N": N, "kIR": 1.0, "dt": dt, "evolver": evolver, "expansion": "true" if expansion else "false",
        "lambda": 1.0, "cmplx_field_initial_norm": "5.6964e18", "cmplx_momentum_initial_norm": "0",
        "gU1s": gU1, "CSU1_charges": 1, "fluct_amplitude": amp,
        "kCutOff": kcut if kcut is not None else N / 4.0, "baseSeed": seed,
    }
    if extra:
        params.update(extra)
    par = ParameterParser(params=params)
    rp = RunParameters(par)
    m = MODELS["lphi4U1"](par, rp)
    f, p, aI, aD = u1_initial_state(m, rp)
    sf = {"aI": aI, "aSI": aI, "aIM": aI, "aDotI": aD, "aDotSI": aD}
    return par, rp, m, f, p, sf


def make_su2_case(N=8, evolver="VV2", expansion=True, dt=0.005, seed="s", amp=1e-2, gU1=0.35, gSU2=0.6,
                  qG=50.0, qH=50.0, kcut=None, extra=None):
    """lphi4SU2U1 parameter set, run parameters, model and initial state (lphi4SU2U1.in values for
    the homogeneous doublet, qG and qH; the gauge couplings of the 384^3 case)."""
    from cosmolattice_b200 import MODELS, ParameterParser, RunParameters
    from cosmolattice_b200.initializers import su2u1_initial_state

    params = {
        "N": N, "kIR": 1.0, "dt": dt, "evolver": evolver, "expansion": "true" if expansion else "false",
        "lambda": 1.0, "qG": qG, "qH": qH, "initial_amplitudes": 0.0, "initial_momenta": 0.0,
        "cmplx_field_initial_norm": 0.0, "cmplx_momentum_initial_norm": 0.0,
        "SU2Doublet_initial_norm": "5.25151e18", "SU2Doublet_initial_momenta_norm": 0.0,
        "gU1s": gU1, "gSU2s": gSU2, "fluct_amplitude": amp,
        "kCutOff": kcut if kcut is not None else N / 4.0, "baseSeed": seed,
    }
    if extra:
        params.update(extra)
    par = ParameterParser(params=params)
    rp = RunParameters(par)
    m = MODELS["lphi4SU2U1"](par, rp)
    f, p, aI, aD = su2u1_initial_state(m, rp)
    sf = {"aI": aI, "aSI": aI, "aIM": aI, "aDotI": aD, "aDotSI": aD}
    return par, rp, m, f, p, sf


@pytest.fixture(scope="session")
def gpu_available():
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


# Per-site parity metrics.  The state is a homogeneous value plus small fluctuations (phi ~ 1 with
# fluctuations ~1e-3 in the scalar cases), so an error bar relative to an array's maximum checks
# the fluctuations only to that ratio.  Two bars see them:
#   fluct: max |a - b| over a component, relative to max |b - <b>| (the fluctuations' own scale);
#   site:  max |a - b| / |b| over the sites where |b| >= SITE_FLOOR * max |b| (a true per-site
#          relative error; below the floor a value's relative error measures only its smallness).
SITE_FLOOR = 1e-1


def site_metrics(a, b, nc, floor=SITE_FLOOR):
    """(site, fluct) errors of a against b, each the worst over the nc components."""
    import numpy as np

    a = np.asarray(a).reshape(nc, -1)
    b = np.asarray(b).reshape(nc, -1)
    site = fluct = 0.0
    for c in range(nc):
        sc = np.abs(b[c]).max()
        if sc == 0:
            continue
        d = np.abs(a[c] - b[c])
        m = np.abs(b[c]) >= floor * sc
        site = max(site, float((d[m] / np.abs(b[c][m])).max()))
        fs = np.abs(b[c] - b[c].mean()).max()
        if fs > 0:
            fluct = max(fluct, float(d.max() / fs))
    return site, fluct
