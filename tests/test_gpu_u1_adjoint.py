"""Adjoint pair (clb_forward / clb_backward) of lphi4U1 against central finite differences (B200).

Observable: the final gauge-energy fraction (E_el + E_mag) / E_tot.  Gradients with respect to the
fluctuation amplitude, the quartic coupling and the gauge coupling are compared with central
differences (relative step h = 1e-4) of (i) the plain GPU path (initial state, clb_initialize,
clb_evolve, clb_measure) and (ii) the CPU oracle.  Agreement bar: 1e-5 relative (the difference
quotient itself carries O(h^2) ~ 1e-8 truncation and ~1e-10 rounding error).
"""
import numpy as np
import pytest

from conftest import make_u1_case

pytestmark = pytest.mark.gpu

KEYS = {"amp": "fluct_amplitude", "c4": "lambda_prog", "gQ": "gU1s"}
BASE = {"amp": 3e-2, "c4": 1.0, "gQ": 0.5}
REL = 1e-5


def case(N, evolver, expansion, dt, over=None):
    v = dict(BASE)
    if over:
        v.update(over)
    return make_u1_case(N=N, evolver=evolver, expansion=expansion, dt=dt, amp=v["amp"], gU1=v["gQ"],
                        extra={"lambda_prog": v["c4"]})


def plain_observable(N, evolver, expansion, dt, n, over=None, oracle=False):
    from cosmolattice_b200 import Lattice
    from cosmolattice_b200.adjoint import observable_from_measurement
    from oracle.oracle import OracleLattice

    par, rp, m, f, p, sf = case(N, evolver, expansion, dt, over)
    lat = OracleLattice(m, rp) if oracle else Lattice(m, rp)
    lat.set_state(f, p, sf)
    lat.initialize()
    lat.evolve(n)
    lat.sync()
    o = observable_from_measurement(lat.measure(1.0))
    lat.close()
    return o


def fd(param, N, evolver, expansion, dt, n, oracle=False):
    h = 1e-4 * BASE[param]
    up = plain_observable(N, evolver, expansion, dt, n, {param: BASE[param] + h}, oracle)
    dn = plain_observable(N, evolver, expansion, dt, n, {param: BASE[param] - h}, oracle)
    return (up - dn) / (2 * h)


@pytest.mark.parametrize("evolver,expansion,K", [("VV2", True, 7), ("VV4", True, 5), ("VV2", False, 40),
                                                 ("LF", True, 7), ("LF", True, 30), ("LF", False, 40)])
def test_gradients_match_gpu_finite_differences(evolver, expansion, K):
    from cosmolattice_b200.adjoint import u1_gradients

    N, dt, n = 12, 0.01, 30
    par, rp, m, f, p, sf = case(N, evolver, expansion, dt)
    O, grads, _ = u1_gradients(m, rp, n, K)
    assert abs(O - plain_observable(N, evolver, expansion, dt, n)) <= 1e-12 * abs(O)
    for prm in ("amp", "c4", "gQ"):
        ref = fd(prm, N, evolver, expansion, dt, n)
        assert abs(grads[prm] - ref) <= REL * abs(ref), (prm, grads[prm], ref)


def test_gradients_match_oracle_finite_differences():
    from cosmolattice_b200.adjoint import u1_gradients

    N, dt, n = 10, 0.01, 20
    par, rp, m, f, p, sf = case(N, "VV4", True, dt)
    O, grads, _ = u1_gradients(m, rp, n, 6)
    for prm in ("amp", "c4", "gQ"):
        ref = fd(prm, N, "VV4", True, dt, n, oracle=True)
        assert abs(grads[prm] - ref) <= REL * abs(ref), (prm, grads[prm], ref)


@pytest.mark.parametrize("evolver,expansion", [("VV2", True), ("VV2", False), ("LF", True), ("LF", False)])
def test_state_cotangent_directional_derivative(evolver, expansion):
    # <fields_bar, v_f> + <momenta_bar, v_p> + aI_bar da + aDot_bar dadot equals the derivative of
    # O along a random start-state direction (no initial aDot correction: through_init = 0)
    from cosmolattice_b200 import Lattice
    from cosmolattice_b200.adjoint import GAUGE_FRACTION, observable_from_measurement

    N, dt, n = 10, 0.01, 25
    par, rp, m, f, p, sf = case(N, evolver, expansion, dt)
    rng = np.random.default_rng(5)
    f = f.copy()
    f[2:] = rng.normal(0, 0.05, f[2:].shape)
    vf = rng.normal(0, 1e-3, f.shape)
    vp = rng.normal(0, 1e-3, p.shape)
    da, dad = (1e-3, 2e-3) if expansion else (0.0, 0.0)  # without expansion a is a constant

    def run(eps, adjoint=False):
        s = dict(sf)
        s["aI"] = s["aSI"] = s["aIM"] = 1.0 + eps * da
        s["aDotI"] = s["aDotSI"] = sf["aDotI"] + eps * dad
        lat = Lattice(m, rp)
        lat.set_state(f + eps * vf, p + eps * vp, s)
        lat.initialize(correct_adot=False)
        if adjoint:
            O = lat.forward(n, 4, GAUGE_FRACTION)
            out = (O,) + lat.backward(through_init=False)
        else:
            lat.evolve(n)
            lat.sync()  # the leapfrog's momenta to integer time, as clb_forward ends
            out = observable_from_measurement(lat.measure(1.0))
        lat.close()
        return out

    O, fb, pb, g = run(0.0, adjoint=True)
    dirder = fb @ vf.ravel() + pb @ vp.ravel() + (g["dO_daI"] * da + g["dO_daDotI"] * dad if expansion else 0.0)
    h = 1e-3
    ref = (run(h) - run(-h)) / (2 * h)
    assert abs(dirder - ref) <= 1e-5 * abs(ref), (dirder, ref)


def test_forward_matches_evolve_bitwise_and_restores_state():
    from cosmolattice_b200 import Lattice

    par, rp, m, f, p, sf = case(13, "VV4", True, 0.01)
    a, b = Lattice(m, rp), Lattice(m, rp)
    for lat in (a, b):
        lat.set_state(f, p, sf)
        lat.initialize()
    a.evolve(9)
    b.forward(9, 4, (0, 0, 1, 1, 0))
    fa, pa, sa = a.get_state()
    fb, pb, sb = b.get_state()
    assert np.array_equal(fa, fb) and np.array_equal(pa, pb) and sa == sb
    b.backward()
    fc, pc, sc = b.get_state()
    assert np.array_equal(fa, fc) and np.array_equal(pa, pc) and sa == sc
    a.close()
    b.close()


def test_adjoint_rejects_unsupported():
    from cosmolattice_b200 import Lattice, _capi

    par, rp, m, f, p, sf = case(8, "PV2", True, 0.01)
    lat = Lattice(m, rp)
    lat.set_state(f, p, sf)
    lat.initialize()
    with pytest.raises(_capi.ClbError) as e:
        lat.forward(3, 2, (0, 0, 1, 1, 0))
    assert e.value.code == _capi.CLB_EUNSUPPORTED
    lat.close()
    par, rp, m, f, p, sf = case(8, "VV2", True, 0.01)
    lat = Lattice(m, rp)
    lat.set_state(f, p, sf)
    lat.initialize()
    with pytest.raises(_capi.ClbError) as e:
        lat.backward()
    assert e.value.code == _capi.CLB_ESTATE
    lat.close()


@pytest.mark.parametrize("evolver", ["VV4", "LF"])
def test_fp32_form_gradients_track_fp64(evolver):
    # FP32 storage forward (FP64 increments and sums), FP64 cotangents: the observable and its
    # gradients follow the FP64 pair to the FP32 trajectory error (bounds: 1e-5 on O, 1e-3 on
    # each gradient relative to the largest one).
    from cosmolattice_b200 import Lattice
    from cosmolattice_b200.adjoint import u1_gradients

    N, dt, n, K = 12, 0.01, 30, 5
    par, rp, m, f, p, sf = case(N, evolver, True, dt)
    O64, g64, _ = u1_gradients(m, rp, n, K)
    lat = Lattice(m, rp, precision="fp32")
    O32, g32, _ = u1_gradients(m, rp, n, K, lattice=lat)
    lat.close()
    scale = max(abs(v) for v in g64.values())
    print("fp32 adjoint: O", abs(O32 - O64) / abs(O64),
          {k: abs(g32[k] - g64[k]) / scale for k in g64})
    assert abs(O32 - O64) <= 1e-5 * abs(O64)
    for k in g64:
        assert abs(g32[k] - g64[k]) <= 1e-3 * scale, (k, g32[k], g64[k])


SPEC_CASES = [
    # (evolver, which, comp, spectrum options): a scalar field, a gauge momentum (a^(2 alpha - 2)
    # factor), a scalar momentum over fewer bins than modes without folding
    ("VV2", 0, 0, {"ps_type": 1, "ps_version": 1, "dk": 1.0, "fold": True, "nbins": 10}),
    ("VV4", 1, 3, {"ps_type": 2, "ps_version": 2, "dk": 1.0, "fold": True, "nbins": 10}),
    ("VV2", 1, 1, {"ps_type": 1, "ps_version": 2, "dk": 1.5, "fold": False, "nbins": 4}),
    ("LF", 1, 0, {"ps_type": 1, "ps_version": 1, "dk": 1.0, "fold": True, "nbins": 10}),
    ("LF", 0, 2, {"ps_type": 2, "ps_version": 2, "dk": 1.0, "fold": True, "nbins": 10}),
]


def spectrum_weights(nbins):
    return np.linspace(0.5, 1.5, nbins) * np.where(np.arange(nbins) % 2 == 0, 1.0, -0.5)


def plain_spectrum_observable(N, evolver, dt, n, which, comp, opts, over=None):
    from cosmolattice_b200 import Lattice

    par, rp, m, f, p, sf = case(N, evolver, True, dt, over)
    lat = Lattice(m, rp)
    lat.set_state(f, p, sf)
    lat.initialize()
    lat.evolve(n)
    lat.sync()
    o = dict(opts)
    _, v, _ = lat.spectrum(which, comp, **o)
    lat.close()
    return float(spectrum_weights(opts["nbins"]) @ v)


@pytest.mark.parametrize("evolver,which,comp,opts", SPEC_CASES)
def test_spectrum_observable_gradients_match_finite_differences(evolver, which, comp, opts):
    # O = sum_b w_b P_b of one component at the end state (clb_forward_spectrum)
    from cosmolattice_b200.adjoint import u1_gradients

    N, dt, n = 12, 0.01, 30
    par, rp, m, f, p, sf = case(N, evolver, True, dt)
    spec = {k: v for k, v in opts.items() if k != "nbins"}
    spec.update(which=which, comp=comp, bin_weights=spectrum_weights(opts["nbins"]))
    O, grads, _ = u1_gradients(m, rp, n, 7, spectrum=spec)
    assert abs(O - plain_spectrum_observable(N, evolver, dt, n, which, comp, opts)) <= 1e-12 * abs(O)
    for prm in ("amp", "c4", "gQ"):
        h = 1e-4 * BASE[prm]
        up = plain_spectrum_observable(N, evolver, dt, n, which, comp, opts, {prm: BASE[prm] + h})
        dn = plain_spectrum_observable(N, evolver, dt, n, which, comp, opts, {prm: BASE[prm] - h})
        ref = (up - dn) / (2 * h)
        assert abs(grads[prm] - ref) <= REL * abs(ref), (prm, grads[prm], ref)


def test_energy_observable_after_spectrum_observable():
    # a plain clb_forward after clb_forward_spectrum is the energy observable again
    from cosmolattice_b200.adjoint import u1_gradients

    from cosmolattice_b200 import Lattice

    N, dt, n = 10, 0.01, 12
    par, rp, m, f, p, sf = case(N, "VV2", True, dt)
    lat = Lattice(m, rp)
    O0, g0, _ = u1_gradients(m, rp, n, 5, lattice=lat)
    u1_gradients(m, rp, n, 5, lattice=lat, spectrum={"which": 0, "comp": 2, "bin_weights": np.ones(6)})
    O1, g1, _ = u1_gradients(m, rp, n, 5, lattice=lat)
    lat.close()
    assert O1 == O0
    for prm in g0:
        assert g1[prm] == g0[prm]


@pytest.mark.parametrize("N,evolver,expansion", [(20, "VV2", True), (36, "VV4", True), (20, "VV2", False)])
def test_staged_sweeps_give_the_site_by_site_gradient(monkeypatch, N, evolver, expansion):
    # the kicks and the adjoint sweep on staged planes (the default) and site by site
    # (CLB_U1_TILE=0) evaluate every site alike; the volume sums and the dot products are added in
    # another order, so the observable and the gradients agree to 1e-12.  N = 20 and 36 leave
    # partial tiles in z and y; x-runs of 16 and 5 planes for the adjoint sweep.
    from cosmolattice_b200.adjoint import u1_gradients

    par, rp, m, f, p, sf = case(N, evolver, expansion, 0.01)
    out = []
    for env in ({"CLB_U1_TILE": "0"}, {}, {"CLB_U1_ADJ_LX": "5"}):
        for k in ("CLB_U1_TILE", "CLB_U1_ADJ_LX"):
            monkeypatch.delenv(k, raising=False)
        for k, v in env.items():
            monkeypatch.setenv(k, v)
        out.append(u1_gradients(m, rp, 12, 5))
    O0, g0, _ = out[0]
    for O, g, _ in out[1:]:
        assert abs(O - O0) <= 1e-12 * abs(O0)
        for prm in ("amp", "c4", "gQ"):
            assert abs(g[prm] - g0[prm]) <= 1e-12 * abs(g0[prm]), (prm, g[prm], g0[prm])
