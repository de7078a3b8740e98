"""Tangent-linear form of lphi4SU2U1 (clb_tangent_*) on the B200.

The observable is the final gauge-energy fraction (E_el + E_mag of U(1) and SU(2)) / E_tot.  Its
derivative with respect to g_SU2 and g_U1 (start state, clb_initialize's aDot correction and the
evolution) is compared with central differences (relative step h = 1e-4) of (i) the plain GPU path
and (ii) the CPU oracle.  Agreement bar: 1e-5 relative, as for the lphi4U1 adjoint.  The state
part of the tangent run must equal the plain run bitwise.
"""
import numpy as np
import pytest

from conftest import make_su2_case

pytestmark = pytest.mark.gpu

REL = 1e-5
BASE = {"gSU2": 0.6, "gU1": 0.35}


def case(N, evolver, expansion, over=None, amp=3e-2):
    g = dict(BASE)
    g.update(over or {})
    return make_su2_case(N=N, evolver=evolver, expansion=expansion, amp=amp, gSU2=g["gSU2"], gU1=g["gU1"])


def plain_observable(N, evolver, expansion, n, over=None, oracle=False, precision="fp64"):
    from cosmolattice_b200 import Lattice
    from cosmolattice_b200.adjoint import su2_observable_from_measurement
    from oracle.oracle import OracleLattice

    par, rp, m, f, p, sf = case(N, evolver, expansion, over)
    lat = OracleLattice(m, rp) if oracle else Lattice(m, rp, precision=precision)
    lat.set_state(f, p, sf)
    lat.initialize()
    lat.evolve(n)
    lat.sync()
    o = su2_observable_from_measurement(lat.measure(1.0))
    lat.close()
    return o


def fd(param, N, evolver, expansion, n, oracle=False):
    h = 1e-4 * BASE[param]
    up = plain_observable(N, evolver, expansion, n, {param: BASE[param] + h}, oracle)
    dn = plain_observable(N, evolver, expansion, n, {param: BASE[param] - h}, oracle)
    return (up - dn) / (2 * h)


@pytest.mark.parametrize("evolver,expansion", [("VV2", True), ("VV4", True), ("VV2", False), ("LF", True)])
def test_gradients_match_gpu_finite_differences(evolver, expansion):
    from cosmolattice_b200.adjoint import su2_gradient

    N, n = 8, 30
    par, rp, m, f, p, sf = case(N, evolver, expansion)
    for prm in ("gSU2", "gU1"):
        O, dO = su2_gradient(m, rp, n, prm, state=(f, p, sf["aI"], sf["aDotI"]))
        assert abs(O - plain_observable(N, evolver, expansion, n)) <= 1e-12 * abs(O)
        ref = fd(prm, N, evolver, expansion, n)
        print(evolver, expansion, prm, dO, ref, abs(dO - ref) / abs(ref))
        assert abs(dO - ref) <= REL * abs(ref), (prm, dO, ref)


def test_gradients_match_oracle_finite_differences():
    from cosmolattice_b200.adjoint import su2_gradient

    N, n = 8, 20
    par, rp, m, f, p, sf = case(N, "VV2", True)
    for prm in ("gSU2", "gU1"):
        O, dO = su2_gradient(m, rp, n, prm, state=(f, p, sf["aI"], sf["aDotI"]))
        ref = fd(prm, N, "VV2", True, n, oracle=True)
        assert abs(dO - ref) <= REL * abs(ref), (prm, dO, ref)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_tangent_form_state_is_plain_state_bitwise(precision):
    from cosmolattice_b200 import Lattice
    from cosmolattice_b200.initializers import su2u1_initial_state_tangent

    par, rp, m, f, p, sf = case(8, "VV2", True)
    out = {}
    for tangent in (False, True):
        lat = Lattice(m, rp, precision=precision)
        lat.set_state(f, p, sf)
        if tangent:
            df, dp, cd = su2u1_initial_state_tangent(m, rp, "gSU2", (f, p))
            lat.tangent_begin(cd, df, dp)
        lat.initialize()
        lat.evolve(23)  # crosses two re-unitarisations of the FP32 form
        out[tangent] = lat.get_state()
        if tangent:
            fd_, pd_, sfd = lat.tangent_get_state()
            assert np.isfinite(fd_).all() and np.isfinite(pd_).all() and abs(pd_).max() > 0
            assert sfd["aI"] != 0 and sfd["aDotI"] != 0
        lat.close()
    (fa, pa, sa), (fb, pb, sb) = out[False], out[True]
    assert np.array_equal(fa, fb) and np.array_equal(pa, pb)
    assert sa == sb


def test_state_tangent_matches_directional_difference():
    # the tangent of the state itself after 20 steps against a central difference of the plain
    # path along the same direction (g_SU2 with its start-state tangent)
    from cosmolattice_b200 import Lattice
    from cosmolattice_b200.initializers import su2u1_initial_state_tangent

    N, n = 8, 20
    par, rp, m, f, p, sf = case(N, "VV2", True)
    lat = Lattice(m, rp)
    lat.set_state(f, p, sf)
    df, dp, cd = su2u1_initial_state_tangent(m, rp, "gSU2", (f, p))
    lat.tangent_begin(cd, df, dp)
    lat.initialize()
    lat.evolve(n)
    tf, tp, tsf = lat.tangent_get_state()
    lat.close()
    h = 1e-4 * BASE["gSU2"]
    res = []
    for g in (BASE["gSU2"] + h, BASE["gSU2"] - h):
        _, rp2, m2, f2, p2, sf2 = case(N, "VV2", True, {"gSU2": g})
        l2 = Lattice(m2, rp2)
        l2.set_state(f2, p2, sf2)
        l2.initialize()
        l2.evolve(n)
        res.append(l2.get_state())
        l2.close()
    dfd = (res[0][0] - res[1][0]) / (2 * h)
    dpd = (res[0][1] - res[1][1]) / (2 * h)
    dad = (res[0][2]["aI"] - res[1][2]["aI"]) / (2 * h)
    for t, r in ((tf, dfd), (tp, dpd)):
        t = t.reshape(-1, N ** 3)
        r = r.reshape(-1, N ** 3)
        for c in range(t.shape[0]):
            sc = np.abs(r[c]).max()
            if sc > 1e-9:
                assert np.abs(t[c] - r[c]).max() <= 1e-4 * sc, (c, np.abs(t[c] - r[c]).max(), sc)
    assert abs(tsf["aI"] - dad) <= 1e-5 * abs(dad)


def test_fp32_form_gradient_tracks_fp64():
    # The gauge-energy fraction starts at zero (unit links) and is 1.6e-5 of E_tot after 40 steps;
    # FP32 storage of the O(1) doublet leaves it an absolute error of ~1e-8 (measured 7e-9, i.e.
    # 4.4e-4 relative) and its derivative 7e-4 relative.  Bounds: 2e-3 and 5e-3.
    from cosmolattice_b200 import Lattice
    from cosmolattice_b200.adjoint import su2_gradient

    N, n = 10, 40
    par, rp, m, f, p, sf = case(N, "VV2", True)
    st = (f, p, sf["aI"], sf["aDotI"])
    O64, d64 = su2_gradient(m, rp, n, "gSU2", state=st)
    lat = Lattice(m, rp, precision="fp32")
    O32, d32 = su2_gradient(m, rp, n, "gSU2", lattice=lat, state=st)
    lat.close()
    print("fp32 tangent: O", abs(O32 - O64) / abs(O64), "dO", abs(d32 - d64) / abs(d64))
    assert abs(O32 - O64) <= 2e-3 * abs(O64)
    assert abs(d32 - d64) <= 5e-3 * abs(d64)


def test_tangent_api_errors():
    from cosmolattice_b200 import Lattice, _capi

    par, rp, m, f, p, sf = case(6, "VV2", True)
    lat = Lattice(m, rp)
    lat.set_state(f, p, sf)
    with pytest.raises(_capi.ClbError) as e:
        lat.tangent_observable([1.0])
    assert e.value.code == _capi.CLB_ESTATE
    with pytest.raises(_capi.ClbError) as e:
        lat.tangent_begin(np.zeros(7))
    assert e.value.code == _capi.CLB_EINVAL
    lat.tangent_begin(np.zeros(6))
    lat.initialize()
    with pytest.raises(_capi.ClbError) as e:
        lat.tangent_observable(np.ones(12))
    assert e.value.code == _capi.CLB_EINVAL
    O, dO = lat.tangent_observable(np.ones(11))
    assert O == pytest.approx(1.0) and dO == 0.0
    E, dE = lat.tangent_energies()
    e = lat.measure(1.0)["energies"]
    assert np.allclose(E, list(e[:10]) + [sum(e[10:13])], rtol=1e-12, atol=0) and not dE.any()
    lat.set_state(f, p, sf)  # ends the tangent form
    lat.initialize()
    with pytest.raises(_capi.ClbError) as e:
        lat.tangent_get_state()
    assert e.value.code == _capi.CLB_ESTATE
    lat.close()


@pytest.mark.parametrize("which,comp", [(0, 3), (0, 11), (1, 10), (1, 7)])
def test_spectrum_tangent_matches_gpu_finite_differences(which, comp):
    # d/dg_SU2 of the binned spectrum (doublet field, an SU(2) link component, SU(2) and U(1)
    # momenta with their a-factors) against central differences of clb_spectrum on the plain path
    from cosmolattice_b200 import Lattice
    from cosmolattice_b200.initializers import su2u1_initial_state_tangent

    N, n = 8, 20
    par, rp, m, f, p, sf = case(N, "VV2", True)
    lat = Lattice(m, rp)
    lat.set_state(f, p, sf)
    df, dp, cd = su2u1_initial_state_tangent(m, rp, "gSU2", (f, p))
    lat.tangent_begin(cd, df, dp)
    lat.initialize()
    lat.evolve(n)
    k, v, dv, c = lat.tangent_spectrum(which=which, comp=comp)
    k0, v0, c0 = lat.spectrum(which=which, comp=comp)
    lat.close()
    assert np.array_equal(c, c0) and np.allclose(v, v0, rtol=1e-12, atol=0)  # bins summed by shared atomics
    h = 1e-4 * BASE["gSU2"]
    res = []
    for g in (BASE["gSU2"] + h, BASE["gSU2"] - h):
        _, rp2, m2, f2, p2, sf2 = case(N, "VV2", True, {"gSU2": g})
        l2 = Lattice(m2, rp2)
        l2.set_state(f2, p2, sf2)
        l2.initialize()
        l2.evolve(n)
        res.append(l2.spectrum(which=which, comp=comp)[1])
        l2.close()
    ref = (res[0] - res[1]) / (2 * h)
    sc = np.abs(ref).max()
    print("spectrum tangent", which, comp, np.abs(dv - ref).max() / sc)
    assert sc > 0 and np.abs(dv - ref).max() <= 1e-5 * sc


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_plain_evolution_after_tangent_end_is_bitwise(precision):
    # the tangent form's kicks form the U(1) link phases themselves; after clb_tangent_end the plain
    # kicks read the phase arrays again, which must hold the phases of the current A
    from cosmolattice_b200 import Lattice

    par, rp, m, f, p, sf = case(8, "VV2", True)
    out = []
    for tangent in (False, True):
        lat = Lattice(m, rp, precision=precision)
        lat.set_state(f, p, sf)
        if tangent:
            lat.tangent_begin([0, 0, 0, 0, 1, 0])
        lat.initialize()
        lat.evolve(7)
        if tangent:
            lat.tangent_end()
        lat.evolve(6)
        out.append(lat.get_state())
        lat.close()
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][1], out[1][1])


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_tangent_kick_split_is_bitwise_the_whole_sweep(monkeypatch, precision):
    # The tangent sweep runs whole, in halves, three or four parts (CLB_SU2_SPLIT 0, 1, 2, 3) with the
    # same per-component arithmetic, so state and tangent agree to the last bit.
    from cosmolattice_b200 import Lattice
    from cosmolattice_b200.initializers import su2u1_initial_state_tangent

    par, rp, m, f, p, sf = case(8, "VV2", True)
    df, dp, cd = su2u1_initial_state_tangent(m, rp, "gSU2", (f, p))
    out = {}
    for split in ("0", "1", "2", "3"):
        monkeypatch.setenv("CLB_SU2_SPLIT", split)
        lat = Lattice(m, rp, precision=precision)
        lat.set_state(f, p, sf)
        lat.tangent_begin(cd, df, dp)
        lat.initialize()
        lat.evolve(12)
        out[split] = (lat.get_state(), lat.tangent_get_state())
        lat.close()
    for split in ("1", "2", "3"):
        for (a, b) in zip(out[split], out["0"]):
            assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]) and a[2] == b[2], split
