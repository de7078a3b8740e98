"""Parity of the CUDA lphi4SU2U1 path with the FP64 CPU oracle (B200).

Same bars as lphi4U1: per-site fields and momenta after 100 steps within 1e-12 of each
component's max |value|, within 2e-12 of its fluctuations max |x - <x>|, and within 1e-11 of each
site's own value where it exceeds 1e-1 of that max (conftest.site_metrics; measured 9e-13); the
same with the 384^3 workload's couplings and time step at 64^3; a(t), aDot, energies, means and the Gauss averages
within 1e-10 relative, the Gauss ratios within 1e-8 relative (difference of nearly equal
terms).  Both Gauss laws are preserved per site on the GPU too.
"""
import math

import numpy as np
import pytest

from conftest import make_su2_case, site_metrics

pytestmark = pytest.mark.gpu

SITE_TOL = 1e-12
FLUCT_TOL = 2e-12
SITE_REL_TOL = 1e-11
AVG_TOL = 1e-10
RATIO_TOL = 1e-8


def rel_comp(a, b, nc):
    a = np.asarray(a).reshape(nc, -1)
    b = np.asarray(b).reshape(nc, -1)
    out = []
    for c in range(nc):
        sc = np.abs(b[c]).max()
        out.append(np.abs(a[c] - b[c]).max() / sc if sc > 0 else np.abs(a[c]).max())
    return max(out)


def random_links(f, rng, s=0.1):
    f = f.copy()
    N = f.shape[1]
    for i in range(3):
        q = rng.normal(0, s, (4, N, N, N))
        q[0] += 1
        f[10 + 4 * i:14 + 4 * i] = q / np.sqrt((q * q).sum(axis=0))
    f[7:10] = rng.normal(0, 0.2, (3, N, N, N))
    return f


def run_pair(N, evolver, expansion, nsteps, measure_every=None, links=False, extra=None, amp=3e-2):
    from cosmolattice_b200 import Lattice
    from oracle.oracle import OracleLattice

    par, rp, m, f, p, sf = make_su2_case(N=N, evolver=evolver, expansion=expansion, amp=amp, extra=extra)
    if links:
        f = random_links(f, np.random.default_rng(4))
    gpu = Lattice(m, rp)
    cpu = OracleLattice(m, rp)
    meas = {"gpu": [], "cpu": []}
    for key, lat in (("gpu", gpu), ("cpu", cpu)):
        lat.set_state(f, p, sf)
        lat.initialize()
        lat.sync()
        m0 = lat.measure(1.0)
        e0 = m0["energies"][-1]
        meas[key].append(m0)
        done = 0
        while done < nsteps:
            k = nsteps - done if measure_every is None else min(measure_every, nsteps - done)
            lat.evolve(k)
            done += k
            if measure_every is not None:
                lat.sync()
                meas[key].append(lat.measure(e0))
        lat.sync()
        meas[key].append(lat.measure(e0))
    out = (gpu.get_state(), cpu.get_state(), meas)
    gpu.close()
    cpu.close()
    return out


def check(g, c, meas):
    (fg, pg, sg), (fc, pc, sc) = g, c
    assert rel_comp(fg, fc, 22) < SITE_TOL, rel_comp(fg, fc, 22)
    assert rel_comp(pg, pc, 19) < SITE_TOL, rel_comp(pg, pc, 19)
    for what, a, b, nc in (("fields", fg, fc, 22), ("momenta", pg, pc, 19)):
        site, fluct = site_metrics(a, b, nc)
        assert site < SITE_REL_TOL, (what, "per-site", site)
        assert fluct < FLUCT_TOL, (what, "fluctuations", fluct)
    for k in ("aI", "aDotI"):
        assert abs(sg[k] - sc[k]) <= AVG_TOL * max(abs(sc[k]), 1e-300), (k, sg[k], sc[k])
    for a, b in zip(meas["gpu"], meas["cpu"]):
        assert len(a["energies"]) == len(b["energies"]) == 14
        for ea, eb in zip(a["energies"], b["energies"]):
            assert abs(ea - eb) <= AVG_TOL * abs(eb) + 1e-30, (a["energies"], b["energies"])
        for k in (1, 2):
            assert abs(a["friedmann"][k] - b["friedmann"][k]) <= AVG_TOL * abs(b["friedmann"][k]) + 1e-300
        assert len(a["means"]) == len(b["means"]) == 7
        for ra, rb in zip(a["means"], b["means"]):
            # the mean of |B| of SU(2) takes sqrt(B^2) per site as the reference does
            # (su2measurer.h:62); near unit links B^2 can round below zero, and both sides then
            # report NaN in the same place
            assert [math.isnan(x) for x in ra] == [math.isnan(y) for y in rb], (ra, rb)
            scales = [max(abs(rb[0]), rb[4]), max(abs(rb[1]), rb[5]), abs(rb[2]), abs(rb[3])]
            for x, y, s in zip(ra[:4], rb[:4], scales):
                if math.isnan(y):
                    continue
                assert abs(x - y) <= AVG_TOL * max(s, 1e-300) + 1e-30, (ra, rb)
        for key in ("gauss_u1", "gauss_su2"):
            ga, gb = a[key], b[key]
            for k in (1, 2):
                assert abs(ga[k] - gb[k]) <= AVG_TOL * abs(gb[k]) + 1e-300, (key, ga, gb)
            assert abs(ga[0] - gb[0]) <= RATIO_TOL * abs(gb[0]) + 1e-300, (key, ga, gb)


@pytest.mark.parametrize("evolver,expansion", [("VV2", True), ("VV2", False), ("VV4", True), ("LF", True)])
def test_lphi4su2u1_100_steps(evolver, expansion):
    g, c, meas = run_pair(8, evolver, expansion, 100)
    check(g, c, meas)


def test_lphi4su2u1_workload_couplings_64_vv2_100_steps():
    # the 384^3 workload's couplings (gSU2 = 0.6, gU1 = 0.35, qG = qH = 50, lambda = 1), time step
    # (0.005), evolver (VV2), expansion and amplitude (1e-3) on a 64^3 lattice, 100 steps
    g, c, meas = run_pair(64, "VV2", True, 100, amp=1e-3)
    check(g, c, meas)


@pytest.mark.parametrize("evolver", ["VV2", "LF"])
def test_lphi4su2u1_links_and_measure_cadence(evolver):
    g, c, meas = run_pair(7, evolver, True, 40, measure_every=9, links=True)
    check(g, c, meas)


def test_gauss_laws_preserved_on_gpu():
    from cosmolattice_b200 import Lattice

    from test_oracle_su2 import gauss_fields

    par, rp, m, f, p, sf = make_su2_case(N=12, evolver="VV2", expansion=True, amp=5e-2)
    f = random_links(f, np.random.default_rng(9), 0.05)
    g1a, g2a, rho = gauss_fields(rp, m, f.ravel(), p.ravel())
    lat = Lattice(m, rp)
    lat.set_state(f, p, sf)
    lat.initialize()
    lat.evolve(100)
    f1, p1, _ = lat.get_state()
    lat.close()
    g1b, g2b, _ = gauss_fields(rp, m, f1, p1)
    assert np.abs(g1b - g1a).max() < 1e-12 * np.abs(rho).max() * rp.dx
    assert np.abs(g2b - g2a).max() < 1e-11 * np.abs(g2a).max() + 1e-14
    U = f1.reshape(22, -1)[10:].reshape(3, 4, -1)
    assert np.abs((U * U).sum(axis=1) - 1).max() < 1e-13


def test_fp32_form_tracks_fp64():
    # FP32 storage and stencils, FP64 increments, sums and a(t), links re-unitarised every 10 steps.
    # The homogeneous doublet (|Phi| ~ 1) is stored in FP32 (unit roundoff 6e-8), so a(t), which
    # here grows 4.7-fold in 100 steps, follows FP64 to 1e-7 (measured 1.6e-8); energies to 1e-5
    # relative (2.2e-7), links unit to 1e-6, Gauss averages and the doublet spectrum to 1e-5.
    from cosmolattice_b200 import Lattice

    par, rp, m, f, p, sf = make_su2_case(N=12, evolver="VV2", expansion=True, amp=3e-2)
    f = random_links(f, np.random.default_rng(6), 0.05)
    res = {}
    for prec in ("fp64", "fp32"):
        lat = Lattice(m, rp, precision=prec)
        lat.set_state(f, p, sf)
        lat.initialize()
        m0 = lat.measure(1.0)
        lat.evolve(100)
        res[prec] = (lat.get_state(), lat.measure(m0["energies"][-1]))
        k, v, c = lat.spectrum(which=0, comp=3)
        res[prec] += (v,)
        lat.close()
    (fa, pa, sa), ma, va = res["fp32"]
    (fb, pb, sb), mb, vb = res["fp64"]
    ediff = max(abs(x - y) / abs(y) for x, y in zip(ma["energies"], mb["energies"]) if y != 0)
    print("fp32-vs-fp64: a", abs(sa["aI"] - sb["aI"]) / sb["aI"], "energies", ediff,
          "gauss", [abs(ma[k][1] - mb[k][1]) / mb[k][1] for k in ("gauss_u1", "gauss_su2")],
          "spectrum", np.abs(va - vb).max() / np.abs(vb).max())
    assert abs(sa["aI"] - sb["aI"]) <= 1e-7 * sb["aI"]
    for x, y in zip(ma["energies"], mb["energies"]):
        assert abs(x - y) <= 1e-5 * abs(y) + 1e-10 * abs(mb["energies"][-1]), (ma["energies"], mb["energies"])
    U = fa.reshape(22, -1)[10:].reshape(3, 4, -1)
    assert np.abs((U * U).sum(axis=1) - 1).max() < 1e-6
    for key in ("gauss_u1", "gauss_su2"):
        assert abs(ma[key][1] - mb[key][1]) <= 1e-5 * mb[key][1]
    assert np.abs(va - vb).max() <= 1e-5 * np.abs(vb).max()


def test_su2_rejects_unsupported():
    from cosmolattice_b200 import Lattice, _capi

    par, rp, m, f, p, sf = make_su2_case(N=6)
    lat = Lattice(m, rp)
    assert (lat.n_field_components, lat.n_momentum_components) == (22, 19)
    lat.set_state(f, p, sf)
    lat.initialize()
    with pytest.raises(_capi.ClbError):
        lat.spectrum(which=1, comp=19)
    from oracle.spectrum import spectrum

    fg, _, _ = lat.get_state()
    k, v, c = lat.spectrum(which=0, comp=3)
    ko, vo, co = spectrum(fg.reshape(22, 6, 6, 6)[3], rp.dx)
    assert c.tolist() == co.tolist() and np.abs(v - vo).max() <= 1e-10 * np.abs(vo).max()
    lat.close()


# ---- position Verlet for lphi4SU2U1 (PositionVerlet::evolve, positionverlet.h:45-99) ----------

@pytest.mark.parametrize("evolver,expansion", [("PV2", True), ("PV2", False), ("PV4", True)])
def test_lphi4su2u1_position_verlet(evolver, expansion):
    g, c, meas = run_pair(8, evolver, expansion, 20, measure_every=7, links=True)
    check(g, c, meas)


def test_lphi4su2u1_position_verlet_fp32_and_tangent_guard():
    from cosmolattice_b200 import Lattice, _capi

    par, rp, m, f, p, sf = make_su2_case(N=8, evolver="PV4", amp=3e-2)
    out = {}
    for prec in ("fp64", "fp32"):
        lat = Lattice(m, rp, precision=prec)
        lat.set_state(f, p, sf)
        if prec == "fp64":
            with pytest.raises(_capi.ClbError):
                lat.tangent_begin([0, 0, 0, 0, 1, 0])  # the tangent-linear form covers LF and VV
        lat.initialize()
        lat.evolve(20)
        lat.sync()
        out[prec] = lat.measure(1.0)
        lat.close()
    assert abs(out["fp32"]["aI"] - out["fp64"]["aI"]) <= 1e-7 * out["fp64"]["aI"]
    for x, y in zip(out["fp32"]["energies"], out["fp64"]["energies"]):
        assert abs(x - y) <= 1e-4 * abs(out["fp64"]["energies"][-1])


# ---- fixed background for lphi4SU2U1 (fixedbackgroundexpansion.h:21-45) ------------------------

@pytest.mark.parametrize("evolver", ["VV2", "LF", "PV2"])
def test_lphi4su2u1_fixed_background(evolver):
    fb = {"fixedBackground": "true", "H0": 2.0e18, "omegaEoS": 0.0}
    g, c, meas = run_pair(8, evolver, True, 20, measure_every=7, links=True, extra=fb)
    check(g, c, meas)


def test_lphi4su2u1_fixed_background_rejects_the_tangent_form():
    from cosmolattice_b200 import Lattice, _capi

    par, rp, m, f, p, sf = make_su2_case(N=6, extra={"fixedBackground": "true", "H0": 2.0e18})
    lat = Lattice(m, rp)
    lat.set_state(f, p, sf)
    with pytest.raises(_capi.ClbError):
        lat.tangent_begin([0, 0, 0, 0, 1, 0])
    lat.close()


@pytest.mark.parametrize("evolver", ["VV2", "LF"])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_kick_split_is_bitwise_the_whole_sweep(monkeypatch, evolver, precision):
    # CLB_SU2_SPLIT: 0 one kick sweep, 1 two halves (S, phi, Phi, A; SU(2)), 2 three parts (S, phi,
    # Phi; A; SU(2)), 3 four parts (S, phi; Phi; A; SU(2)).  Each component's kernel and each partial
    # slot's sum run the same arithmetic over the same sites in every form, so states, a(t) and
    # energies agree to the last bit.
    from cosmolattice_b200 import Lattice

    par, rp, m, f, p, sf = make_su2_case(N=12, evolver=evolver, expansion=True, amp=3e-2)
    f = random_links(f, np.random.default_rng(8), 0.05)
    res = {}
    for split in ("0", "1", "2", "3"):
        monkeypatch.setenv("CLB_SU2_SPLIT", split)
        lat = Lattice(m, rp, precision=precision)
        lat.set_state(f, p, sf)
        lat.initialize()
        lat.evolve(7)
        lat.evolve(5)
        lat.sync()
        res[split] = (lat.get_state(), lat.measure(1.0))
        lat.close()
    (f0, p0, s0), m0 = res["0"]
    for split in ("1", "2", "3"):
        (fs, ps, ss), ms = res[split]
        assert np.array_equal(fs, f0) and np.array_equal(ps, p0), split
        assert ss == s0, split
        assert ms["energies"] == m0["energies"], split
