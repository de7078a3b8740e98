"""Parity of the CUDA complex scalar + U(1) path (lphi4U1) with the FP64 CPU oracle (B200).

Tolerances: started from identical arrays, per-site fields and momenta after 100 steps within
1e-12 of each component's max |value|, within 2e-12 of the component's fluctuations max |x - <x>|,
and within 1e-11 of each site's own value where it exceeds 1e-1 of that max (conftest.site_metrics;
the gauge fields start at zero and stay small, and the device's sin/cos of the link phases differ
from the host's by an ulp: measured 3.8e-12 at 128^3 VV4); the same at the 128^3 VV4 geometry of
the gradient workload; a(t), aDot, energies,
means and the Gauss-law averages av|LHS|, av|RHS| within 1e-10 relative.  The Gauss ratio
av|LHS-RHS|/av|sum of squares| is formed from the difference of two nearly equal per-site terms
(cancellation of about 1e3 here), so it is compared within 1e-8 relative.
"""
import numpy as np
import pytest

from conftest import make_u1_case, site_metrics

pytestmark = pytest.mark.gpu

SITE_TOL = 1e-12
FLUCT_TOL = 2e-12
SITE_REL_TOL = 1e-11
AVG_TOL = 1e-10
GAUSS_RATIO_TOL = 1e-8


def rel_comp(a, b, N):
    a = np.asarray(a).reshape(5, -1)
    b = np.asarray(b).reshape(5, -1)
    out = []
    for c in range(5):
        sc = np.abs(b[c]).max()
        out.append(np.abs(a[c] - b[c]).max() / sc if sc > 0 else np.abs(a[c]).max())
    return max(out)


def run_pair(N, evolver, expansion, nsteps, measure_every=None, dt=0.01, amp=2e-2, links=0.0, extra=None):
    from cosmolattice_b200 import Lattice
    from oracle.oracle import OracleLattice

    par, rp, m, f, p, sf = make_u1_case(N=N, evolver=evolver, expansion=expansion, dt=dt, amp=amp, extra=extra)
    if links:
        rng = np.random.default_rng(11)
        f = f.copy()
        f[2:] = rng.normal(0.0, links, f[2:].shape)
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


def check_state(g, c, N):
    (fg, pg, sg), (fc, pc, sc) = g, c
    assert rel_comp(fg, fc, N) < SITE_TOL, rel_comp(fg, fc, N)
    assert rel_comp(pg, pc, N) < SITE_TOL, rel_comp(pg, pc, N)
    for what, a, b in (("fields", fg, fc), ("momenta", pg, pc)):
        site, fluct = site_metrics(a, b, 5)
        assert site < SITE_REL_TOL, (what, "per-site", site)
        assert fluct < FLUCT_TOL, (what, "fluctuations", fluct)
    for k in ("aI", "aDotI"):
        assert abs(sg[k] - sc[k]) <= AVG_TOL * max(abs(sc[k]), 1e-300), (k, sg[k], sc[k])


def check_meas(mg, mc):
    for a, b in zip(mg, mc):
        for ea, eb in zip(a["energies"], b["energies"]):
            assert abs(ea - eb) <= AVG_TOL * abs(eb) + 1e-300, (a["energies"], b["energies"])
        for k in (1, 2):
            assert abs(a["friedmann"][k] - b["friedmann"][k]) <= AVG_TOL * abs(b["friedmann"][k]) + 1e-300
        assert len(a["means"]) == len(b["means"]) == 4
        for ra, rb in zip(a["means"], b["means"]):
            scales = [max(abs(rb[0]), rb[4]), max(abs(rb[1]), rb[5]), abs(rb[2]), abs(rb[3])]
            for x, y, sc in zip(ra[:4], rb[:4], scales):
                assert abs(x - y) <= AVG_TOL * max(sc, 1e-300), (ra, rb)
        ga, gb = a["gauss_u1"], b["gauss_u1"]
        for k in (1, 2):
            assert abs(ga[k] - gb[k]) <= AVG_TOL * abs(gb[k]) + 1e-300, (ga, gb)
        assert abs(ga[0] - gb[0]) <= GAUSS_RATIO_TOL * abs(gb[0]) + 1e-300, (ga, gb)


@pytest.mark.parametrize("evolver,expansion", [("VV2", True), ("VV2", False), ("VV4", True), ("LF", True),
                                               ("LF", False), ("VV6", True)])
def test_lphi4u1_100_steps(evolver, expansion):
    N = 16
    g, c, meas = run_pair(N, evolver, expansion, 100)
    check_state(g, c, N)
    check_meas(meas["gpu"], meas["cpu"])


@pytest.mark.parametrize("evolver", ["VV2", "LF"])
def test_lphi4u1_measure_cadence_and_links(evolver):
    # measurements between evolve calls (the LF sync/measure side effects), random initial links
    N = 12
    g, c, meas = run_pair(N, evolver, True, 60, measure_every=7, links=0.05)
    check_state(g, c, N)
    check_meas(meas["gpu"], meas["cpu"])


def test_lphi4u1_ragged_size_and_history():
    # N not a multiple of any tile; per-step history rows of a(t)
    from cosmolattice_b200 import Lattice

    N = 13
    par, rp, m, f, p, sf = make_u1_case(N=N, evolver="VV2", expansion=True)
    g, c, meas = run_pair(N, "VV2", True, 30)
    check_state(g, c, N)
    lat = Lattice(m, rp)
    lat.set_state(f, p, sf)
    lat.initialize()
    lat.evolve(10)
    h = lat.history()
    _, _, s = lat.get_state()
    assert h.shape == (10, 5)
    assert h[-1, 0] == s["aI"] and h[-1, 1] == s["aDotI"]
    assert np.all(np.diff(h[:, 0]) > 0)
    lat.close()


def test_gauss_law_preserved_on_gpu():
    from cosmolattice_b200 import Lattice

    from test_oracle_u1 import gauss_field

    N = 24
    par, rp, m, f, p, sf = make_u1_case(N=N, evolver="VV4", expansion=True, amp=5e-2, dt=0.005)
    G0, r0 = gauss_field(rp, m, f.ravel(), p.ravel())
    lat = Lattice(m, rp)
    lat.set_state(f, p, sf)
    lat.initialize()
    lat.evolve(200)
    f1, p1, _ = lat.get_state()
    lat.close()
    G1, r1 = gauss_field(rp, m, f1, p1)
    assert np.abs(r1 - r0).max() > 1e-6 * np.abs(r0).max()
    assert np.abs(G1 - G0).max() < 1e-12 * np.abs(r0).max()


def test_u1_rejects_unsupported_requests():
    from cosmolattice_b200 import Lattice, _capi

    par, rp, m, f, p, sf = make_u1_case(N=8)
    lat = Lattice(m, rp)
    lat.set_state(f, p, sf)
    lat.initialize()
    with pytest.raises(_capi.ClbError) as e:
        lat.spectrum(which=0, comp=5)
    assert e.value.code == _capi.CLB_EINVAL
    with pytest.raises(ValueError):
        lat.set_state(f[:2], p[:2], sf)
    lat.close()


def test_u1_spectra_match_numpy():
    # field and momentum spectra of matter (a^{2 alpha - 6}) and gauge (a^{2 alpha - 2}) components
    from cosmolattice_b200 import Lattice
    from oracle.spectrum import spectrum

    N = 16
    par, rp, m, f, p, sf = make_u1_case(N=N, evolver="VV2", expansion=True)
    lat = Lattice(m, rp)
    lat.set_state(f, p, sf)
    lat.initialize()
    lat.evolve(20)
    fg, pg, s = lat.get_state()
    fg, pg = fg.reshape(5, N, N, N), pg.reshape(5, N, N, N)
    for which, arr in ((0, fg), (1, pg)):
        for comp in (0, 1, 3):
            fac = 1.0 if which == 0 else s["aI"] ** (2 * m.alpha - (2 if comp >= 2 else 6))
            k, v, c = lat.spectrum(which=which, comp=comp)
            ko, vo, co = spectrum(arr[comp], rp.dx, factor=fac)
            assert c.tolist() == co.tolist()
            assert np.abs(v - vo).max() <= 1e-10 * np.abs(vo).max()
    lat.close()


def test_u1_fp32_form_tracks_fp64():
    # FP32 storage and stencils, FP64 momentum increments, drifts, volume sums and a(t).  Measured
    # over 100 VV2 steps with expansion (N = 16, random links): a(t) and the energies follow FP64
    # within the bounds below, the Gauss constraint stays satisfied to FP32 roundoff, and the
    # spectra of a matter and a gauge component agree to 1e-5 of their peak.
    from cosmolattice_b200 import Lattice

    par, rp, m, f, p, sf = make_u1_case(N=16, evolver="VV2", expansion=True, amp=2e-2)
    rng = np.random.default_rng(11)
    f = f.copy()
    f[2:] = rng.normal(0.0, 0.05, f[2:].shape)
    res = {}
    for prec in ("fp64", "fp32"):
        lat = Lattice(m, rp, precision=prec)
        lat.set_state(f, p, sf)
        lat.initialize()
        m0 = lat.measure(1.0)
        lat.evolve(100)
        lat.sync()
        mm = lat.measure(m0["energies"][-1])
        sp = [lat.spectrum(which=w, comp=c)[1] for w, c in ((0, 0), (0, 3), (1, 2))]
        res[prec] = (lat.get_state(), mm, sp)
        lat.close()
    (fa, pa, sa), ma, va = res["fp32"]
    (fb, pb, sb), mb, vb = res["fp64"]
    etot = mb["energies"][-1]
    ediff = max(abs(x - y) / etot for x, y in zip(ma["energies"], mb["energies"]))
    sdiff = max(np.abs(x - y).max() / np.abs(y).max() for x, y in zip(va, vb))
    print("u1 fp32-vs-fp64: a", abs(sa["aI"] - sb["aI"]) / sb["aI"], "energies/Etot", ediff,
          "gauss ratio", ma["gauss_u1"][0], mb["gauss_u1"][0], "spectra", sdiff,
          "fields", rel_comp(fa, fb, 16), "momenta", rel_comp(pa, pb, 16))
    assert abs(sa["aI"] - sb["aI"]) <= 1e-7 * sb["aI"]
    assert ediff <= 1e-5
    assert ma["gauss_u1"][0] <= 1e-4
    assert abs(ma["gauss_u1"][2] - mb["gauss_u1"][2]) <= 1e-4 * mb["gauss_u1"][2]
    assert sdiff <= 1e-5


# ---- position Verlet for lphi4U1 (PositionVerlet::evolve, positionverlet.h:45-99) -------------

@pytest.mark.parametrize("evolver,expansion", [("PV2", True), ("PV2", False), ("PV4", True), ("PV6", True)])
def test_lphi4u1_position_verlet(evolver, expansion):
    g, c, meas = run_pair(16, evolver, expansion, 30, measure_every=7, links=0.05)
    check_state(g, c, 16)
    check_meas(meas["gpu"], meas["cpu"])


def test_lphi4u1_position_verlet_fp32_and_adjoint_guard():
    from cosmolattice_b200 import Lattice, _capi

    par, rp, m, f, p, sf = make_u1_case(N=16, evolver="PV4", dt=0.01, amp=2e-2)
    out = {}
    for prec in ("fp64", "fp32"):
        lat = Lattice(m, rp, precision=prec)
        lat.set_state(f, p, sf)
        lat.initialize()
        lat.evolve(20)
        lat.sync()
        out[prec] = lat.measure(1.0)
        if prec == "fp64":
            with pytest.raises(_capi.ClbError):
                lat.forward(4, 2, [0, 0, 1, 1, 0])  # the adjoint covers the VV evolvers
        lat.close()
    assert abs(out["fp32"]["aI"] - out["fp64"]["aI"]) <= 1e-7 * out["fp64"]["aI"]
    for x, y in zip(out["fp32"]["energies"], out["fp64"]["energies"]):
        assert abs(x - y) <= 1e-4 * abs(out["fp64"]["energies"][-1])


# ---- fixed background for lphi4U1 (fixedbackgroundexpansion.h:21-45) ---------------------------

@pytest.mark.parametrize("evolver", ["VV2", "VV4", "LF", "PV2"])
def test_lphi4u1_fixed_background(evolver):
    fb = {"fixedBackground": "true", "H0": 2.0e18, "omegaEoS": 1.0 / 3.0}
    g, c, meas = run_pair(16, evolver, True, 30, measure_every=7, links=0.05, extra=fb)
    check_state(g, c, 16)
    check_meas(meas["gpu"], meas["cpu"])


def test_lphi4u1_fixed_background_rejects_the_adjoint():
    from cosmolattice_b200 import Lattice, _capi

    par, rp, m, f, p, sf = make_u1_case(N=8, extra={"fixedBackground": "true", "H0": 2.0e18})
    lat = Lattice(m, rp)
    lat.set_state(f, p, sf)
    lat.initialize()
    with pytest.raises(_capi.ClbError):
        lat.forward(4, 2, [0, 0, 1, 1, 0])  # the adjoint covers the self-consistent expansion
    lat.close()


def test_gradient_workload_geometry_128_vv4_100_steps():
    # the lphi4U1 gradient workload's lattice: 128^3, VV4, dt = 0.005, g = 0.5, amplitude 1e-3,
    # self-consistent expansion, 100 steps from identical arrays
    N = 128
    g, c, meas = run_pair(N, "VV4", True, 100, dt=0.005, amp=1e-3, extra={"gU1s": 0.5})
    check_state(g, c, N)
    check_meas(meas["gpu"], meas["cpu"])


@pytest.mark.parametrize("N,evolver,expansion,precision", [(20, "VV2", False, "fp64"), (36, "VV4", False, "fp64"),
                                                           (36, "LF", True, "fp64"), (20, "VV2", True, "fp32"),
                                                           (36, "PV2", False, "fp32")])
def test_staged_kick_equals_site_kick(monkeypatch, N, evolver, expansion, precision):
    # the kick on staged planes (k_u1_kick_tile, the default) and the site-by-site kick (CLB_U1_TILE=0)
    # evaluate every site with the same arithmetic: without expansion (no volume sums feed back) the
    # states agree bitwise; with expansion a(t) takes the sums in another order, 1e-13.  N = 20 and
    # 36 leave partial tiles in z (32 sites) and y (8 rows); x-runs of 16 and 5 planes.
    from cosmolattice_b200 import Lattice

    par, rp, m, f, p, sf = make_u1_case(N=N, evolver=evolver, expansion=expansion, amp=3e-2)
    out = []
    for env in ({"CLB_U1_TILE": "0"}, {}, {"CLB_U1_TILE_LX": "5"}):
        monkeypatch.delenv("CLB_U1_TILE", raising=False)
        monkeypatch.delenv("CLB_U1_TILE_LX", raising=False)
        for k, v in env.items():
            monkeypatch.setenv(k, v)
        lat = Lattice(m, rp, precision=precision)
        lat.set_state(f, p, sf)
        lat.initialize()
        lat.evolve(12)
        lat.sync()
        out.append(lat.get_state())
        lat.close()
    (f0, p0, s0) = out[0]
    for fg, pg, sg in out[1:]:
        if not expansion:
            assert np.array_equal(fg, f0) and np.array_equal(pg, p0)
        else:
            assert np.abs(fg - f0).max() <= 1e-13 * np.abs(f0).max()
            assert np.abs(pg - p0).max() <= 1e-13 * np.abs(p0).max()
            assert abs(sg["aI"] - s0["aI"]) <= 1e-14 * s0["aI"]
