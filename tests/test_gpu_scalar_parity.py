"""Parity of the CUDA scalar-singlet path with the FP64 CPU oracle (runs on a B200).

Tolerances (the north star's (a)): started from identical arrays, after 100 steps, fields and
momenta per site within 1e-12 relative to the array's max |value| and to each site's own value
wherever it exceeds 1e-1 of the array's max (conftest.site_metrics), and within 2e-12 of the
fluctuations' own scale max |x - <x>| (the field is ~1 with fluctuations ~1e-3, so the first bar
alone would check them only to 1e-9; measured up to 1.5e-12, for the momenta of the position-
Verlet runs, whose stages hold more rounded drifts).  a(t), aDot, volume averages and energies
within 1e-10 relative.  The same bars hold at the headline geometry (512^3, kIR = 1/8).  The
FP32/FP64-split form is checked against the same oracle with its own stated bounds, in the linear
regime and in a nonlinear one (fluctuations of 30% of the field).
"""
import numpy as np
import pytest

from conftest import make_scalar_case, site_metrics

pytestmark = pytest.mark.gpu

SITE_TOL = 1e-12
FLUCT_TOL = 2e-12
AVG_TOL = 1e-10


def rel(a, b):
    return np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-300)


def run_pair(N, evolver, expansion, nsteps, model="lphi4_1f", path="fused", precision="fp64", measure_every=None,
             dt=0.01, amp=1e-3, extra=None):
    from cosmolattice_b200 import Lattice
    from oracle.oracle import OracleLattice

    par, rp, m, f, p, sf = make_scalar_case(N=N, evolver=evolver, expansion=expansion, model=model, dt=dt, amp=amp,
                                            extra=extra)
    gpu = Lattice(m, rp, precision=precision, path=path)
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


def check_state(g, c, site_tol=SITE_TOL, sf_tol=AVG_TOL, fluct_tol=FLUCT_TOL):
    (fg, pg, sg), (fc, pc, sc) = g, c
    assert rel(fg, fc) < site_tol, rel(fg, fc)
    assert rel(pg, pc) < site_tol, rel(pg, pc)
    nc = 1 if round(fg.size ** (1 / 3)) ** 3 == fg.size else 2  # N^3 or 2 N^3 values (one or two fields)
    for what, a, b in (("fields", fg, fc), ("momenta", pg, pc)):
        site, fluct = site_metrics(a, b, nc)
        assert site < site_tol, (what, "per-site", site)
        assert fluct < fluct_tol, (what, "fluctuations", fluct)
    for k in ("aI", "aDotI"):
        assert abs(sg[k] - sc[k]) <= sf_tol * max(abs(sc[k]), 1e-300), (k, sg[k], sc[k])


def check_meas(mg, mc, tol=AVG_TOL):
    for a, b in zip(mg, mc):
        assert rel(a["energies"], b["energies"]) < tol
        for ea, eb in zip(a["energies"], b["energies"]):
            assert abs(ea - eb) <= tol * abs(eb) + 1e-300, (ea, eb)
        assert abs(a["friedmann"][1] - b["friedmann"][1]) <= tol * abs(b["friedmann"][1]) + 1e-300
        assert abs(a["friedmann"][2] - b["friedmann"][2]) <= tol * abs(b["friedmann"][2]) + 1e-300
        for ra, rb in zip(a["means"], b["means"]):
            # <phi>, <dphi/dt>, <phi^2>, <(dphi/dt)^2>; a mean that averages to ~0 is compared on
            # the scale of its field's rms
            scales = [max(abs(rb[0]), rb[4]), max(abs(rb[1]), rb[5]), abs(rb[2]), abs(rb[3])]
            for x, y, sc in zip(ra[:4], rb[:4], scales):
                assert abs(x - y) <= tol * max(sc, 1e-300), (x, y)


@pytest.mark.parametrize("path", ["fused", "reference"])
@pytest.mark.parametrize("expansion", [True, False])
def test_lphi4_64_vv2_100_steps(path, expansion):
    g, c, meas = run_pair(64, "VV2", expansion, 100, path=path)
    check_state(g, c)
    check_meas(meas["gpu"], meas["cpu"])


@pytest.mark.parametrize("evolver", ["VV4", "VV6", "VV8", "VV10", "VV6_2"])
def test_higher_order_vv(evolver):
    g, c, meas = run_pair(24, evolver, True, 20)
    check_state(g, c)
    check_meas(meas["gpu"], meas["cpu"])


@pytest.mark.parametrize("path", ["fused", "reference"])
@pytest.mark.parametrize("expansion", [True, False])
def test_leapfrog_with_syncs(path, expansion):
    # LF momenta live at half steps; sync + measure every 7 steps exercises the half-kick restart
    # and the averages refreshed by the Friedmann measurement (energies.h:219).
    g, c, meas = run_pair(32, "LF", expansion, 50, path=path, measure_every=7)
    check_state(g, c)
    check_meas(meas["gpu"], meas["cpu"])


@pytest.mark.parametrize("evolver", ["VV2", "LF"])
def test_two_field_lphi4(evolver):
    g, c, meas = run_pair(32, evolver, True, 40, model="lphi4")
    check_state(g, c)
    check_meas(meas["gpu"], meas["cpu"])


@pytest.mark.parametrize("N", [2, 3, 12, 20, 48, 40])
def test_ragged_sizes(N):
    # sizes that do not fill the 32 x 8 column tile, including the smallest periodic lattices
    g, c, meas = run_pair(N, "VV2", True, 15, amp=1e-2)
    check_state(g, c)
    check_meas(meas["gpu"], meas["cpu"])


def test_measure_cadence_vv():
    g, c, meas = run_pair(32, "VV4", True, 30, measure_every=4)
    check_state(g, c)
    check_meas(meas["gpu"], meas["cpu"])


def test_deterministic_reductions():
    from cosmolattice_b200 import Lattice

    par, rp, m, f, p, sf = make_scalar_case(N=48, evolver="VV2", expansion=True)
    outs = []
    for _ in range(2):
        lat = Lattice(m, rp)
        lat.set_state(f, p, sf)
        lat.initialize()
        lat.evolve(25)
        outs.append(lat.get_state())
        lat.close()
    assert np.array_equal(outs[0][0], outs[1][0]) and np.array_equal(outs[0][1], outs[1][1])
    assert outs[0][2] == outs[1][2]


def test_fp32_split_against_fp64():
    # FP32 fields/momenta/stencils with FP64 reductions and a(t): field error bounded by FP32
    # rounding accumulated over the run; a(t) and the Friedmann constraint follow FP64 closely.
    g, c, meas = run_pair(64, "VV2", True, 100, precision="fp32")
    (fg, pg, sg), (fc, pc, sc) = g, c
    assert rel(fg, fc) < 1e-6
    fluct_g = fg - fg.mean()
    fluct_c = fc - fc.mean()
    assert rel(fluct_g, fluct_c) < 1e-3
    assert abs(sg["aI"] - sc["aI"]) / sc["aI"] < 1e-7
    fr_g = meas["gpu"][-1]["friedmann"][0]
    fr_c = meas["cpu"][-1]["friedmann"][0]
    assert abs(fr_g - fr_c) < 1e-6


def test_errors_surface_through_the_abi():
    from cosmolattice_b200 import Lattice, _capi

    par, rp, m, f, p, sf = make_scalar_case(N=8, evolver="VV2", expansion=True)
    lat = Lattice(m, rp)
    with pytest.raises(_capi.ClbError) as ei:
        lat.evolve(1)
    assert ei.value.code == _capi.CLB_ESTATE
    bad = f.copy()
    bad.ravel()[5] = np.nan
    lat.set_state(bad, p, sf)
    with pytest.raises(_capi.ClbError) as ei:
        lat.initialize()
    assert ei.value.code == _capi.CLB_ENONFINITE
    lat.close()


# ---- position Verlet (PositionVerlet::evolve, positionverlet.h:45-99) --------------------------

@pytest.mark.parametrize("path", ["fused", "reference"])
@pytest.mark.parametrize("expansion", [True, False])
def test_pv2_64_100_steps(path, expansion):
    g, c, meas = run_pair(64, "PV2", expansion, 100, path=path)
    check_state(g, c)
    check_meas(meas["gpu"], meas["cpu"])


@pytest.mark.parametrize("evolver", ["PV4", "PV6", "PV8", "PV10", "PV6_2"])
def test_higher_order_pv(evolver):
    g, c, meas = run_pair(24, evolver, True, 20)
    check_state(g, c)
    check_meas(meas["gpu"], meas["cpu"])


def test_pv_two_fields_and_measure_cadence():
    g, c, meas = run_pair(32, "PV4", True, 30, model="lphi4", measure_every=4)
    check_state(g, c)
    check_meas(meas["gpu"], meas["cpu"])


@pytest.mark.parametrize("path", ["fused", "reference"])
def test_pv_fp32_split_against_fp64(path):
    g, c, meas = run_pair(48, "PV4", True, 50, precision="fp32", path=path)
    (fg, pg, sg), (fc, pc, sc) = g, c
    assert rel(fg, fc) < 1e-6
    assert rel(fg - fg.mean(), fc - fc.mean()) < 1e-3
    assert abs(sg["aI"] - sc["aI"]) / sc["aI"] < 1e-7
    assert abs(meas["gpu"][-1]["friedmann"][0] - meas["cpu"][-1]["friedmann"][0]) < 1e-6


def test_pv_history_rows_match_measurements():
    # the fused path's step-end drift sweep books the integer-time field averages of each step
    from cosmolattice_b200 import Lattice

    par, rp, m, f, p, sf = make_scalar_case(N=24, evolver="PV4", expansion=True)
    lat = Lattice(m, rp)
    lat.set_state(f, p, sf)
    lat.initialize()
    lat.evolve(6)
    hist = lat.history()
    lat.sync()
    mm = lat.measure(1.0)
    lat.close()
    assert len(hist) == 6
    assert abs(hist[-1][0] - mm["aI"]) <= 1e-15 * mm["aI"]
    assert abs(hist[-1][1] - mm["aDotI"]) <= 1e-15 * abs(mm["aDotI"])


# ---- fixed background (FixedBackgroundExpansion, fixedbackgroundexpansion.h:21-45) --------------

# H0 = 0.5 in program units: omega_* = sqrt(lambda) phi_0 = 5.6964e18 GeV for the lphi4_1f case
FB = {"fixedBackground": "true", "H0": 0.5 * 5.6964e18, "omegaEoS": 1.0 / 3.0}


@pytest.mark.parametrize("path", ["fused", "reference"])
@pytest.mark.parametrize("evolver", ["VV2", "VV4", "PV2", "PV4"])
def test_fixed_background_parity(path, evolver):
    g, c, meas = run_pair(32, evolver, True, 30, path=path, extra=FB, measure_every=7)
    check_state(g, c)
    check_meas(meas["gpu"], meas["cpu"])


@pytest.mark.parametrize("path", ["fused", "reference"])
def test_fixed_background_leapfrog_with_syncs(path):
    g, c, meas = run_pair(32, "LF", True, 30, path=path, extra=FB, measure_every=7)
    check_state(g, c)
    check_meas(meas["gpu"], meas["cpu"])


def test_fixed_background_scale_factor_closed_form():
    # a(t) = (1 + H0/p t)^p, aDot = H0 (1 + H0/p t)^(p-1), p = 2/(3(1 + w) - 2 alpha), at t = n dt
    g, c, meas = run_pair(16, "VV2", True, 40, extra=FB)
    (fg, pg, sg) = g
    p = 2.0 / (3.0 * (1.0 + 1.0 / 3.0) - 2.0 * 1.0)
    t = 0.0
    for _ in range(40):
        t += 0.01
    a = (1 + 0.5 / p * t) ** p
    ad = 0.5 * (1 + 0.5 / p * t) ** (p - 1)
    assert abs(sg["aI"] - a) <= 1e-15 * a
    assert abs(sg["aDotI"] - ad) <= 1e-15 * ad


KNOBS = ("CLB_SWEEP_SHAPE", "CLB_SWEEP_XS", "CLB_SWEEP_RING_KB", "CLB_PDL")


@pytest.mark.parametrize("precision,tol,atol", [("fp64", 1e-12, 1e-13), ("fp32", 1e-6, 1e-9)])
def test_sweep_launch_knobs_compute_the_same_step(monkeypatch, precision, tol, atol):
    # Block shape, x-run (64, 8 and 4 planes per block), ring depth and dependent launch change only
    # how the sweep is scheduled: the state after 20 VV2 steps matches the default's within the
    # reordering of the volume sums' block partials (1e-12 FP64; FP32 storage 1e-6).  The FP32
    # form sums each plane in FP32 first, in an order set by the tile shape, so its a(t) moves in
    # the 12th digit (2.8e-12 between two shapes), far inside its 1e-7 bar against FP64.
    from cosmolattice_b200 import Lattice

    par, rp, m, f, p, sf = make_scalar_case(N=64, evolver="VV2", expansion=True, amp=1e-2)
    settings = [{}, {"CLB_SWEEP_SHAPE": "0"}, {"CLB_SWEEP_SHAPE": "1"}, {"CLB_SWEEP_SHAPE": "2"},
                {"CLB_SWEEP_SHAPE": "3"}, {"CLB_SWEEP_SHAPE": "4"},
                {"CLB_SWEEP_XS": "1"}, {"CLB_SWEEP_XS": "8"}, {"CLB_SWEEP_XS": "16"},
                {"CLB_SWEEP_RING_KB": "64"}, {"CLB_PDL": "0"}]
    out = []
    for env in settings:
        for k in KNOBS:
            monkeypatch.delenv(k, raising=False)
        for k, v in env.items():
            monkeypatch.setenv(k, v)
        lat = Lattice(m, rp, precision=precision)
        lat.set_state(f, p, sf)
        lat.initialize()
        lat.evolve(20)
        out.append(lat.get_state())
        lat.close()
    f0, p0, s0 = out[0]
    for env, (fs, ps, ss) in zip(settings[1:], out[1:]):
        assert np.abs(fs - f0).max() <= tol * np.abs(f0).max(), env
        assert np.abs(ps - p0).max() <= tol * np.abs(p0).max(), env
        assert abs(ss["aI"] - s0["aI"]) <= atol * s0["aI"], env


# ---- the configurations' own geometry ------------------------------------------------------------

def test_headline_geometry_512_vv2_100_steps():
    # the 512^3 lattice of the throughput workload (kIR = 1/8, the 64^3 case's spacing; dt = 0.01,
    # VV2, expansion), 100 steps from identical arrays, against the oracle on all host cores;
    # fields, momenta, a(t), energies and the field spectrum (443 bins, counts bit-exact)
    import sys

    from cosmolattice_b200 import Lattice, ParameterParser, RunParameters, lphi4_1f
    from cosmolattice_b200.initializers import scalar_initial_state
    from oracle.oracle import OracleLattice
    from oracle.spectrum import spectrum

    sys.path.insert(0, __import__("os").path.dirname(__import__("os").path.dirname(__file__)))
    import bench

    par = ParameterParser(params=bench.workload_params(512, 100))
    rp = RunParameters(par)
    m = lphi4_1f(par, rp)
    f, p, aI, aD = scalar_initial_state(m, rp)
    sf = {"aI": aI, "aSI": aI, "aIM": aI, "aDotI": aD, "aDotSI": aD}
    out = {}
    for key, lat in (("gpu", Lattice(m, rp)), ("cpu", OracleLattice(m, rp))):
        lat.set_state(f, p, sf)
        lat.initialize()
        lat.sync()
        e0 = lat.measure(1.0)["energies"][-1]
        lat.evolve(100)
        lat.sync()
        mm = lat.measure(e0)
        spec = lat.spectrum(which=0) if key == "gpu" else None
        out[key] = (lat.get_state(), mm, spec)
        lat.close()
    del f, p
    (g, mg, sg), (c, mc, _) = out["gpu"], out["cpu"]
    check_state(g, c)
    check_meas([mg], [mc])
    k, v, cnt = sg
    ko, vo, co = spectrum(c[0].reshape(512, 512, 512), rp.dx)
    assert cnt.tolist() == co.tolist()
    band = vo > 1e-6 * vo.max()
    assert np.all(np.abs(v - vo)[band] <= AVG_TOL * np.abs(vo)[band])


@pytest.mark.parametrize("amp", [0.1, 0.3])
def test_fp32_split_nonlinear_regime(amp):
    # Fluctuations of 8% (amp 0.1) and 25% (amp 0.3) of the field at the start: the FP32 form
    # stores fluctuations about the FP64 homogeneous value, which gains nothing once they are a
    # large part of the field, and its kick is a plain FP32 fused multiply-add.  Against the FP64
    # oracle after 100 steps: Friedmann constraint within 1e-6, the field spectrum within 1e-4 over
    # its populated band (the north star's bars), energies within 1e-5, a(t) within 1e-7.
    g, c, meas = run_pair(64, "VV2", True, 100, precision="fp32", amp=amp)
    (fg, pg, sg), (fc, pc, sc) = g, c
    assert abs(sg["aI"] - sc["aI"]) <= 1e-7 * sc["aI"]
    mg, mc = meas["gpu"][-1], meas["cpu"][-1]
    assert abs(mg["friedmann"][0] - mc["friedmann"][0]) <= 1e-6
    for x, y in zip(mg["energies"], mc["energies"]):
        assert abs(x - y) <= 1e-5 * abs(y), (mg["energies"], mc["energies"])
    from oracle.spectrum import spectrum

    dx = 2 * np.pi / 64
    _, vg, cg = spectrum(fg.reshape(64, 64, 64), dx)
    _, vc, cc = spectrum(fc.reshape(64, 64, 64), dx)
    band = vc > 1e-6 * vc.max()
    assert np.all(np.abs(vg - vc)[band] <= 1e-4 * vc[band])
