"""Gravitational waves (clb_gws_*, clb_gw_spectrum) on the B200: the scalar singlets' sector, and
the gauge models' (lphi4U1, lphi4SU2U1) with the complex-scalar and U(1) sources of PITensor.h.

Against the oracle's restatement (the reference's default: a leapfrog for the GWs staggered over
the VV matter evolver, evolver.h:102-138; the kernel of gwskernels.h:27-33 with the PITensor.h
source): the GW field and momenta per site within 1e-12 of each component's max after 30 steps
taken in three calls with syncs between them, the matter state as in the scalar parity tests.
The GW energy spectrum against a numpy restatement of the TT projectors (gwsprojector.h) on the
same momenta: 1e-10 per populated bin, counts bit-exact.  A longitudinal-plus-trace tensor
projects to zero.  Parity with TempLat is unpinned: its ConstructSymTraceless, forwDiff and the
spectrum's integrate() are not on disk (the stated choices are in clb_gws.cu).
"""
import math

import numpy as np
import pytest

from conftest import make_scalar_case

pytestmark = pytest.mark.gpu


FB = {"fixedBackground": "true", "H0": 2.0e18}  # a fixed radiation-like background


def _pair(model, evolver, precision="fp64", N=24, extra=None):
    from cosmolattice_b200 import Lattice
    from oracle.oracle import OracleLattice

    par, rp, m, f, p, sf = make_scalar_case(N=N, evolver=evolver, model=model, amp=3e-2, extra=extra)
    gpu, cpu = Lattice(m, rp, precision=precision), OracleLattice(m, rp)
    for lat in (gpu, cpu):
        lat.gws_enable()
        lat.set_state(f, p, sf)
        lat.initialize()
        for _ in range(3):
            lat.evolve(10)
            lat.sync()
    return rp, m, gpu, cpu


@pytest.mark.parametrize("model,evolver,fb", [("lphi4_1f", "VV2", False), ("lphi4_1f", "VV4", False),
                                             ("lphi4", "VV2", False), ("lphi4_1f", "LF", False),
                                             ("lphi4_1f", "PV2", False), ("lphi4_1f", "PV4", False),
                                             ("lphi4_1f", "VV2", True), ("lphi4_1f", "LF", True),
                                             ("lphi4_1f", "PV2", True)])
def test_gw_evolution_matches_oracle(model, evolver, fb):
    rp, m, gpu, cpu = _pair(model, evolver, extra=FB if fb else None)
    ug, pg = gpu.gws_get_state()
    uc, pc = cpu.gws_get_state()
    (fg, _, sg), (fc, _, sc) = gpu.get_state(), cpu.get_state()
    gpu.close()
    cpu.close()
    assert np.abs(pc).max() > 0 and np.abs(uc).max() > 0
    for a, b in ((ug, uc), (pg, pc)):
        for c in range(5):
            x, y = a.reshape(5, -1)[c], b.reshape(5, -1)[c]
            assert np.abs(x - y).max() <= 1e-12 * np.abs(y).max(), c
    assert np.abs(fg - fc).max() <= 1e-12 * np.abs(fc).max()
    assert abs(sg["aI"] - sc["aI"]) <= 1e-12 * sc["aI"]


@pytest.mark.parametrize("prj", [1, 2, 3])
@pytest.mark.parametrize("ps_type", [1, 2])
def test_gw_spectrum_matches_numpy(prj, ps_type):
    from oracle.spectrum import gw_spectrum

    rp, m, gpu, cpu = _pair("lphi4_1f", "VV2")
    cpu.close()
    N = rp.N
    k, v, cnt, frac = gpu.gw_spectrum(prj_type=prj, ps_type=ps_type)
    mm = gpu.measure(1.0)
    _, pi = gpu.gws_get_state()
    gpu.close()
    fac = (m.fStar / m.MPl) ** 2 / (4 * mm["aI"] ** 6 * mm["energies"][-1])
    ko, vo, co = gw_spectrum(pi.reshape(5, N, N, N), rp.dx, prj_type=prj, ps_type=ps_type, factor=fac)
    assert cnt.tolist() == co.tolist()
    band = vo > 1e-8 * vo.max()
    assert band.sum() > 3
    assert np.all(np.abs(v - vo)[band] <= 1e-10 * vo[band])
    assert np.allclose(k, ko, rtol=1e-12)
    ntil = ko / rp.kIR
    assert abs(frac - sum(vo[b] * 1.0 / ntil[b] for b in range(len(vo)) if co[b] > 0 and ntil[b] > 0)) <= 1e-10 * frac


def test_longitudinal_and_trace_parts_project_to_zero():
    # pi_ij = kL_i kL_j f(k) + delta_ij g(k), stored traceless, in Fourier space with the type-1
    # lattice momenta: the TT projector annihilates it, so its spectrum is rounding only, while a
    # transverse-traceless tensor of the same size keeps its power
    from cosmolattice_b200 import Lattice

    N = 16
    par, rp, m, f, p, sf = make_scalar_case(N=N, evolver="VV2", amp=1e-2)
    rng = np.random.default_rng(5)
    nx = np.fft.fftfreq(N, 1.0 / N)
    kL = [np.sin(2 * math.pi / N * nx)[:, None, None], np.sin(2 * math.pi / N * nx)[None, :, None],
          np.sin(2 * math.pi / N * nx)[None, None, :]]
    fk = np.fft.fftn(rng.normal(size=(N, N, N)))
    gk = np.fft.fftn(rng.normal(size=(N, N, N)))

    def comp(i, j):
        return np.real(np.fft.ifftn(kL[i] * kL[j] * fk + (gk if i == j else 0)))

    t = [[comp(i, j) for j in range(3)] for i in range(3)]
    tr3 = (t[0][0] + t[1][1] + t[2][2]) / 3
    pi_long = np.stack([t[0][0] - tr3, t[0][1], t[0][2], t[1][1] - tr3, t[1][2]])
    # transverse-traceless: modes with k along z only, u_11 = -u_22 = h(k), u_12 = h2(k)
    hz = np.fft.fftn(rng.normal(size=(N, N, N)))
    sel = (nx[:, None, None] == 0) & (nx[None, :, None] == 0) & (nx[None, None, :] != 0)
    h1 = np.real(np.fft.ifftn(np.where(sel, hz, 0)))
    pi_tt = np.stack([h1, h1, np.zeros_like(h1), -h1, np.zeros_like(h1)])
    out = {}
    for name, arr in (("long", pi_long), ("tt", pi_tt)):
        lat = Lattice(m, rp)
        lat.gws_enable()
        lat.set_state(f, p, sf)
        lat.initialize()
        lat.gws_set_state(np.zeros(5 * N ** 3), arr.ravel())
        _, v, _, _ = lat.gw_spectrum(prj_type=1)
        out[name] = v
        lat.close()
    scale = np.abs(pi_long).max() ** 2 / np.abs(pi_tt).max() ** 2
    assert out["tt"].max() > 0
    # rounding: the longitudinal tensor's projected power is ~1e-17 of its unprojected size
    assert out["long"].max() <= 1e-13 * scale * out["tt"].max()


def test_fp32_gws_track_fp64():
    rp, m, g64, cpu = _pair("lphi4_1f", "VV2")
    cpu.close()
    _, v64, _, f64 = g64.gw_spectrum()
    g64.close()
    rp, m, g32, cpu = _pair("lphi4_1f", "VV2", precision="fp32")
    cpu.close()
    _, v32, _, f32 = g32.gw_spectrum()
    g32.close()
    band = v64 > 1e-6 * v64.max()
    assert np.all(np.abs(v32 - v64)[band] <= 1e-4 * v64[band])
    assert abs(f32 - f64) <= 1e-4 * f64


def test_gws_refuse_the_scalar_reference_path():
    # the scalar singlets' GWs ride the fused path's loops; the reference-order path has none
    from cosmolattice_b200 import Lattice, _capi

    par, rp, m, f, p, sf = make_scalar_case(N=8)
    lat = Lattice(m, rp, path="reference")
    with pytest.raises(_capi.ClbError) as ei:
        lat.gws_enable()
    assert ei.value.code == _capi.CLB_EUNSUPPORTED
    lat.close()


def test_gauge_gws_refuse_the_adjoint_and_tangent_forms():
    # the adjoint pair and the tangent-linear form do not advance the GW sector, so neither runs
    # beside it
    from cosmolattice_b200 import Lattice, _capi
    from conftest import make_su2_case, make_u1_case

    par, rp, m, f, p, sf = make_u1_case(N=8)
    lat = Lattice(m, rp)
    lat.gws_enable()
    lat.set_state(f, p, sf)
    lat.initialize()
    with pytest.raises(_capi.ClbError) as ei:
        lat.forward(4, 2, [0, 0, 1, 1, 0])
    assert ei.value.code == _capi.CLB_EUNSUPPORTED
    lat.close()
    par, rp, m, f, p, sf = make_su2_case(N=8)
    for order in ("gws_first", "tangent_first"):
        lat = Lattice(m, rp)
        lat.set_state(f, p, sf)
        if order == "gws_first":
            lat.gws_enable()
            with pytest.raises(_capi.ClbError) as ei:
                lat.tangent_begin([0, 0, 0, 0, 1, 0])
        else:
            lat.tangent_begin([0, 0, 0, 0, 1, 0])
            with pytest.raises(_capi.ClbError) as ei:
                lat.gws_enable()
        assert ei.value.code == _capi.CLB_EUNSUPPORTED
        lat.close()


def _gauge_case(model, evolver, N, extra=None):
    from conftest import make_su2_case, make_u1_case

    if model == "lphi4U1":
        return make_u1_case(N=N, evolver=evolver, amp=3e-2, extra=extra)
    return make_su2_case(N=N, evolver=evolver, amp=3e-2, extra=extra)


def _gauge_pair(model, evolver, precision="fp64", N=12, gws=True, extra=None):
    from cosmolattice_b200 import Lattice
    from oracle.oracle import OracleLattice

    par, rp, m, f, p, sf = _gauge_case(model, evolver, N, extra)
    gpu, cpu = Lattice(m, rp, precision=precision), OracleLattice(m, rp)
    for lat in (gpu, cpu):
        if gws:
            lat.gws_enable()
        lat.set_state(f, p, sf)
        lat.initialize()
        for _ in range(3):
            lat.evolve(10)
            lat.sync()
    return rp, m, gpu, cpu


@pytest.mark.parametrize("model,evolver,fb", [("lphi4U1", "VV2", False), ("lphi4U1", "VV4", False),
                                             ("lphi4SU2U1", "VV2", False), ("lphi4U1", "LF", False),
                                             ("lphi4SU2U1", "LF", False), ("lphi4U1", "PV2", False),
                                             ("lphi4SU2U1", "PV4", False), ("lphi4U1", "VV2", True),
                                             ("lphi4U1", "LF", True), ("lphi4SU2U1", "VV2", True),
                                             ("lphi4U1", "PV2", True), ("lphi4SU2U1", "PV2", True)])
def test_gauge_gw_evolution_matches_oracle(model, evolver, fb):
    # the complex scalar, U(1) electric and magnetic (and for lphi4SU2U1 singlet) sources of
    # PITensor.h: GW field and momenta per component within 1e-12 of the component's max after 30
    # steps in three calls with syncs, against the oracle's restatement (fb: a fixed background)
    rp, m, gpu, cpu = _gauge_pair(model, evolver, extra=FB if fb else None)
    ug, pg = gpu.gws_get_state()
    uc, pc = cpu.gws_get_state()
    sg, sc = gpu.get_state()[2], cpu.get_state()[2]
    gpu.close()
    cpu.close()
    assert np.abs(pc).max() > 0 and np.abs(uc).max() > 0
    worst = 0.0
    for a, b in ((ug, uc), (pg, pc)):
        for c in range(5):
            x, y = a.reshape(5, -1)[c], b.reshape(5, -1)[c]
            worst = max(worst, np.abs(x - y).max() / np.abs(y).max())
    print(model, evolver, "fixed background" if fb else "", "GW rel. error", worst)
    assert worst <= 1e-12
    assert abs(sg["aI"] - sc["aI"]) <= 1e-12 * sc["aI"]


@pytest.mark.parametrize("model,evolver,fb", [("lphi4U1", "VV2", False), ("lphi4SU2U1", "VV2", False),
                                             ("lphi4U1", "LF", False), ("lphi4SU2U1", "VV2", True)])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_gauge_gws_leave_the_matter_evolution_bitwise(model, evolver, fb, precision):
    # the GWs do not act back, and their per-step schedule is that of one-step evolve calls: the
    # matter state and the scale factor equal those of a run without GWs to the last bit
    from cosmolattice_b200 import Lattice

    par, rp, m, f, p, sf = _gauge_case(model, evolver, 12, FB if fb else None)
    out = []
    for gws in (True, False):
        lat = Lattice(m, rp, precision=precision)
        if gws:
            lat.gws_enable()
        lat.set_state(f, p, sf)
        lat.initialize()
        lat.evolve(7)
        lat.sync()
        lat.evolve(5)
        out.append(lat.get_state())
        lat.close()
    (fa, pa, sa), (fb, pb, sb) = out
    assert np.array_equal(fa, fb) and np.array_equal(pa, pb) and sa == sb


def test_fp32_gauge_gws_track_fp64():
    rp, m, g64, cpu = _gauge_pair("lphi4U1", "VV2")
    cpu.close()
    u64, p64 = g64.gws_get_state()
    g64.close()
    rp, m, g32, cpu = _gauge_pair("lphi4U1", "VV2", precision="fp32")
    cpu.close()
    u32, p32 = g32.gws_get_state()
    g32.close()
    rel = max(np.abs(a - b).max() / np.abs(b).max() for a, b in ((u32, u64), (p32, p64)))
    print("fp32 gauge GW rel. error", rel)
    assert rel <= 3e-4


def test_gauge_gw_spectrum_matches_numpy():
    from oracle.spectrum import gw_spectrum

    rp, m, gpu, cpu = _gauge_pair("lphi4U1", "VV2")
    cpu.close()
    N = rp.N
    k, v, cnt, frac = gpu.gw_spectrum(prj_type=1, ps_type=1)
    mm = gpu.measure(1.0)
    _, pi = gpu.gws_get_state()
    gpu.close()
    fac = (m.fStar / m.MPl) ** 2 / (4 * mm["aI"] ** 6 * mm["energies"][-1])
    ko, vo, co = gw_spectrum(pi.reshape(5, N, N, N), rp.dx, prj_type=1, ps_type=1, factor=fac)
    assert cnt.tolist() == co.tolist()
    band = vo > 1e-8 * vo.max()
    assert band.sum() > 3
    assert np.all(np.abs(v - vo)[band] <= 1e-10 * vo[band])
    assert frac > 0


def test_run_writes_gw_files(tmp_path):
    from cosmolattice_b200 import ParameterParser, run

    params = {"N": 16, "kIR": 1.0, "dt": 0.01, "evolver": "VV2", "expansion": "true", "lambda": 1.0,
              "tMax": 0.3, "tOutputFreq": 0.1, "tOutputInfreq": 0.1, "kCutOff": 4, "fluct_amplitude": 3e-2,
              "initial_amplitudes": "5.6964e18", "initial_momenta": "0", "withGWs": "true", "print_headers": "true"}
    _, lat = run(ParameterParser(params=params), "lphi4_1f", outdir=str(tmp_path))
    lat.close()
    lines = open(tmp_path / "average_energies_gws.txt").read().splitlines()
    assert lines[0] == "#t    rhoGW_over_rho    rhoGW" and len(lines) == 4
    vals = np.array([list(map(float, l.split())) for l in lines[1:]])
    assert vals[0, 1] == 0.0 and np.all(vals[1:, 1] > 0)  # the GWs start at zero and grow
    assert (tmp_path / "spectra_energy_gws.txt").exists()
