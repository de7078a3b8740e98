"""The C++20 host program (cosmolattice_b200/host/cosmolattice_b200.cpp): the reference's main loop
(source/cosmolattice.cpp:134-201) for lphi4, lphi4U1 and lphi4SU2U1 (with or without GWs) over the
C ABI.

CPU: it is built with the library and rejects an incomplete parameter set before any CUDA call.
GPU: its output files equal, row by row, the measurements of the same run driven from Python over
the same ABI (same device seed, same cadence), to the 15 significant digits the files carry.
"""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "cosmolattice_b200", "lib", "cosmolattice_b200")

PARAMS = {
    "N": 32, "kIR": 1.0, "dt": 0.01, "tMax": 0.5, "tOutputFreq": 0.1, "evolver": "VV2", "expansion": "true",
    "lambda": 1.0, "initial_amplitudes": "5.6964e18", "initial_momenta": "0", "fluct_amplitude": 1e-3,
    "kCutOff": 8.0, "baseSeed": "host",
}


def built():
    if not os.path.exists(BIN):
        from cosmolattice_b200.build import build_host

        build_host()
    return BIN


def test_host_rejects_missing_parameters():
    r = subprocess.run([built(), "N=8", "kIR=1"], capture_output=True, text=True)
    assert r.returncode == 1
    assert "Parameter dt is missing." in r.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("evolver,extra", [("VV2", {}), ("PV4", {}), ("LF", {"fixedBackground": "true", "H0": 2.0e18})])
def test_host_matches_python_over_the_abi(tmp_path, evolver, extra):
    from cosmolattice_b200 import Lattice, ParameterParser, RunParameters, lphi4_1f
    from cosmolattice_b200.initializers import device_ic_params
    from cosmolattice_b200.lattice import c_round

    params = dict(PARAMS, evolver=evolver, **extra)
    seed = 7
    args = [f"{k}={v}" for k, v in params.items()] + [f"outputfile={tmp_path}", f"deviceSeed={seed}"]
    r = subprocess.run([built()] + args, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    host_en = np.loadtxt(tmp_path / "average_energies.txt", ndmin=2)
    host_sf = np.loadtxt(tmp_path / "average_scale_factor.txt", ndmin=2)

    par = ParameterParser(params=params)
    rp = RunParameters(par)
    m = lphi4_1f(par, rp)
    lat = Lattice(m, rp)
    p, aI, aD = device_ic_params(m, rp, seed=seed)
    lat.generate_state(p, {"aI": aI, "aSI": aI, "aIM": aI, "aDotI": aD, "aDotSI": aD})
    lat.initialize(correct_adot=True)
    out_freq = c_round(rp.tOutFreq / rp.dt)
    rows_en, rows_sf = [], []
    t, i, e0 = rp.t0, 0, None
    while t < rp.tMax - rp.dt / 2.0:
        if i % out_freq == 0:
            lat.sync()
            mm = lat.measure(e0 if e0 is not None else 1.0)
            if e0 is None:
                e0 = mm["energies"][-1]
            rows_en.append([t] + mm["energies"])
            rows_sf.append([t, mm["aI"], mm["aDotI"], mm["hubble"]])
        n = max(1, min(out_freq - i % out_freq, c_round((rp.tMax - t) / rp.dt)))
        lat.evolve(n)
        t += n * rp.dt
        i += n
    lat.close()
    py_en, py_sf = np.array(rows_en), np.array(rows_sf)
    assert host_en.shape == py_en.shape and host_sf.shape == py_sf.shape
    assert np.allclose(host_en, py_en, rtol=1e-13, atol=0)
    assert np.allclose(host_sf, py_sf, rtol=1e-13, atol=0)


GAUGE = {
    "lphi4U1": {"N": 12, "kIR": 1.0, "dt": 0.01, "tMax": 0.3, "tOutputFreq": 0.05, "tOutputInfreq": 0.1,
                "evolver": "VV2", "expansion": "true", "lambda": 1.0, "cmplx_field_initial_norm": "5.6964e18",
                "gU1s": 0.5, "fluct_amplitude": 1e-2, "kCutOff": 3.0, "baseSeed": "host"},
    "lphi4SU2U1": {"N": 8, "kIR": 1.0, "dt": 0.005, "tMax": 0.15, "tOutputFreq": 0.025, "tOutputInfreq": 0.05,
                   "evolver": "VV2", "expansion": "true", "lambda": 1.0, "qG": 50, "qH": 50,
                   "SU2Doublet_initial_norm": "5.25151e18", "gU1s": 0.35, "gSU2s": 0.6, "fluct_amplitude": 1e-2,
                   "kCutOff": 2.0, "baseSeed": "host"},
}


def _python_files(model_name, params, seed, outdir):
    """The same run driven from Python over the ABI: device initial state with the same seed, the
    reference's cadence, files written by lattice.Measurer."""
    from cosmolattice_b200 import MODELS, Lattice, ParameterParser, RunParameters
    from cosmolattice_b200.initializers import device_ic_params
    from cosmolattice_b200.lattice import Measurer, c_round

    par = ParameterParser(params=dict(params, print_headers="true"))
    rp = RunParameters(par)
    m = MODELS[model_name](par, rp)
    lat = Lattice(m, rp)
    if rp.withGWs:
        lat.gws_enable()
    p, aI, aD = device_ic_params(m, rp, seed=seed)
    lat.generate_state(p, {"aI": aI, "aSI": aI, "aIM": aI, "aDotI": aD, "aDotSI": aD})
    lat.initialize(correct_adot=True)
    meas = Measurer(m, rp, outdir)
    t, i = rp.t0, 0
    while t < rp.tMax - rp.dt / 2.0:
        if i % meas.outputFreq == 0 or i % meas.spectraFreq == 0:
            lat.sync()
        if i % meas.outputFreq == 0:
            meas.measure(i, t, lat)
        if i % meas.spectraFreq == 0:
            meas.measure_spectra(t, lat)
            if rp.withGWs:
                meas.measure_gws(t, lat)
        n = min(meas.outputFreq - i % meas.outputFreq, meas.spectraFreq - i % meas.spectraFreq)
        n = max(1, min(n, c_round((rp.tMax - t) / rp.dt)))
        lat.evolve(n)
        t += n * rp.dt
        i += n
    meas.close()
    lat.close()


def _numbers(path):
    rows = []
    for line in open(path):
        if line.strip() and not line.startswith("#") and not line.startswith("1:"):
            rows.append([float(x) for x in line.split()])
    return np.array(rows)


@pytest.mark.gpu
@pytest.mark.parametrize("model", list(GAUGE))
def test_host_gauge_models_match_python(tmp_path, model):
    # every file the host writes for the gauge models (energies, Friedmann, scale factor, the means
    # of every field, both Gauss laws, the spectra) equals the Python-driven run's file of the same
    # name, line by line, within 1e-13 of each column's largest value (NaN where the reference's
    # sqrt of a rounded-negative SU(2) B^2 gives one, on both sides)
    params = GAUGE[model]
    seed = 11
    hdir, pdir = tmp_path / "host", tmp_path / "py"
    hdir.mkdir()
    args = [f"{k}={v}" for k, v in params.items()] + [f"model={model}", f"outputfile={hdir}", f"deviceSeed={seed}",
                                                      "print_headers=true"]
    r = subprocess.run([built()] + args, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    _python_files(model, params, seed, str(pdir))
    hfiles, pfiles = sorted(os.listdir(hdir)), sorted(os.listdir(pdir))
    assert hfiles == pfiles
    for name in hfiles:
        assert open(hdir / name).readline() == open(pdir / name).readline(), name  # same header
        a, b = _numbers(hdir / name), _numbers(pdir / name)
        assert a.shape == b.shape, name
        assert np.array_equal(np.isnan(a), np.isnan(b)), name
        # each column within 1e-13 of its largest magnitude: the two hosts form the initial-state
        # masses in their own operation order, so values that average to zero differ by 1e-19.
        # The Gauss files' violation column is itself a ratio of rounding residue (~1e-12) to the
        # charge scale: it is held to 1e-13 absolute instead.
        scale = np.nanmax(np.abs(b), axis=0, keepdims=True)
        if "gauss" in name:
            scale[0, 1] = 1.0
        assert np.all(np.nan_to_num(np.abs(a - b)) <= 1e-13 * scale), name


@pytest.mark.gpu
@pytest.mark.parametrize("model,evolver", [("lphi4U1", "VV2"), ("lphi4SU2U1", "LF")])
def test_host_gws_match_python(tmp_path, model, evolver):
    # withGWs: the host's spectra_energy_gws.txt and average_energies_gws.txt (gwsmeasurer.h:41-53)
    # equal the Python-driven run's, line by line, within 1e-13 of each column's largest value; a
    # restart file saved with GWs carries them (restart = true needs them when withGWs is set)
    params = dict(GAUGE[model], evolver=evolver, withGWs="true")
    seed = 13
    hdir, pdir = tmp_path / "host", tmp_path / "py"
    hdir.mkdir()
    save = tmp_path / "gw.clb"
    args = [f"{k}={v}" for k, v in params.items()] + [f"model={model}", f"outputfile={hdir}", f"deviceSeed={seed}",
                                                      "print_headers=true", f"saveFile={save}"]
    r = subprocess.run([built()] + args, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    _python_files(model, params, seed, str(pdir))
    for name in ("spectra_energy_gws.txt", "average_energies_gws.txt"):
        assert open(hdir / name).readline() == open(pdir / name).readline(), name
        a, b = _numbers(hdir / name), _numbers(pdir / name)
        assert a.shape == b.shape and len(a) > 2, name
        scale = np.nanmax(np.abs(b), axis=0, keepdims=True)
        assert np.all(np.abs(a - b) <= 1e-13 * scale), name
    assert _numbers(hdir / "average_energies_gws.txt")[-1, 1] > 0  # the GWs grew from zero
    hdr = np.fromfile(save, dtype="<i8", count=10)
    assert hdr[2 + 7] & 1  # the GW flag of the header's last word
    # a restart with GWs reads them back; without a GW flag in the file it is refused
    plain = tmp_path / "plain.clb"
    r = subprocess.run([built()] + [a for a in args if not a.startswith(("withGWs", "saveFile"))] +
                       [f"saveFile={plain}"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    for path, ok in ((save, True), (plain, False)):
        rdir = tmp_path / ("r_ok" if ok else "r_no")
        rdir.mkdir()
        rr = subprocess.run([built()] + [a for a in args if not a.startswith(("outputfile", "saveFile", "tMax"))] +
                            [f"outputfile={rdir}", "restart=true", f"restartFile={path}",
                             f"tMax={float(params['tMax']) + 5 * float(params['dt'])}"],
                            capture_output=True, text=True, timeout=300)
        assert (rr.returncode == 0) == ok, rr.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("model,evolver", [("lphi4", "VV2"), ("lphi4U1", "LF"), ("lphi4SU2U1", "VV2")])
def test_host_restart_continues_the_run(tmp_path, model, evolver):
    # a run saved half way (saveFile) and restarted from the file (restart = true) writes, for the
    # second half, the rows that the uninterrupted run writes
    params = dict(GAUGE.get(model, PARAMS), evolver=evolver)
    dt = float(params["dt"])
    t_half = 10 * dt
    base = [f"{k}={v}" for k, v in params.items() if k != "tMax"] + [f"model={model}", "deviceSeed=5",
                                                                      f"tOutputFreq={5 * dt}", f"tOutputInfreq={5 * dt}"]
    whole, first, second = tmp_path / "whole", tmp_path / "first", tmp_path / "second"
    for d in (whole, first, second):
        d.mkdir()
    path = tmp_path / "half.clb"
    runs = [base + [f"tMax={2 * t_half}", f"outputfile={whole}"],
            base + [f"tMax={t_half}", f"outputfile={first}", f"saveFile={path}"],
            base + [f"tMax={2 * t_half}", f"outputfile={second}", "restart=true", f"restartFile={path}"]]
    for args in runs:
        r = subprocess.run([built()] + args, capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stderr
    a = _numbers(whole / "average_energies.txt")
    b = _numbers(second / "average_energies.txt")
    assert len(b) == 2 and np.allclose(a[-2:, 0], b[:, 0], rtol=1e-15)  # t = 10 dt, 15 dt
    assert np.allclose(a[-2:], b, rtol=1e-11, atol=0)
