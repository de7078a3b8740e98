"""The C++20 host program (cosmolattice_b200/host/cosmolattice_b200.cpp): the reference's main loop
(source/cosmolattice.cpp:134-201) for lphi4 over the C ABI.

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
