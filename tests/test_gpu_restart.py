"""Checkpoint and restart (SimulationManager::saveSim / loadSim, simulationmanager.h:69-141) through
cosmolattice_b200.restart on the B200.

A run saved after 20 steps and restarted into a fresh handle for 20 more steps ends where the same
40 steps end without the interruption.  The restart refreshes the cached volume averages from the
saved state (Averages::setAllAverages), so they can differ from the carried ones by the order of
the volume sums: state within 1e-13 of the uninterrupted run, energies within 1e-12.  The leapfrog
restarts unsynced (its momenta at the half step), as the reference's does.
"""
import numpy as np
import pytest

from conftest import make_scalar_case, make_su2_case, make_u1_case

pytestmark = pytest.mark.gpu

CASES = {
    "lphi4_1f": lambda ev: make_scalar_case(N=24, evolver=ev, amp=1e-2),
    "lphi4U1": lambda ev: make_u1_case(N=12, evolver=ev),
    "lphi4SU2U1": lambda ev: make_su2_case(N=8, evolver=ev, amp=3e-2),
}


@pytest.mark.parametrize("model", list(CASES))
@pytest.mark.parametrize("evolver", ["VV2", "LF"])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_restart_continues_the_run(tmp_path, model, evolver, precision):
    from cosmolattice_b200 import Lattice, restart

    par, rp, m, f, p, sf = CASES[model](evolver)
    path = str(tmp_path / "run.clb")
    whole = Lattice(m, rp, precision=precision)
    whole.set_state(f, p, sf)
    whole.initialize()
    whole.evolve(20)
    restart.save_sim(path, whole, m, 20 * rp.dt, par.params)
    whole.evolve(20)
    whole.sync()
    mw = whole.measure(1.0)
    fw, pw, sw = whole.get_state()
    whole.close()

    again = Lattice(m, rp, precision=precision)
    t, text = restart.load_sim(path, again, m)
    assert abs(t - 20 * rp.dt) < 1e-15 and "dt = " in text
    again.evolve(20)
    again.sync()
    ma = again.measure(1.0)
    fa, pa, sa = again.get_state()
    again.close()
    tol = 1e-13 if precision == "fp64" else 1e-6
    for x, y in ((fa, fw), (pa, pw)):
        n = x.size // rp.N ** 3
        for c in range(n):
            a, b = x.reshape(n, -1)[c], y.reshape(n, -1)[c]
            assert np.abs(a - b).max() <= tol * max(np.abs(b).max(), 1e-300), c
    assert abs(sa["aI"] - sw["aI"]) <= tol * sw["aI"]
    for x, y in zip(ma["energies"], mw["energies"]):
        assert abs(x - y) <= 1e3 * tol * abs(mw["energies"][-1])


def test_restart_with_fixed_background_is_refused(tmp_path):
    from cosmolattice_b200 import Lattice, _capi, restart

    par, rp, m, f, p, sf = make_scalar_case(N=8, extra={"fixedBackground": "true", "H0": 2.0e18})
    lat = Lattice(m, rp)
    lat.set_state(f, p, sf)
    lat.initialize()
    path = str(tmp_path / "fb.clb")
    restart.save_sim(path, lat, m, 0.0)
    with pytest.raises(_capi.ClbError) as ei:
        restart.load_sim(path, lat, m)
    assert ei.value.code == _capi.CLB_EUNSUPPORTED
    lat.close()
