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


@pytest.mark.parametrize("model", ["lphi4_1f", "lphi4U1"])
def test_restart_carries_the_gws(tmp_path, model):
    # saveSim/loadSim with GWs (simulationmanager.h:76-77, 112-113): the GW field and momenta come
    # back bitwise, and after the restart the GW leapfrog starts unsynced (GWsynced(!doWeRestart),
    # evolver.h:52); 10 more steps match the oracle restarted from the same arrays within 1e-12 of
    # each component's maximum.  A lattice with GWs refuses a file without them.
    from cosmolattice_b200 import Lattice, restart
    from oracle.oracle import OracleLattice

    case = make_scalar_case(N=12, amp=3e-2) if model == "lphi4_1f" else make_u1_case(N=12, amp=3e-2)
    par, rp, m, f, p, sf = case
    lat = Lattice(m, rp)
    lat.gws_enable()
    lat.set_state(f, p, sf)
    lat.initialize()
    lat.evolve(10)
    lat.sync()
    u0, p0 = lat.gws_get_state()
    F0, P0, S0 = lat.get_state()
    path = str(tmp_path / "gw.clb")
    restart.save_sim(path, lat, m, 10 * rp.dt)
    lat.close()

    again = Lattice(m, rp)
    again.gws_enable()
    restart.load_sim(path, again, m)
    u1, p1 = again.gws_get_state()
    assert np.array_equal(u0, u1) and np.array_equal(p0, p1)
    again.evolve(10)
    again.sync()
    ug, pg = again.gws_get_state()
    again.close()

    cpu = OracleLattice(m, rp)
    cpu.gws_enable()
    cpu.set_state(F0, P0, S0)
    cpu.gws_set_state(u0, p0)
    cpu.initialize(restart=True)
    cpu.evolve(10)
    cpu.sync()
    uc, pc = cpu.gws_get_state()
    cpu.close()
    for a, b in ((ug, uc), (pg, pc)):
        for c in range(5):
            x, y = a.reshape(5, -1)[c], b.reshape(5, -1)[c]
            assert np.abs(x - y).max() <= 1e-12 * np.abs(y).max(), c

    plain = Lattice(m, rp)
    plain.set_state(f, p, sf)
    plain.initialize()
    path2 = str(tmp_path / "plain.clb")
    restart.save_sim(path2, plain, m, 0.0)
    plain.close()
    withgw = Lattice(m, rp)
    withgw.gws_enable()
    with pytest.raises(ValueError):
        restart.load_sim(path2, withgw, m)
    withgw.close()
    # a run without GWs reads a file with them, as loadSim reads the GW datasets only for a model
    # with GWs
    nogw = Lattice(m, rp)
    restart.load_sim(path, nogw, m)
    Fn, Pn, _ = nogw.get_state()
    nogw.close()
    assert np.array_equal(Fn, F0) and np.array_equal(Pn, P0)
