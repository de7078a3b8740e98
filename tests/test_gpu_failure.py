"""Failure detection of the scalar sweep's bounded waits (runs on a B200, faults nothing).

The sweep waits on shared-memory barriers for its TMA tile loads, each wait bounded by a number
of tries.  CLB_WAIT_TRIES, read when a handle is created, lowers that bound; at 0 every wait gives
up at once.  The sweep must then flag the abort, drain its loads still in flight under its own
fixed bound, and return; the call reports CLB_ETIMEOUT, the handle can be destroyed, and the
context stays usable for the next handle.
"""
import os

import numpy as np
import pytest

from conftest import make_scalar_case

pytestmark = pytest.mark.gpu


def _timed_out_handle(precision):
    from cosmolattice_b200 import Lattice

    par, rp, m, f, p, sf = make_scalar_case(N=32, evolver="VV2")
    os.environ["CLB_WAIT_TRIES"] = "0"
    try:
        lat = Lattice(m, rp, precision=precision, path="fused")
    finally:
        del os.environ["CLB_WAIT_TRIES"]
    return lat, f, p, sf


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_wait_that_runs_out_reports_etimeout(precision):
    from cosmolattice_b200 import _capi

    lat, f, p, sf = _timed_out_handle(precision)
    lat.set_state(f, p, sf)
    with pytest.raises(_capi.ClbError) as ei:
        lat.initialize()
        lat.evolve(3)
    assert ei.value.code == _capi.CLB_ETIMEOUT
    assert "bounded wait" in str(ei.value)
    lat.close()  # the handle is destroyed cleanly after the abort


def test_context_usable_after_timeout():
    from cosmolattice_b200 import Lattice
    from oracle.oracle import OracleLattice

    lat, f, p, sf = _timed_out_handle("fp64")
    lat.set_state(f, p, sf)
    with pytest.raises(Exception):
        lat.initialize()
        lat.evolve(2)
    lat.close()

    par, rp, m, f, p, sf = make_scalar_case(N=32, evolver="VV2")
    gpu = Lattice(m, rp, precision="fp64", path="fused")
    cpu = OracleLattice(m, rp)
    for lat in (gpu, cpu):
        lat.set_state(f, p, sf)
        lat.initialize()
        lat.evolve(5)
    (fg, pg, sg), (fc, pc, sc) = gpu.get_state(), cpu.get_state()
    gpu.close()
    cpu.close()
    assert np.abs(fg - fc).max() <= 1e-12 * np.abs(fc).max()
    assert np.abs(pg - pc).max() <= 1e-12 * np.abs(pc).max()
    assert abs(sg["aI"] - sc["aI"]) <= 1e-12 * sc["aI"]
