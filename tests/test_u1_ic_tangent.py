"""The start-state tangents of the lphi4U1 initial state (used by the adjoint gradients) against
central differences of the initial-state generator itself (CPU)."""
import numpy as np
import pytest

from conftest import make_u1_case

KEYS = {"amp": "fluct_amplitude", "c4": "lambda_prog", "gQ": "gU1s"}


@pytest.mark.parametrize("param", ["amp", "c4", "gQ"])
def test_tangent_matches_central_difference(param):
    from cosmolattice_b200.initializers import u1_initial_state_tangent

    base = {"amp": 2e-2, "c4": 1.0, "gQ": 0.5}
    par, rp, m, f, p, sf = make_u1_case(N=12, amp=base["amp"], gU1=base["gQ"])
    df, dp = u1_initial_state_tangent(m, rp, param)
    h = 1e-4 * base[param]
    states = []
    for sgn in (1, -1):
        val = base[param] + sgn * h
        extra = {KEYS[param]: val} if param != "gQ" else {}
        _, _, _, f2, p2, _ = make_u1_case(N=12, amp=val if param == "amp" else base["amp"],
                                          gU1=val if param == "gQ" else base["gQ"], extra=extra)
        states.append((f2, p2))
    fd_f = (states[0][0] - states[1][0]) / (2 * h)
    fd_p = (states[0][1] - states[1][1]) / (2 * h)
    sc_f = max(np.abs(fd_f).max(), 1e-300)
    sc_p = max(np.abs(fd_p).max(), 1e-300)
    assert np.abs(df - fd_f).max() <= 1e-6 * sc_f + 1e-300
    assert np.abs(dp - fd_p).max() <= 1e-6 * sc_p


@pytest.mark.parametrize("param", ["gSU2", "gU1"])
def test_su2u1_tangent_matches_central_difference(param):
    # lphi4SU2U1: the Gauss-solved gauge momenta are linear in the couplings
    from conftest import make_su2_case
    from cosmolattice_b200.initializers import su2u1_initial_state_tangent

    base = {"gSU2": 0.6, "gU1": 0.35}
    par, rp, m, f, p, sf = make_su2_case(N=8, amp=3e-2, gSU2=base["gSU2"], gU1=base["gU1"])
    df, dp, cd = su2u1_initial_state_tangent(m, rp, param, (f, p))
    assert cd.tolist() == ([0, 0, 0, 0, 1, 0] if param == "gSU2" else [0, 0, 1, 1, 0, 0])
    h = 1e-4 * base[param]
    states = []
    for sgn in (1, -1):
        g = dict(base)
        g[param] += sgn * h
        states.append(make_su2_case(N=8, amp=3e-2, gSU2=g["gSU2"], gU1=g["gU1"])[3:5])
    fd_f = (states[0][0] - states[1][0]) / (2 * h)
    fd_p = (states[0][1] - states[1][1]) / (2 * h)
    assert np.abs(fd_f).max() == 0 and np.abs(df).max() == 0
    assert np.abs(dp - fd_p).max() <= 1e-6 * np.abs(fd_p).max()
