"""Known-answer tests that pin the CPU oracle (no GPU).

The reference's tests hold no golden vectors for the evolution (its only numeric test is the
couplings manager), so the oracle is pinned by physics with closed forms:
  (i)   free-field plane wave: the velocity-Verlet map of one lattice mode is x_n = A cos(n theta)
        with cos(theta) = 1 - (omega dt)^2 / 2 and omega^2 = sum_i (2/dx sin(pi n_i/N))^2;
  (ii)  time reversibility of VV2/VV4 and PV2/PV4 without expansion;
  (iii) energy error of VVn and PVn convergent as dt^n without expansion;
  (iv)  homogeneous lambda phi^4 with self-consistent expansion against scipy's solve_ivp of the
        background equations (velocityverlet.h, scalefactorkernels.h in the continuum-time limit).
"""
import math

import numpy as np
import pytest

from conftest import make_scalar_case
from oracle.oracle import OracleLattice


def run_oracle(rp, m, f, p, sf, n, measure=False):
    o = OracleLattice(m, rp)
    o.set_state(f, p, sf)
    o.initialize()
    o.sync()
    m0 = o.measure(1.0) if measure else None
    o.evolve(n)
    o.sync()
    m1 = o.measure(m0["energies"][-1]) if measure else None
    out = o.get_state()
    o.close()
    return out, m0, m1


@pytest.mark.parametrize("evolver", ["VV2", "LF"])
def test_free_plane_wave_closed_form(evolver):
    N, dt, nsteps = 16, 0.05, 40
    par, rp, m, f, p, sf = make_scalar_case(N=N, evolver=evolver, expansion=False, dt=dt, amp=0.0,
                                            extra={"lambda_prog": 0.0})
    nvec = (1, 2, 3)
    x = np.arange(N)
    X, Y, Z = np.meshgrid(x, x, x, indexing="ij")
    mode = np.cos(2 * np.pi * (nvec[0] * X + nvec[1] * Y + nvec[2] * Z) / N)
    A = 0.3
    f = (A * mode)[None]
    p = np.zeros_like(f)
    w2 = sum((2 / rp.dx * math.sin(math.pi * n / N)) ** 2 for n in nvec)
    (fo, po, _), _, _ = run_oracle(rp, m, f, p, {"aI": 1, "aSI": 1, "aIM": 1}, nsteps)
    if evolver == "VV2":
        theta = math.acos(1 - w2 * dt * dt / 2)
        expect = A * math.cos(nsteps * theta) * mode
    else:
        # leapfrog with the initial half kick (weight 0.5) is the same Stormer-Verlet map
        theta = math.acos(1 - w2 * dt * dt / 2)
        expect = A * math.cos(nsteps * theta) * mode
    assert np.abs(fo.reshape(N, N, N) - expect).max() < 1e-12


@pytest.mark.parametrize("evolver", ["VV2", "VV4", "PV2", "PV4"])
def test_time_reversibility(evolver):
    par, rp, m, f, p, sf = make_scalar_case(N=8, evolver=evolver, expansion=False, dt=0.02, amp=1e-2)
    (f1, p1, s1), _, _ = run_oracle(rp, m, f, p, sf, 30)
    import copy

    rp2 = copy.copy(rp)
    rp2.dt = -rp.dt
    (f2, p2, _), _, _ = run_oracle(rp2, m, f1, p1, s1, 30)
    assert np.abs(f2 - f.ravel()).max() < 1e-13
    assert np.abs(p2 - p.ravel()).max() < 1e-13


@pytest.mark.parametrize("evolver,order", [("VV2", 2), ("VV4", 4), ("VV6", 6), ("PV2", 2), ("PV4", 4), ("PV6", 6)])
def test_energy_error_order(evolver, order):
    errs = []
    for dt in (0.04, 0.02):
        n = int(round(0.8 / dt))
        par, rp, m, f, p, sf = make_scalar_case(N=8, evolver=evolver, expansion=False, dt=dt, amp=0.05, kcut=3)
        _, m0, m1 = run_oracle(rp, m, f, p, sf, n, measure=True)
        errs.append(m1["friedmann"][0])
    ratio = errs[0] / errs[1]
    assert ratio > 0.6 * 2 ** order, (errs, ratio)


def _background_error(evolver, dt, T=1.0):
    from scipy.integrate import solve_ivp

    par, rp, m, f, p, sf = make_scalar_case(N=4, evolver=evolver, expansion=True, dt=dt, amp=0.0)
    n = int(round(T / rp.dt))
    (fo, po, so), _, _ = run_oracle(rp, m, f, p, sf, n)
    al = m.alpha
    fm2 = (m.fStar / m.MPl) ** 2
    c0 = m.c0

    def rhs(t, y):
        phi, pi, a, ad = y
        V = 0.25 * c0 * phi ** 4
        Ek = 0.5 * pi * pi * a ** -6
        F = a ** (2 * al + 1) / 3.0 * fm2 * ((al - 2) * Ek + (al + 1) * V)
        return [a ** (al - 3) * pi, -a ** (3 + al) * c0 * phi ** 3, ad, F]

    # initial aDot as the oracle's Friedmann correction (modelinitializer.h:77-78)
    phi0, pi0, a0 = f.ravel()[0], p.ravel()[0], sf["aI"]
    rho = 0.5 * pi0 ** 2 * a0 ** -6 + 0.25 * c0 * phi0 ** 4
    ad0 = math.sqrt(a0 ** (2 * al + 2) / 3 * fm2 * rho)
    sol = solve_ivp(rhs, (0, T), [phi0, pi0, a0, ad0], rtol=1e-13, atol=1e-15, method="DOP853")
    phiT, piT, aT, adT = sol.y[:, -1]
    assert np.ptp(fo) == 0.0  # the lattice stays homogeneous
    return (abs(fo[0] - phiT), abs(po[0] - piT), abs(so["aI"] - aT) / aT, abs(so["aDotI"] - adT) / abs(adT))


def test_homogeneous_background_with_expansion_vv6():
    errs = _background_error("VV6", 0.004)
    assert max(errs) < 1e-11, errs


@pytest.mark.parametrize("evolver", ["VV2", "LF", "PV2"])
def test_homogeneous_background_second_order(evolver):
    e1 = _background_error(evolver, 0.004)[0]
    e2 = _background_error(evolver, 0.002)[0]
    assert 3.6 < e1 / e2 < 4.4, (e1, e2)


def test_reference_vv4_weights_are_reproduced():
    # velocityverletparameters.h:26 quotes w1 = -1.702414403875838200264, which differs from
    # Yoshida's -2^(1/3)/(2-2^(1/3)) = -1.7024143839193153 at the 8th digit, so a VV4 step advances
    # t by (1 - 2.0e-8) dt.  The drop-in keeps the reference's numbers: a homogeneous VV4 run lags the
    # exact background by a dt-independent amount.
    w0, w1 = 1.351207191959657771818, -1.702414403875838200264
    assert abs((2 * w0 + w1) - (1 - 1.9956522656628e-08)) < 1e-15
    e_a = _background_error("VV4", 0.004)[0]
    e_b = _background_error("VV4", 0.002)[0]
    assert 1e-8 < e_a < 2e-8 and abs(e_a - e_b) / e_a < 0.1


def test_fixed_background_run_parameters():
    # FixedBackgroundExpansion needs a non-zero H0 (fixedbackgroundexpansion.h:28-31); the initial
    # a = 1 and aDot = H0 / omega_* (scalefactorinitializer.h:37-43)
    from cosmolattice_b200.initializers import initial_scale_factor
    from cosmolattice_b200.params import RunParametersInconsistent

    with pytest.raises(RunParametersInconsistent):
        make_scalar_case(N=8, extra={"fixedBackground": "true"})
    par, rp, m, f, p, sf = make_scalar_case(N=8, extra={"fixedBackground": "true", "H0": 2.0e18, "omegaEoS": 0.0})
    assert rp.fixedBackground and rp.omegaEoS == 0.0
    assert initial_scale_factor(m, rp) == (1.0, 2.0e18 / m.omegaStar)


def test_fixed_background_oracle_scale_factor():
    # matter domination (w = 0, alpha = 1): p = 2, a = (1 + H0 t / 2)^2 exactly at t = n dt (PV2:
    # its one weight is 1; the reference's PV4/VV4 weights sum to 1 - 2e-8, so their last stage
    # ends 2e-8 dt short of t + dt, velocityverletparameters.h:26)
    par, rp, m, f, p, sf = make_scalar_case(N=6, evolver="PV2", dt=0.02,
                                            extra={"fixedBackground": "true", "H0": 0.3 * m_omega(), "omegaEoS": 0.0})
    (fo, po, so), _, _ = run_oracle(rp, m, f, p, sf, 25)
    t = 0.0
    for _ in range(25):
        t += 0.02
    assert abs(so["aI"] - (1 + 0.3 / 2 * t) ** 2) <= 1e-15 * so["aI"]
    assert abs(so["aDotI"] - 0.3 * (1 + 0.3 / 2 * t)) <= 1e-15 * so["aDotI"]


def m_omega():
    # omega_* of the lphi4_1f case: sqrt(lambda) phi_0 with lambda = 1
    return 5.6964e18
