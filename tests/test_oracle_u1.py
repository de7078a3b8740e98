"""Known-answer tests that pin the complex scalar + U(1) oracle (no GPU).

Closed-form properties of the lattice gauge theory the reference discretises:
  (i)   Gauss's law G(x) = sum_i (pi_i(x) - pi_i(x - i))/dx + dx rho(x) is preserved by every
        kick and drift (gausslaws.h:34-53 with the kernels of u1kernels.h and
        complexscalarkernels.h), so G after many steps equals G at the start to roundoff;
  (ii)  the RandomWithMatter initial state (u1initializer.h:77-117) solves Gauss's law for every
        non-zero mode: the residual is the (conserved) total charge, a constant;
  (iii) gauge covariance: phi -> e^{i theta} phi, A_i -> A_i + (theta(x+i) - theta(x))/(dx gQ)
        commutes with the evolution and leaves the energies unchanged;
  (iv)  without expansion the energy error of VV2 / VV4 converges as dt^2 / dt^4.
"""
import numpy as np
import pytest

from conftest import make_u1_case
from oracle.oracle import OracleLattice


def gauss_field(rp, m, f, p):
    N = rp.N
    f = f.reshape(5, N, N, N)
    p = p.reshape(5, N, N, N)
    lhs = sum(p[2 + i] - np.roll(p[2 + i], 1, axis=i) for i in range(3)) / rp.dx
    rho = 2.0 / rp.dx * (m.fStar / m.omegaStar) ** 2 * m.gQ * (p[0] * f[1] - p[1] * f[0])
    return lhs + rp.dx * rho, rp.dx * rho


def run(rp, m, f, p, sf, n, measure=False):
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


def test_initial_state_solves_gauss_law_up_to_total_charge():
    par, rp, m, f, p, sf = make_u1_case(N=12)
    G, r = gauss_field(rp, m, f.ravel(), p.ravel())
    # residual is uniform and equal to minus the mean charge term (the k = 0 mode cannot be solved)
    assert np.abs(G - G.mean()).max() < 1e-15 * np.abs(r).max() * 100
    assert abs(G.mean() - r.mean()) < 1e-16 + 1e-12 * abs(r.mean())
    assert np.abs(f[2:]).max() == 0.0


@pytest.mark.parametrize("evolver,expansion", [("VV2", True), ("VV4", False), ("LF", True)])
def test_gauss_law_preserved(evolver, expansion):
    par, rp, m, f, p, sf = make_u1_case(N=10, evolver=evolver, expansion=expansion, amp=5e-2)
    G0, r0 = gauss_field(rp, m, f.ravel(), p.ravel())
    (f1, p1, _), _, _ = run(rp, m, f, p, sf, 40)
    G1, r1 = gauss_field(rp, m, f1, p1)
    assert np.abs(r1 - r0).max() > 1e-6 * np.abs(r0).max()  # the charge density did move
    assert np.abs(G1 - G0).max() < 1e-12 * np.abs(r0).max()


def test_gauge_covariance():
    par, rp, m, f, p, sf = make_u1_case(N=8, evolver="VV2", expansion=True, amp=5e-2)
    N = rp.N
    rng = np.random.default_rng(3)
    th = rng.uniform(-np.pi, np.pi, (N, N, N))
    f = f.copy()
    f[2:] = rng.normal(0, 0.05, (3, N, N, N))  # non-trivial links
    p = p.copy()

    def transform(f, p):
        f, p = f.reshape(5, N, N, N).copy(), p.reshape(5, N, N, N).copy()
        z, w = f[0] + 1j * f[1], p[0] + 1j * p[1]
        z, w = np.exp(1j * th) * z, np.exp(1j * th) * w
        f[0], f[1], p[0], p[1] = z.real, z.imag, w.real, w.imag
        for i in range(3):
            f[2 + i] += (np.roll(th, -1, axis=i) - th) / (rp.dx * m.gQ)
        return f, p

    (fa, pa, sa), ma0, ma1 = run(rp, m, f, p, sf, 20, measure=True)
    ft, pt = transform(f, p)
    (fb, pb, sb), mb0, mb1 = run(rp, m, ft, pt, sf, 20, measure=True)
    assert np.allclose(ma0["energies"], mb0["energies"], rtol=1e-10, atol=0)
    assert np.allclose(ma1["energies"], mb1["energies"], rtol=1e-9, atol=1e-18)
    assert abs(sa["aI"] - sb["aI"]) < 1e-12
    fa_t, pa_t = transform(fa, pa)
    fb, pb = fb.reshape(5, N, N, N), pb.reshape(5, N, N, N)
    scale = np.abs(fb[:2]).max()
    assert np.abs(fa_t[:2] - fb[:2]).max() < 1e-10 * scale
    # links agree modulo 2 pi / (dx gQ)
    period = 2 * np.pi / (rp.dx * m.gQ)
    dA = (fa_t[2:] - fb[2:]) / period
    assert np.abs(dA - np.round(dA)).max() * period < 1e-9


@pytest.mark.parametrize("evolver,order", [("VV2", 2), ("VV4", 4)])
def test_energy_error_order(evolver, order):
    errs = []
    for dt in (0.04, 0.02):
        n = int(round(0.8 / dt))
        par, rp, m, f, p, sf = make_u1_case(N=8, evolver=evolver, expansion=False, dt=dt, amp=0.1, kcut=3)
        _, m0, m1 = run(rp, m, f, p, sf, n, measure=True)
        errs.append(m1["friedmann"][0])
    ratio = errs[0] / errs[1]
    assert 2 ** order * 0.7 < ratio < 2 ** order * 1.4, (errs, ratio)
