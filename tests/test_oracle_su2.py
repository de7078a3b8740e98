"""Known-answer tests that pin the lphi4SU2U1 oracle (no GPU).

TempLat's SU(2) types are not part of the reference tree, so the link, algebra, plaquette and
exponential conventions are stated choices (oracle_su2.cpp header).  These tests show that with
them the reference's normalisations give a consistent lattice gauge theory:
  (i)   energy error of VV2 / VV4 converges as dt^2 / dt^4 without expansion;
  (ii)  both Gauss laws (gausslaws.h:34-80) are preserved per site by every step, with and
        without expansion (the residual at t = 0 is the k = 0 charge, which stays constant);
  (iii) a random SU(2) x U(1) gauge transformation commutes with the evolution and leaves every
        energy component unchanged;
  (iv)  links stay unit quaternions.
"""
import numpy as np
import pytest

from conftest import make_su2_case
from oracle.oracle import OracleLattice


def qmul(a, b):
    a0, a1, a2, a3 = a
    b0, b1, b2, b3 = b
    return np.array([a0 * b0 - (a1 * b1 + a2 * b2 + a3 * b3),
                     a0 * b1 + b0 * a1 - (a2 * b3 - a3 * b2),
                     a0 * b2 + b0 * a2 - (a3 * b1 - a1 * b3),
                     a0 * b3 + b0 * a3 - (a1 * b2 - a2 * b1)])


def qdag(a):
    return np.array([a[0], -a[1], -a[2], -a[3]])


def qapply(q, u, v):
    return (q[0] + 1j * q[3]) * u + (q[2] + 1j * q[1]) * v, (-q[2] + 1j * q[1]) * u + (q[0] - 1j * q[3]) * v


def gauss_fields(rp, m, f, p):
    N = rp.N
    f = f.reshape(22, N, N, N)
    p = p.reshape(19, N, N, N)
    dx = rp.dx
    r2 = (m.fStar / m.omegaStar) ** 2
    u, v = f[3] + 1j * f[4], f[5] + 1j * f[6]
    pu, pv = p[3] + 1j * p[4], p[5] + 1j * p[6]
    # U(1)
    lhs = sum(p[7 + i] - np.roll(p[7 + i], 1, axis=i) for i in range(3)) / dx
    rho = 2 / dx * r2 * (m.gQ_C * (p[1] * f[2] - p[2] * f[1]) + m.gQ_D * np.imag(np.conj(pu) * u + np.conj(pv) * v))
    gu1 = lhs + dx * rho
    # SU(2)
    isig = [(1j * v, 1j * u), (v, -u), (1j * u, -1j * v)]
    gsu2 = []
    for b in range(3):
        L = 0
        for i in range(3):
            U = np.roll(f[10 + 4 * i:14 + 4 * i], 1, axis=i + 1)
            pim = np.roll(p[10 + 3 * i:13 + 3 * i], 1, axis=i + 1)
            r = qmul(qmul(qdag(U), np.concatenate([np.zeros((1,) + pim.shape[1:]), pim])), U)
            L = L + (p[10 + 3 * i + b] - r[1 + b]) / dx
        a, c = isig[b]
        R = -(r2 / 2 * (m.gQ_S * np.real(np.conj(a) * pu + np.conj(c) * pv)))
        gsu2.append(L - R)
    return gu1, np.array(gsu2), rho


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


@pytest.mark.parametrize("evolver,order", [("VV2", 2), ("VV4", 4)])
def test_energy_error_order(evolver, order):
    errs = []
    for dt in (0.008, 0.004):
        par, rp, m, f, p, sf = make_su2_case(N=6, evolver=evolver, expansion=False, dt=dt, amp=0.05, kcut=2)
        _, m0, m1 = run(rp, m, f, p, sf, int(round(0.16 / dt)), measure=True)
        errs.append(m1["friedmann"][0])
    ratio = errs[0] / errs[1]
    assert 2 ** order * 0.7 < ratio < 2 ** order * 1.4, (errs, ratio)


@pytest.mark.parametrize("evolver,expansion", [("VV2", True), ("VV4", False), ("LF", True)])
def test_gauss_laws_preserved(evolver, expansion):
    par, rp, m, f, p, sf = make_su2_case(N=6, evolver=evolver, expansion=expansion, amp=0.05)
    rng = np.random.default_rng(2)
    f = f.copy()
    f[7:10] = rng.normal(0, 0.3, f[7:10].shape)  # non-trivial U(1) links
    g1a, g2a, rho = gauss_fields(rp, m, f.ravel(), p.ravel())
    # the initial state solves both laws for every non-zero mode
    assert np.abs(g2a - g2a.mean(axis=(1, 2, 3), keepdims=True)).max() < 1e-12 * np.abs(p[10:]).max() / rp.dx
    (f1, p1, _), _, _ = run(rp, m, f, p, sf, 30)
    g1b, g2b, rho1 = gauss_fields(rp, m, f1, p1)
    assert np.abs(rho1 - rho).max() > 1e-6 * np.abs(rho).max()
    assert np.abs(g1b - g1a).max() < 1e-12 * np.abs(rho).max() * rp.dx
    assert np.abs(g2b - g2a).max() < 1e-11 * np.abs(g2a).max() + 1e-14


def test_gauge_covariance_and_unit_links():
    par, rp, m, f, p, sf = make_su2_case(N=6, evolver="VV2", expansion=True, amp=0.05)
    N = rp.N
    rng = np.random.default_rng(7)
    f = f.copy()
    # random non-trivial SU(2) links and U(1) field
    for i in range(3):
        q = rng.normal(0, 0.2, (4, N, N, N))
        q[0] += 1
        f[10 + 4 * i:14 + 4 * i] = q / np.sqrt((q * q).sum(axis=0))
    f[7:10] = rng.normal(0, 0.3, (3, N, N, N))
    G = rng.normal(0, 1, (4, N, N, N))
    G /= np.sqrt((G * G).sum(axis=0))
    chi = rng.uniform(-1, 1, (N, N, N))

    def transform(f, p):
        f, p = f.reshape(22, N, N, N).copy(), p.reshape(19, N, N, N).copy()
        for arr, base in ((f, 3), (p, 3)):
            u, v = qapply(G, arr[base] + 1j * arr[base + 1], arr[base + 2] + 1j * arr[base + 3])
            ph = np.exp(1j * m.gQ_D * chi)
            u, v = ph * u, ph * v
            arr[base], arr[base + 1], arr[base + 2], arr[base + 3] = u.real, u.imag, v.real, v.imag
        for arr in (f, p):
            z = np.exp(1j * m.gQ_C * chi) * (arr[1] + 1j * arr[2])
            arr[1], arr[2] = z.real, z.imag
        for i in range(3):
            f[7 + i] += (np.roll(chi, -1, axis=i) - chi) / rp.dx
            Gp = np.roll(G, -1, axis=i + 1)
            f[10 + 4 * i:14 + 4 * i] = qmul(qmul(G, f[10 + 4 * i:14 + 4 * i]), qdag(Gp))
            pq = np.concatenate([np.zeros((1, N, N, N)), p[10 + 3 * i:13 + 3 * i]])
            p[10 + 3 * i:13 + 3 * i] = qmul(qmul(G, pq), qdag(G))[1:]
        return f, p

    (fa, pa, sa), ma0, ma1 = run(rp, m, f, p, sf, 15, measure=True)
    ft, pt = transform(f, p)
    (fb, pb, sb), mb0, mb1 = run(rp, m, ft, pt, sf, 15, measure=True)
    assert np.allclose(ma0["energies"], mb0["energies"], rtol=1e-9, atol=1e-15)
    assert np.allclose(ma1["energies"], mb1["energies"], rtol=1e-8, atol=1e-14)
    assert abs(sa["aI"] - sb["aI"]) < 1e-12
    fa_t, pa_t = transform(fa, pa)
    fb = fb.reshape(22, N, N, N)
    # gauge-covariant fields agree; U(1) links agree modulo 2 pi / (dx g) of each charge
    assert np.abs(fa_t[0] - fb[0]).max() < 1e-10
    assert np.abs(fa_t[1:7] - fb[1:7]).max() < 1e-10
    assert np.abs(fa_t[10:] - fb[10:]).max() < 1e-10
    for i in range(3):
        U = fb[10 + 4 * i:14 + 4 * i]
        assert np.abs((U * U).sum(axis=0) - 1).max() < 1e-13
