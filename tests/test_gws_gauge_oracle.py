"""The oracle's GW source for the gauge models (PITensor.h) against a numpy restatement.

One step from u = pi_u = 0 right after initialize kicks the GW momenta by (dt/2) a^(1+alpha) 2 Pi:
the Laplacian of u = 0 vanishes and the first GW kick after a sync has weight 1/2 (evolver.h:104-107).
So pi_u after one evolve step is that product, with Pi the traceless part of the anisotropic tensor
of the start state, and u = pow(a_SI, alpha - 3) dt pi_u after the step's GW drift.  numpy forms Pi
on its own: 2 Re[D_i phi conj(D_j phi)] from the forward covariant differences of the complex
scalar, -1/a^2/(fStar/omegaStar)^2 pi_A,i pi_A,j (electric), the same of (curl A)_i (curl A)_j
(magnetic), and for lphi4SU2U1 the singlet's forwDiff_i S forwDiff_j S.  The SU(2) doublet and the
SU(2) field source no GWs.  Bound: 1e-12 of the largest component.
"""
import numpy as np
import pytest

from conftest import make_su2_case, make_u1_case

PAIRS = [(0, 0), (0, 1), (0, 2), (1, 1), (1, 2), (2, 2)]


def _fwd(f, i):
    return np.roll(f, -1, axis=i)  # f(x + i), axes (x, y, z)


def _tensor(phr, phi, A, pA, dx, g, aI, rfo2, S=None):
    ph = phr + 1j * phi
    D = []
    for i in range(3):
        th = (-dx * g) * A[i]
        w = (np.cos(th) + 1j * np.sin(th)) * (_fwd(phr, i) + 1j * _fwd(phi, i))
        D.append((w - ph) / dx)

    def fd(f, i):
        return (_fwd(f, i) - f) / dx

    B = [fd(A[2], 1) - fd(A[1], 2), fd(A[0], 2) - fd(A[2], 0), fd(A[1], 0) - fd(A[0], 1)]
    pref = (-1.0 / aI ** 2) / rfo2
    T = []
    for i, j in PAIRS:
        t = 2 * np.real(D[i] * np.conj(D[j])) + pref * pA[i] * pA[j] + pref * B[i] * B[j]
        if S is not None:
            t = t + fd(S, i) * fd(S, j)
        T.append(t)
    tr = (T[0] + T[3] + T[5]) / 3
    return np.stack([T[0] - tr, T[1], T[2], T[3] - tr, T[4]])


@pytest.mark.parametrize("model", ["lphi4U1", "lphi4SU2U1"])
def test_oracle_gauge_gw_source_matches_numpy(model):
    from oracle.oracle import OracleLattice

    rng = np.random.default_rng(5)
    if model == "lphi4U1":
        par, rp, m, f, p, sf = make_u1_case(N=8, amp=3e-2)
        f = f.reshape(5, -1).copy()
        f[2:5] = 1e-2 * rng.standard_normal(f[2:5].shape)  # A != 0, so B enters
        comps = {"phi": (0, 1), "A": (2, 3, 4), "S": None, "g": m.desc().couplings[1]}
    else:
        par, rp, m, f, p, sf = make_su2_case(N=8, amp=3e-2)
        f = f.reshape(22, -1).copy()
        f[0] += 1e-2 * rng.standard_normal(f[0].shape)
        f[1:3] += 1e-2 * rng.standard_normal(f[1:3].shape)
        f[7:10] = 1e-2 * rng.standard_normal(f[7:10].shape)
        comps = {"phi": (1, 2), "A": (7, 8, 9), "S": 0, "g": m.desc().couplings[2]}
    N = rp.N
    o = OracleLattice(m, rp)
    o.gws_enable()
    o.set_state(f.ravel(), p, sf)
    o.initialize()
    f0, p0, s0 = o.get_state()
    o.evolve(1)
    u, pi = o.gws_get_state()
    s1 = o.get_state()[2]
    o.close()
    F = f0.reshape(-1, N, N, N)
    P = p0.reshape(-1, N, N, N)
    A = [F[c] for c in comps["A"]]
    pA = [P[c] for c in comps["A"]]
    S = F[comps["S"]] if comps["S"] is not None else None
    Pi = _tensor(F[comps["phi"][0]], F[comps["phi"][1]], A, pA, rp.dx, comps["g"], s0["aI"],
                 (m.fStar / m.omegaStar) ** 2, S)
    want = 0.5 * rp.dt * s0["aI"] ** (1 + m.alpha) * 2 * Pi
    got = pi.reshape(5, N, N, N)
    scale = np.abs(want).max()
    assert scale > 0
    assert np.abs(got - want).max() <= 1e-12 * scale
    assert np.allclose(u.reshape(5, N, N, N), s1["aSI"] ** (m.alpha - 3) * rp.dt * got, rtol=1e-14, atol=0)
    # the electric and the magnetic parts both enter at this state
    zero = [0 * a for a in A]
    no_e = _tensor(F[comps["phi"][0]], F[comps["phi"][1]], A, zero, rp.dx, comps["g"], s0["aI"],
                   (m.fStar / m.omegaStar) ** 2, S)
    pref = (-1.0 / s0["aI"] ** 2) / (m.fStar / m.omegaStar) ** 2
    curl = [(_fwd(A[2], 1) - A[2]) - (_fwd(A[1], 2) - A[1]), (_fwd(A[0], 2) - A[0]) - (_fwd(A[2], 0) - A[2]),
            (_fwd(A[1], 0) - A[1]) - (_fwd(A[0], 1) - A[0])]
    mag = pref * (curl[0] / rp.dx) ** 2
    assert np.abs(Pi - no_e).max() > 1e-6 * np.abs(Pi).max()
    assert np.abs(mag).max() > 1e-6 * np.abs(Pi).max()
