"""The oracle of the device initial-condition generator (oracle/ic_recipe.py), on the CPU.

* Its Philox4x64-10 against numpy's independent implementation (np.random.Philox, whose first
  block is the one of counter + 1) and the published all-zero known-answer vector.
* Hermitian kz = 0 and N/2 planes: rfftn(irfftn(modes)) returns the modes.
* The gauge momenta satisfy the discrete Gauss laws with A = 0 and unit links
  (u1initializer.h:90-114): sum_i (pi_i(x) - pi_i(x - i)) = -dx^2 rho.
* device_ic_params fills the matter components in each model's field order.
"""
import math

import numpy as np
import pytest

from oracle import ic_recipe as icr


def test_philox_matches_numpy_bit_generator():
    rng = np.random.default_rng(3)
    for _ in range(5):
        k0, k1 = (int(x) for x in rng.integers(0, 2 ** 63, size=2, dtype=np.uint64))
        c0 = int(rng.integers(0, 2 ** 40))
        bg = np.random.Philox(key=np.array([k0, k1], dtype=np.uint64), counter=np.array([c0, 0, 0, 0], dtype=np.uint64))
        raw = bg.random_raw(4 * 6)
        w = icr.philox4x64(np.arange(c0 + 1, c0 + 7, dtype=np.uint64), k0, k1)
        for i in range(6):
            for j in range(4):
                assert int(w[j][i]) == int(raw[4 * i + j])


def test_philox_known_answer():
    w = icr.philox4x64(np.zeros(1, dtype=np.uint64), 0, 0)
    assert [int(x[0]) for x in w] == [0x16554D9ECA36314C, 0xDB20FE9D672D0FDC, 0xD7E772CEE186176B, 0x7E68B68AEC7BA23B]


def test_uniform_range():
    u = icr.uniform(np.array([0, (1 << 64) - 1], dtype=np.uint64))
    assert u[0] == 0.0 and u[1] == 1.0 - 2.0 ** -53


@pytest.mark.parametrize("N", [8, 9, 12])
def test_modes_are_hermitian(N):
    g = icr.ModeGrid(N)
    dx = 2 * np.pi / N
    A = 1e-2 * (N * dx / dx ** 2) ** 1.5 / math.sqrt(2.0)
    for fk in icr.singlet_modes(g, 7, 0, 1.0, A, 1e9, 3.0, 0.2) + tuple(
            x for pair in icr.complex_modes(g, 7, 1.0, A, 1e9, [1.0, 2.0], 0.2) for x in pair):
        back = np.fft.rfftn(icr.to_space(fk, N), axes=(0, 1, 2))
        assert np.max(np.abs(back - fk)) <= 1e-12 * np.max(np.abs(fk))
        assert fk[0, 0, 0] == 0


def _params(nm, charge):
    return {"seed": 11, "amplitude": 1e-2, "k_cutoff": 3.0, "adot": 0.25, "mass2": [3.0, 1.0, 2.0, 0.5, 0.7, 0.9, 1.1][:nm],
            "fld0": [0.9, 0.1, -0.2, 0.3, 0.1, 0.2, -0.1][:nm], "pi0": [0.01, 0.02, 0.0, -0.01, 0.0, 0.03, 0.0][:nm],
            "charge": charge}


def _div_back(P, comps):
    return sum(P[c] - np.roll(P[c], 1, axis=i) for i, c in enumerate(comps))


def test_u1_gauss_law():
    N, dx, r2, g = 12, 2 * np.pi / 12, 2.0, 0.5
    F, P = icr.generate_state(icr.MODEL_LPHI4U1, N, dx, r2, _params(2, [g, 0, 0, 0]))
    rho = 2.0 / dx * r2 * g * (P[0] * F[1] - P[1] * F[0])
    lhs = _div_back(P, [2, 3, 4])
    assert np.max(np.abs(lhs + dx * dx * (rho - rho.mean()))) <= 1e-12 * np.max(np.abs(lhs))
    assert np.all(F[2:] == 0)


def test_su2u1_gauss_laws():
    N, dx, r2 = 8, 2 * np.pi / 8, 2.0
    gS, gC, gD = 0.6, 0.35, 0.2
    F, P = icr.generate_state(icr.MODEL_LPHI4SU2U1, N, dx, r2, _params(7, [gS, gC, gD, 0]))
    u, v = F[3] + 1j * F[4], F[5] + 1j * F[6]
    pu, pv = P[3] + 1j * P[4], P[5] + 1j * P[6]
    rho = 2.0 / dx * r2 * (gC * (P[1] * F[2] - P[2] * F[1]) + gD * np.imag(np.conj(pu) * u + np.conj(pv) * v))
    lhs = _div_back(P, [7, 8, 9])
    assert np.max(np.abs(lhs + dx * dx * (rho - rho.mean()))) <= 1e-12 * np.max(np.abs(lhs))
    isig = [(1j * v, 1j * u), (v, -u), (1j * u, -1j * v)]
    for b in range(3):
        a, c = isig[b]
        rb = r2 / 2 * gS * np.real(np.conj(a) * pu + np.conj(c) * pv) / dx
        lhs = _div_back(P, [10 + b, 13 + b, 16 + b])
        assert np.max(np.abs(lhs + dx * dx * (rb - rb.mean()))) <= 1e-12 * np.max(np.abs(lhs))
    for i in range(3):
        assert np.all(F[10 + 4 * i] == 1.0) and np.all(F[11 + 4 * i: 14 + 4 * i] == 0.0)


def test_singlet_mode_variance():
    # <|phi_k|^2> = norm_k^2 (left and right movers each of variance 2 norm^2 in |.|^2, halved by the 1/sqrt2)
    N = 24
    g = icr.ModeGrid(N)
    dx = 2 * np.pi / N
    A = 1e-2 * (N * dx / dx ** 2) ** 1.5 / math.sqrt(2.0)
    phi, _ = icr.singlet_modes(g, 5, 0, 1.0, A, 1e9, 3.0, 0.0)
    norm, _ = icr._norm(g, 1.0, A, 1e9, 3.0)
    sel = ~(g.zero | g.conj | g.real) & (g.nz > 0)
    ratio = np.mean(np.abs(phi[sel]) ** 2 / norm[sel] ** 2)
    assert abs(ratio - 2.0) < 0.05


def test_device_ic_params_component_order():
    from conftest import make_scalar_case, make_su2_case, make_u1_case
    from cosmolattice_b200.initializers import device_ic_params

    _, rp, m, *_ = make_scalar_case(N=8, model="lphi4")
    p, aI, aD = device_ic_params(m, rp, seed=1)
    assert len(p["mass2"]) == 2 and p["fld0"][0] == m.fldS0[0] / m.fStar and p["charge"] == [0.0] * 4
    _, rp, m, *_ = make_u1_case(N=8)
    p, aI, aD = device_ic_params(m, rp)
    assert len(p["mass2"]) == 2 and p["charge"][0] == m.gQ and 0 <= p["seed"] < 2 ** 64
    _, rp, m, *_ = make_su2_case(N=8)
    p, aI, aD = device_ic_params(m, rp, seed=2)
    assert len(p["mass2"]) == 7 and p["mass2"][3:] == list(m.masses2D[:4])
    assert p["charge"][:3] == [m.gQ_S, m.gQ_C, m.gQ_D] and p["amplitude"] == m.fluct_amplitude
