"""Test infrastructure (the oracle): CPU restatement of the device initial-condition generator
behind clb_generate_state.  Only tests import it; nothing in the package calls it.

The physics follows the reference's initializers:
* singlets: FluctuationsGenerator::getFluctuationsNorm / conjugateGaussianFluctuations
  (initializers/fluctuationsgenerator.h:39-71, 130-150);
* complex scalar: U1Initializer::addFluctuationsCScalarFromPhases (initializers/u1initializer.h:157-230);
* SU(2) doublet: SU2Initializer::addFluctuationsSU2DoubletFromPhases
  (initializers/su2initializer.h:115-186);
* gauge momenta from the Gauss laws with A = 0 and unit links (u1initializer.h:90-114,
  su2initializer.h:65-85);
* homogeneous parts added afterwards (scalarsingletinitializer.h:41-77).

The random numbers are this library's own: Philox4x64-10 (Salmon, Moraes, Dror, Shaw, "Parallel
random numbers: as easy as 1, 2, 3", SC11), key (seed, stream), counter (mode index, 0, 0, 0),
one block of four 64-bit words per mode and stream; u = (word >> 11) 2^-53.  The reference's
TempLat streams cannot be reproduced outside TempLat.  Streams: singlet i: 1 + i (Gaussian left
mover from words 0, 1, right mover from words 2, 3, Box-Muller); complex scalar: 16 (phases
e00, e01, e10, Rayleigh amplitude 0), 17 (Rayleigh amplitude 1); doublet: 32 (Rayleigh
amplitudes 0-3), 33 (left phases 0-3), 34 (right phase 0).

The kz = 0 and (even N) kz = N/2 planes are made Hermitian: a mode whose partner (-kx, -ky) has a
smaller index takes the conjugate of the partner's values, a self-conjugate mode keeps the real
part.  The configuration-space field is then the real inverse transform of the drawn modes
(normalised 1/N^3).
"""
from __future__ import annotations

import math

import numpy as np
import scipy.fft as sfft

MASK = (1 << 64) - 1
PHILOX_M0, PHILOX_M1 = 0xD2E7470EE14C6C93, 0xCA5A826395121157
PHILOX_W0, PHILOX_W1 = 0x9E3779B97F4A7C15, 0xBB67AE8584CAA73B

STREAM_SINGLET, STREAM_COMPLEX, STREAM_DOUBLET = 1, 16, 32
MODEL_LPHI4, MODEL_LPHI4U1, MODEL_LPHI4SU2U1 = 1, 2, 3


def _mulhilo(m: int, b: np.ndarray):
    """(high, low) 64-bit words of the 128-bit product m * b (b uint64 array), in 32-bit limbs."""
    b = b.astype(np.uint64, copy=False)
    m_lo, m_hi = np.uint64(m & 0xFFFFFFFF), np.uint64(m >> 32)
    b_lo, b_hi = b & np.uint64(0xFFFFFFFF), b >> np.uint64(32)
    t = m_lo * b_lo
    u = m_hi * b_lo + (t >> np.uint64(32))
    w = m_lo * b_hi + (u & np.uint64(0xFFFFFFFF))
    hi = m_hi * b_hi + (u >> np.uint64(32)) + (w >> np.uint64(32))
    lo = b * np.uint64(m)
    return hi, lo


def philox4x64(ctr0: np.ndarray, key0: int, key1: int, ctr1=None, ctr2=None, ctr3=None):
    """Philox4x64-10 of counters (ctr0, ctr1, ctr2, ctr3) (missing words 0) under key (key0, key1)."""
    with np.errstate(over="ignore"):
        c0 = np.asarray(ctr0, dtype=np.uint64)
        z = np.zeros_like(c0)
        c1 = z if ctr1 is None else np.asarray(ctr1, dtype=np.uint64) + z
        c2 = z if ctr2 is None else np.asarray(ctr2, dtype=np.uint64) + z
        c3 = z if ctr3 is None else np.asarray(ctr3, dtype=np.uint64) + z
        k0, k1 = key0 & MASK, key1 & MASK
        for _ in range(10):
            hi0, lo0 = _mulhilo(PHILOX_M0, c0)
            hi1, lo1 = _mulhilo(PHILOX_M1, c2)
            c0, c1, c2, c3 = hi1 ^ c1 ^ np.uint64(k0), lo1, hi0 ^ c3 ^ np.uint64(k1), lo0
            k0, k1 = (k0 + PHILOX_W0) & MASK, (k1 + PHILOX_W1) & MASK
    return c0, c1, c2, c3


def uniform(words: np.ndarray) -> np.ndarray:
    """Uniform doubles in [0, 1) from the top 53 bits of 64-bit words."""
    return (words >> np.uint64(11)).astype(np.float64) * 2.0 ** -53


def _cis(u):
    return np.cos(2 * np.pi * u) + 1j * np.sin(2 * np.pi * u)


def _rayleigh(u):
    return np.sqrt(-2.0 * np.log1p(-u))


class ModeGrid:
    """Half spectrum (N, N, N//2+1): signed wave numbers, canonical draw indices and the
    Hermitian-plane bookkeeping."""

    def __init__(self, N: int):
        self.N = N
        nzh = N // 2 + 1
        kx, ky, kz = np.meshgrid(np.arange(N), np.arange(N), np.arange(nzh), indexing="ij")
        self.nx = np.where(kx <= N // 2, kx, kx - N)
        self.ny = np.where(ky <= N // 2, ky, ky - N)
        self.nz = kz
        self.n2 = self.nx * self.nx + self.ny * self.ny + self.nz * self.nz
        idx = (kx * N + ky) * nzh + kz
        herm = (kz == 0) | ((N % 2 == 0) & (kz == N // 2))
        pidx = (((N - kx) % N) * N + (N - ky) % N) * nzh + kz
        self.canon = np.where(herm, np.minimum(idx, pidx), idx).astype(np.uint64)
        self.conj = herm & (idx > pidx)
        self.real = herm & (idx == pidx)
        self.zero = self.n2 == 0

    def finish(self, v: np.ndarray) -> np.ndarray:
        v = np.where(self.conj, np.conj(v), v)
        v = np.where(self.real, v.real + 0j, v)
        return np.where(self.zero, 0j, v)


def _norm(g: ModeGrid, kIR: float, A: float, kcut: float, m2: float):
    """H(kcut - k) A / sqrt(2 omega), omega = sqrt(k^2 + max(m2, 0)) (fluctuationsgenerator.h:39-65)."""
    k = np.sqrt(g.n2.astype(np.float64)) * kIR
    omega = np.sqrt(k * k + (m2 if m2 > 0 else 0.0))
    with np.errstate(divide="ignore"):
        norm = np.where((k <= kcut) & ~g.zero, A / np.sqrt(2.0 * omega), 0.0)
    return norm, omega


def singlet_modes(g: ModeGrid, seed: int, i: int, kIR, A, kcut, m2, adot):
    """(phi_k, pi_k) of singlet i: phi = (fL + fR)/sqrt2, pi = i omega (fL - fR)/sqrt2 - aDot phi
    (fluctuationsgenerator.h:130-150)."""
    w = philox4x64(g.canon, seed, STREAM_SINGLET + i)
    u = [uniform(x) for x in w]
    norm, omega = _norm(g, kIR, A, kcut, m2)
    fL = norm * _rayleigh(u[0]) * _cis(u[1])
    fR = norm * _rayleigh(u[2]) * _cis(u[3])
    phi = (fL + fR) / math.sqrt(2.0)
    pi = 1j * omega * (fL - fR) / math.sqrt(2.0) - adot * phi
    return g.finish(phi), g.finish(pi)


def complex_modes(g: ModeGrid, seed: int, kIR, A, kcut, m2, adot):
    """[(phi_c, pi_c)] of the complex scalar's two real components (u1initializer.h:157-230):
    a_c Rayleigh, e11 = e01 e10 conj(e00), phi_c = a_c (e_c0 + e_c1)/2,
    pi_c = -i omega_0 a_c (e_c0 - e_c1)/2 - aDot phi_c."""
    w16 = [uniform(x) for x in philox4x64(g.canon, seed, STREAM_COMPLEX)]
    w17 = [uniform(x) for x in philox4x64(g.canon, seed, STREAM_COMPLEX + 1)]
    e00, e01, e10 = _cis(w16[0]), _cis(w16[1]), _cis(w16[2])
    e11 = e01 * e10 * np.conj(e00)
    ray = [_rayleigh(w16[3]), _rayleigh(w17[0])]
    omega0 = _norm(g, kIR, A, kcut, m2[0])[1]
    out = []
    for c, (ea, eb) in enumerate(((e00, e01), (e10, e11))):
        a = _norm(g, kIR, A, kcut, m2[c])[0] * ray[c]
        f = a * (ea + eb) / 2.0
        p = -1j * omega0 * a * (ea - eb) / 2.0 - adot * f
        out.append((g.finish(f), g.finish(p)))
    return out


def doublet_modes(g: ModeGrid, seed: int, kIR, A, kcut, m2, adot):
    """[(Phi_c, pi_c)] of the doublet's four real components (su2initializer.h:115-186): a_c
    Rayleigh, left phases l_c, r_c = r_0 l_c conj(l_0), Phi_c = a_c (l_c + r_c)/2,
    pi_c = -i omega_0 a_c (l_c - r_c)/2 - aDot Phi_c / sqrt2."""
    ray = [_rayleigh(uniform(x)) for x in philox4x64(g.canon, seed, STREAM_DOUBLET)]
    left = [_cis(uniform(x)) for x in philox4x64(g.canon, seed, STREAM_DOUBLET + 1)]
    r0 = _cis(uniform(philox4x64(g.canon, seed, STREAM_DOUBLET + 2)[0]))
    omega0 = _norm(g, kIR, A, kcut, m2[0])[1]
    out = []
    for c in range(4):
        a = _norm(g, kIR, A, kcut, m2[c])[0] * ray[c]
        r = r0 * left[c] * np.conj(left[0])
        f = a * (left[c] + r) / 2.0
        p = -1j * omega0 * a * (left[c] - r) / 2.0 - adot * f / math.sqrt(2.0)
        out.append((g.finish(f), g.finish(p)))
    return out


def to_space(modes: np.ndarray, N: int) -> np.ndarray:
    return sfft.irfftn(modes, s=(N, N, N), axes=(0, 1, 2))


def gauss_solve(g: ModeGrid, dx: float, rho: np.ndarray):
    """pi_i = IFFT(conj(q_i) / sum_j |q_j|^2 FFT(-dx^2 rho)), q_j = 1 - exp(-2 pi i n_j / N), zero
    mode 0: sum_i (pi_i(x) - pi_i(x - i)) = -dx^2 rho (u1initializer.h:90-114)."""
    N = g.N
    j0 = sfft.rfftn(-dx * dx * rho, axes=(0, 1, 2))
    q = [1.0 - np.exp(-2j * np.pi * n / N) for n in (g.nx, g.ny, g.nz)]
    k2 = sum(np.abs(x) ** 2 for x in q)
    k2 = np.where(g.zero, 1.0, k2)
    return [to_space(np.where(g.zero, 0j, np.conj(x) / k2 * j0), N) for x in q]


def generate_state(kind: int, N: int, dx: float, r2: float, p: dict, n_scalars: int = 1):
    """(fields, momenta) of clb_generate_state for model kind (1 lphi4, 2 lphi4U1, 3 lphi4SU2U1).
    p: seed, amplitude, k_cutoff, adot, mass2, fld0, pi0 (matter components in the model's field
    order), charge; r2 = (fStar / omegaStar)^2."""
    g = ModeGrid(N)
    L = N * dx
    kIR = 2 * np.pi / L
    A = p["amplitude"] * (L / dx ** 2) ** 1.5 / math.sqrt(2.0)
    seed, kc, ad = int(p["seed"]), p["k_cutoff"], p["adot"]
    m2, f0, q0, ch = list(p["mass2"]), list(p["fld0"]), list(p["pi0"]), list(p["charge"])
    shape = (N, N, N)
    if kind == MODEL_LPHI4:
        F = np.zeros((n_scalars,) + shape)
        P = np.zeros_like(F)
        for i in range(n_scalars):
            fk, pk = singlet_modes(g, seed, i, kIR, A, kc, m2[i], ad)
            F[i] = to_space(fk, N) + f0[i]
            P[i] = to_space(pk, N) + q0[i]
        return F, P
    if kind == MODEL_LPHI4U1:
        F = np.zeros((5,) + shape)
        P = np.zeros_like(F)
        for c, (fk, pk) in enumerate(complex_modes(g, seed, kIR, A, kc, m2[0:2], ad)):
            F[c] = to_space(fk, N) + f0[c]
            P[c] = to_space(pk, N) + q0[c]
        rho = 2.0 / dx * r2 * ch[0] * (P[0] * F[1] - P[1] * F[0])  # mattercurrents.h:27-48
        for i, x in enumerate(gauss_solve(g, dx, rho)):
            P[2 + i] = x
        return F, P
    if kind == MODEL_LPHI4SU2U1:
        F = np.zeros((22,) + shape)
        P = np.zeros((19,) + shape)
        fk, pk = singlet_modes(g, seed, 0, kIR, A, kc, m2[0], ad)
        F[0] = to_space(fk, N) + f0[0]
        P[0] = to_space(pk, N) + q0[0]
        for c, (fk, pk) in enumerate(complex_modes(g, seed, kIR, A, kc, m2[1:3], ad)):
            F[1 + c] = to_space(fk, N) + f0[1 + c]
            P[1 + c] = to_space(pk, N) + q0[1 + c]
        for c, (fk, pk) in enumerate(doublet_modes(g, seed, kIR, A, kc, m2[3:7], ad)):
            F[3 + c] = to_space(fk, N) + f0[3 + c]
            P[3 + c] = to_space(pk, N) + q0[3 + c]
        u, v = F[3] + 1j * F[4], F[5] + 1j * F[6]
        pu, pv = P[3] + 1j * P[4], P[5] + 1j * P[6]
        gS, gC, gD = ch[0], ch[1], ch[2]
        # SU(2) charge rho_b = r2/2 gS Re((i sigma_b Phi)^+ pi) (mattercurrents.h:86-98)
        isig = [(1j * v, 1j * u), (v, -u), (1j * u, -1j * v)]
        for b in range(3):
            a, c = isig[b]
            rho = r2 / 2 * (gS * np.real(np.conj(a) * pu + np.conj(c) * pv))
            for i, x in enumerate(gauss_solve(g, dx, rho / dx)):
                P[10 + 3 * i + b] = x
        for i in range(3):
            F[10 + 4 * i] = 1.0
        rho = 2.0 / dx * r2 * (gC * (P[1] * F[2] - P[2] * F[1]) + gD * np.imag(np.conj(pu) * u + np.conj(pv) * v))
        for i, x in enumerate(gauss_solve(g, dx, rho)):
            P[7 + i] = x
        return F, P
    raise ValueError(f"unknown model kind {kind}")
