"""Radially binned power spectrum, numpy restatement (TEST INFRASTRUCTURE ONLY).

Follows PowerSpectrumMeasurer::powerSpectrum (include/CosmoInterface/measurements/powerspectrum.h:
84-134) with the bin rule of clb_spectrum: b = floor(|n| / dk) over the full N^3 grid of integer
wave vectors, modes with b >= nbins folded into the last bin (fold) or left out.  The half
spectrum of rfftn stands for the full grid with weight 2 for kz not in {0, N/2}.
`brute_force_counts` enumerates the full grid with Python loops (small N only) and pins the
weighted half-spectrum counts.
"""
from __future__ import annotations

import math

import numpy as np


def _n_norm(N):
    nx = np.fft.fftfreq(N, 1.0 / N)
    nz = np.fft.rfftfreq(N, 1.0 / N)
    n2 = nx[:, None, None] ** 2 + nx[None, :, None] ** 2 + nz[None, None, :] ** 2
    w = np.full(nz.shape, 2.0)
    w[0] = 1.0
    if N % 2 == 0:
        w[-1] = 1.0
    return np.sqrt(n2), np.broadcast_to(w[None, None, :], n2.shape)


def bins_of(N, dk, nbins, fold):
    nn, w = _n_norm(N)
    b = np.floor(nn / dk).astype(np.int64)
    if fold:
        b = np.minimum(b, nbins - 1)
        keep = np.ones_like(b, dtype=bool)
    else:
        keep = b < nbins
    return nn, w, b, keep


def spectrum(f, dx, ps_type=1, ps_version=1, dk=1.0, nbins=None, fold=True, factor=1.0):
    """(k, value, counts) of the real N^3 array f."""
    N = f.shape[0]
    if nbins is None:
        nbins = int(math.floor(math.sqrt(3.0) / 2.0 * N / dk))
    fk = np.fft.rfftn(np.asarray(f, dtype=np.float64))
    p = fk.real ** 2 + fk.imag ** 2
    nn, w, b, keep = bins_of(N, dk, nbins, fold)
    bb = b[keep]
    ww = w[keep]
    s = np.bincount(bb, weights=ww * p[keep], minlength=nbins)[:nbins]
    sn = np.bincount(bb, weights=ww * nn[keep], minlength=nbins)[:nbins]
    c = np.bincount(bb, weights=ww, minlength=nbins)[:nbins].astype(np.int64)
    kIR = 2 * math.pi / (N * dx)
    out = np.zeros(nbins)
    k = np.zeros(nbins)
    for i in range(nbins):
        ntil = sn[i] / c[i] if (ps_version == 1 and c[i] > 0) else (i + 0.5) * dk
        k[i] = ntil * kIR
        if c[i] == 0:
            continue
        if ps_type == 1:
            out[i] = kIR * ntil * dx / dk / float(N) ** 5 / 2.0 / math.pi * s[i]
        else:
            t = kIR * ntil * dx / N
            out[i] = t * t * t / dk / 2.0 / (math.pi * math.pi) * (s[i] / c[i])
    return k, factor * out, c


def brute_force_counts(N, dk, nbins, fold):
    """Mode counts per bin by enumerating every (nx, ny, nz) of the full N^3 grid."""
    counts = [0] * nbins
    freqs = [j if j <= N // 2 else j - N for j in range(N)]
    for a in freqs:
        for b in freqs:
            for c in freqs:
                idx = int(math.floor(math.sqrt(a * a + b * b + c * c) / dk))
                if idx >= nbins:
                    if not fold:
                        continue
                    idx = nbins - 1
                counts[idx] += 1
    return counts


def gw_projected(uk, N, prj_type):
    """|Tr(Lambda u Lambda u^*)|-style projected power per mode of the five transformed components
    uk[5] (u_11, u_12, u_13, u_22, u_23; u_33 = -u_11 - u_22) with the TT projector of
    GWProjectorType1/2/3 (definitions/gwsprojector.h): lattice momenta kL_i = sin(2 pi n_i / N)
    (type 1) or sin -/+ i (1 - cos) (types 2, 3).  The zero mode, where kL = 0, contributes 0.
    Mode indices i <= N/2 stand for n = i, the others for i - N (the Nyquist index is +N/2 on every
    axis: at the corner mode (N/2, N/2, N/2) the type-1 momenta are three rounding-sized sin(pi)
    values, whose signs set the projector)."""
    idx = np.arange(N)
    nx = np.where(idx <= N // 2, idx, idx - N).astype(np.float64)
    nz = np.arange(N // 2 + 1, dtype=np.float64)
    kir = 2 * math.pi / N
    n = [nx[:, None, None], nx[None, :, None], nz[None, None, :]]
    if prj_type == 1:
        kL = [np.sin(kir * ni) + 0j for ni in n]
    else:
        sgn = -1.0 if prj_type == 2 else 1.0
        kL = [np.sin(kir * ni) + 1j * sgn * (1.0 - np.cos(kir * ni)) for ni in n]
    kL = [np.broadcast_to(k, uk[0].shape) for k in kL]
    kL2 = sum(np.abs(k) ** 2 for k in kL)
    zero = kL2 == 0
    kL2 = np.where(zero, 1.0, kL2)
    c = np.conj
    P = [1 - c(kL[0]) * kL[0] / kL2, -c(kL[0]) * kL[1] / kL2, -c(kL[0]) * kL[2] / kL2,
         1 - c(kL[1]) * kL[1] / kL2, -c(kL[1]) * kL[2] / kL2, 1 - c(kL[2]) * kL[2] / kL2]
    u = uk
    if prj_type == 1:  # real projector: P^* = P
        P = [p.real + 0j for p in P]

    def pu(uu):
        return [P[0] * uu[0] + P[1] * uu[1] + P[2] * uu[2],
                P[0] * uu[1] + P[1] * uu[3] + P[2] * uu[4],
                P[0] * uu[2] + P[1] * uu[4] - P[2] * (uu[0] + uu[3]),
                c(P[1]) * uu[0] + P[3] * uu[1] + P[4] * uu[2],
                c(P[1]) * uu[1] + P[3] * uu[3] + P[4] * uu[4],
                c(P[1]) * uu[2] + P[3] * uu[4] - P[4] * (uu[0] + uu[3]),
                c(P[2]) * uu[0] + c(P[4]) * uu[1] + P[5] * uu[2],
                c(P[2]) * uu[1] + c(P[4]) * uu[3] + P[5] * uu[4],
                c(P[2]) * uu[2] + c(P[4]) * uu[4] - P[5] * (uu[0] + uu[3])]

    Pu = pu(u)
    Pus = pu([c(x) for x in u])
    Tr1 = (Pu[0] * Pus[0] + Pu[1] * Pus[3] + Pu[2] * Pus[6] + Pu[3] * Pus[1] + Pu[4] * Pus[4] + Pu[5] * Pus[7]
           + Pu[6] * Pus[2] + Pu[7] * Pus[5] + Pu[8] * Pus[8])
    Tr2 = Pu[0] + Pu[4] + Pu[8]
    Tr2s = Pus[0] + Pus[4] + Pus[8]
    val = np.abs(Tr1 - 0.5 * Tr2 * Tr2s)
    return np.where(zero, 0.0, val)


def gw_spectrum(piu, dx, prj_type=2, ps_type=1, ps_version=1, dk=1.0, nbins=None, fold=True, factor=1.0):
    """(k, value, counts) of the GW energy spectrum of the five GW momentum components piu
    (5 x N^3) before the (fStar/MPl)^2 / (4 a^6 rho) factor, which `factor` supplies
    (PowerSpectrumMeasurer::powerSpectrumGW, powerspectrum.h:51-71)."""
    N = piu.shape[1]
    if nbins is None:
        nbins = int(math.floor(math.sqrt(3.0) / 2.0 * N / dk))
    uk = [np.fft.rfftn(np.asarray(piu[c], dtype=np.float64)) for c in range(5)]
    p = gw_projected(uk, N, prj_type)
    nn, w, b, keep = bins_of(N, dk, nbins, fold)
    bb, ww = b[keep], w[keep]
    s = np.bincount(bb, weights=ww * p[keep], minlength=nbins)[:nbins]
    sn = np.bincount(bb, weights=ww * nn[keep], minlength=nbins)[:nbins]
    cnt = np.bincount(bb, weights=ww, minlength=nbins)[:nbins].astype(np.int64)
    kIR = 2 * math.pi / (N * dx)
    out = np.zeros(nbins)
    k = np.zeros(nbins)
    for i in range(nbins):
        ntil = sn[i] / cnt[i] if (ps_version == 1 and cnt[i] > 0) else (i + 0.5) * dk
        k[i] = ntil * kIR
        if cnt[i] == 0:
            continue
        if ps_type == 1:
            out[i] = kIR * ntil * dx / dk / float(N) ** 5 / 2.0 / math.pi * s[i]
        else:
            t = kIR * ntil * dx / N
            out[i] = t * t * t / dk / 2.0 / (math.pi * math.pi) * (s[i] / cnt[i])
    return k, factor * out, cnt
