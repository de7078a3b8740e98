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
