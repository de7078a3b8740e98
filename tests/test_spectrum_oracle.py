"""The spectrum oracle's binning against a brute-force enumeration of the full k-space (no GPU)."""
import math

import numpy as np
import pytest

from oracle.spectrum import bins_of, brute_force_counts, spectrum


@pytest.mark.parametrize("N", [4, 5, 8, 9, 12])
@pytest.mark.parametrize("fold", [True, False])
def test_weighted_half_spectrum_counts_equal_full_grid(N, fold):
    dk = 1.0
    nbins = int(math.floor(math.sqrt(3) / 2 * N / dk)) if fold else N // 2
    nn, w, b, keep = bins_of(N, dk, nbins, fold)
    counts = np.bincount(b[keep], weights=w[keep], minlength=nbins)[:nbins].astype(np.int64)
    assert counts.tolist() == brute_force_counts(N, dk, nbins, fold)
    if fold:
        assert counts.sum() == N ** 3


def test_spectrum_sum_rule():
    # Parseval: with every mode counted once, sum_bins (value / prefactor) = N^3 sum_x f^2
    rng = np.random.default_rng(3)
    N, dx = 16, 0.3
    f = rng.standard_normal((N, N, N))
    k, v, c = spectrum(f, dx, ps_type=1, ps_version=2, dk=1.0)
    kIR = 2 * math.pi / (N * dx)
    ntil = (np.arange(len(v)) + 0.5)
    pref = kIR * ntil * dx / 1.0 / float(N) ** 5 / 2.0 / math.pi
    total = (v / pref).sum()
    assert abs(total - N ** 3 * (f ** 2).sum()) < 1e-9 * total
    assert c.sum() == N ** 3


def test_plane_wave_spectrum_type2():
    # PS_type 2 divides by the count: a single plane wave lands in one bin with the expected power
    N, dx = 16, 0.5
    x = np.arange(N)
    X, Y, Z = np.meshgrid(x, x, x, indexing="ij")
    f = np.cos(2 * np.pi * 3 * X / N)
    k, v, c = spectrum(f, dx, ps_type=2, ps_version=1, dk=1.0)
    nz = np.nonzero(v > 1e-20 * v.max())[0]  # other bins hold FFT roundoff only
    assert list(nz) == [3]
    # |f_k|^2 = (N^3/2)^2 at n = (+-3, 0, 0); bin 3 holds the modes with 3 <= |n| < 4
    expect_avg = 2 * (N ** 3 / 2) ** 2 / c[3]
    kIR = 2 * np.pi / (N * dx)
    ntil = k[3] / kIR  # PS_version 1: the mean |n| of the bin's modes
    assert 3.0 <= ntil < 4.0
    t = kIR * ntil * dx / N
    assert abs(v[3] - t ** 3 / 2 / np.pi ** 2 * expect_avg) < 1e-12 * v[3]
