"""clb_spectrum (cuFFT D2Z + radial binning on the B200) against the numpy spectrum oracle.

Tolerances: spectra and bin k values within 1e-10 relative (per bin, against the largest bin);
per-bin mode counts bit-exact.
"""
import numpy as np
import pytest

from conftest import make_scalar_case

pytestmark = pytest.mark.gpu

TOL = 1e-10


def _lattice(N, evolver="VV2", precision="fp64", steps=5, model="lphi4_1f"):
    from cosmolattice_b200 import Lattice

    par, rp, m, f, p, sf = make_scalar_case(N=N, evolver=evolver, expansion=True, model=model, amp=1e-2)
    lat = Lattice(m, rp, precision=precision)
    lat.set_state(f, p, sf)
    lat.initialize()
    lat.evolve(steps)
    lat.sync()
    return lat, rp, m


def _close(a, b, tol=TOL):
    a, b = np.asarray(a), np.asarray(b)
    scale = max(np.abs(b).max(), 1e-300)
    return np.abs(a - b).max() <= tol * scale


@pytest.mark.parametrize("N", [32, 33, 48])
@pytest.mark.parametrize("ps_type,ps_version", [(1, 1), (2, 1), (1, 2), (2, 2)])
def test_field_and_momentum_spectra(N, ps_type, ps_version):
    from oracle.spectrum import spectrum

    lat, rp, m = _lattice(N)
    f, p, sf = lat.get_state()
    f3, p3 = f.reshape(N, N, N), p.reshape(N, N, N)
    for which, arr, factor in ((0, f3, 1.0), (1, p3, sf["aI"] ** (2 * m.alpha - 6))):
        k, v, c = lat.spectrum(which=which, ps_type=ps_type, ps_version=ps_version)
        ko, vo, co = spectrum(arr, rp.dx, ps_type=ps_type, ps_version=ps_version, factor=factor)
        assert c.tolist() == co.tolist()
        assert c.sum() == N ** 3
        assert _close(v, vo), (which, np.abs(v - vo).max() / np.abs(vo).max())
        assert _close(k, ko)
    lat.close()


@pytest.mark.parametrize("dk", [1.0, 2.0, 0.5])
def test_half_lattice_bins_without_fold(dk):
    from oracle.spectrum import spectrum

    N = 40
    lat, rp, m = _lattice(N)
    f, _, _ = lat.get_state()
    nb = int(N / 2 / dk)
    k, v, c = lat.spectrum(which=0, dk=dk, nbins=nb, fold=False)
    ko, vo, co = spectrum(f.reshape(N, N, N), rp.dx, dk=dk, nbins=nb, fold=False)
    assert c.tolist() == co.tolist()
    assert _close(v, vo)
    lat.close()


def test_two_field_component_selection():
    from oracle.spectrum import spectrum

    N = 24
    lat, rp, m = _lattice(N, model="lphi4")
    f, _, _ = lat.get_state()
    for comp in (0, 1):
        _, v, c = lat.spectrum(which=0, comp=comp)
        _, vo, co = spectrum(f.reshape(2, N, N, N)[comp], rp.dx)
        assert c.tolist() == co.tolist() and _close(v, vo)
    lat.close()


def test_fp32_state_spectrum_tracks_fp64():
    # Same initial arrays, 50 steps: over the populated band (bins holding more than 1e-6 of the
    # peak power; beyond the initial cutoff the FP64 bins hold roundoff only) the FP32/FP64-split
    # run's field spectrum stays within 1e-4 of FP64, and within 1e-4 of the peak everywhere.
    a, rp, m = _lattice(64, steps=50, precision="fp64")
    b, _, _ = _lattice(64, steps=50, precision="fp32")
    _, va, ca = a.spectrum(which=0)
    _, vb, cb = b.spectrum(which=0)
    assert ca.tolist() == cb.tolist()
    band = va > 1e-6 * va.max()
    rel = np.abs(va - vb)[band] / np.abs(va)[band]
    assert band.sum() > 5 and rel.max() < 1e-4, rel.max()
    assert np.abs(va - vb).max() < 1e-4 * va.max()
    a.close()
    b.close()
