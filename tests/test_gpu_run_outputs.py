"""The reference main loop over the GPU library (lattice.run): output files in the reference's
text layout (measurementssaverstd.h:61-82, spectrumsaverstd.h:54-96) and their cadence
(measurer.h:48-53, 87-197), for a scalar and a gauge model (B200)."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _read(path):
    with open(path) as fh:
        return fh.read().splitlines()


@pytest.mark.parametrize("model", ["lphi4_1f", "lphi4U1"])
def test_run_writes_reference_files(tmp_path, model):
    from cosmolattice_b200 import ParameterParser, run

    params = {"N": 16, "kIR": 1.0, "dt": 0.01, "evolver": "VV2", "expansion": "true", "lambda": 1.0,
              "tMax": 0.5, "tOutputFreq": 0.1, "tOutputInfreq": 0.25, "kCutOff": 4, "fluct_amplitude": 1e-2,
              "print_headers": "true"}
    if model == "lphi4_1f":
        params.update({"initial_amplitudes": "5.6964e18", "initial_momenta": "0"})
    else:
        params.update({"cmplx_field_initial_norm": "5.6964e18", "gU1s": 0.5})
    history, lat = run(ParameterParser(params=params), model, outdir=str(tmp_path))
    lat.close()
    files = sorted(os.listdir(tmp_path))
    assert "average_energies.txt" in files and "average_scale_factor.txt" in files
    en = _read(tmp_path / "average_energies.txt")
    assert en[0].startswith("#t")
    # the loop runs while t < tMax - dt/2 and measures before evolving: t = 0, 0.1, ..., 0.4
    assert len(en) - 1 == 5
    spec_files = [f for f in files if f.startswith("spectra_")]
    assert spec_files
    nb = int(np.floor(np.sqrt(3.0) / 2.0 * 16))
    for f in spec_files:
        lines = _read(tmp_path / f)
        assert lines[0].startswith("1:binCentralValue")
        blocks = "\n".join(lines[1:]).strip().split("\n\n")
        assert len(blocks) == 2  # t = 0, 0.25
        rows = [list(map(float, r.split())) for r in blocks[0].splitlines()]
        assert len(rows) == nb
        assert abs(rows[0][0] - 0.5) < 1e-12 and abs(rows[1][0] - 1.5) < 1e-12  # bin centres x kIR
    if model == "lphi4U1":
        assert "average_gauss_U1_0.txt" in files and "average_norm_U1_0.txt" in files


# ---- file values against the oracle -------------------------------------------------------------

def _oracle_lattice_factory():
    """An oracle-driven lattice for lattice.run: the FP64 CPU restatement, with the spectra of its
    state from the numpy spectrum oracle (momentum factors a^(2 alpha - 6) for matter and
    a^(2 alpha - 2) for gauge components, as clb_spectrum applies them)."""
    from oracle.oracle import OracleLattice
    from oracle.spectrum import spectrum

    class OracleRun(OracleLattice):
        def __init__(self, model, rp):
            super().__init__(model, rp)
            self.model = model

        def spectrum(self, which=0, comp=0, ps_type=1, ps_version=1, dk=1.0, nbins=None, fold=True):
            f, p, sf = self.get_state()
            N = self.rp.N
            arr = (f if which == 0 else p).reshape(-1, N, N, N)[comp]
            m = self.model
            gauge = (getattr(m, "NSU2", 0) and comp >= 7) or (not getattr(m, "NSU2", 0) and getattr(m, "NU1", 0)
                                                              and comp >= 2)
            factor = 1.0 if which == 0 else sf["aI"] ** (2 * m.alpha - (2 if gauge else 6))
            return spectrum(arr, self.rp.dx, ps_type=ps_type, ps_version=ps_version, dk=dk, nbins=nbins, fold=fold,
                            factor=factor)

    return OracleRun


CASES = {
    "lphi4_1f": {"initial_amplitudes": "5.6964e18", "initial_momenta": "0"},
    "lphi4": {"initial_amplitudes": "5.6964e18 1e17", "initial_momenta": "0 0", "q": 1.5},
    "lphi4U1": {"cmplx_field_initial_norm": "5.6964e18", "gU1s": 0.5},
    "lphi4SU2U1": {"qG": 50, "qH": 50, "initial_amplitudes": 0.0, "initial_momenta": 0.0,
                   "cmplx_field_initial_norm": 0.0, "cmplx_momentum_initial_norm": 0.0,
                   "SU2Doublet_initial_norm": "5.25151e18", "SU2Doublet_initial_momenta_norm": 0.0,
                   "gU1s": 0.35, "gSU2s": 0.6, "dt": 0.005},
}

# energiesmeasurer.h:127-150 for each model
ENERGY_HEADERS = {
    "lphi4_1f": "t E^kin_scal0 E^grad_scal0 Vpot_term_0 E_tot",
    "lphi4": "t E^kin_scal0 E^grad_scal0 E^kin_scal1 E^grad_scal1 Vpot_term_0 Vpot_term_1 E_tot",
    "lphi4U1": "t E^kin_cmplxscal0 E^grad_cmplxscal0 E^kin_U10 E^grad_U10 Vpot_term_0 E_tot",
    "lphi4SU2U1": "t E^kin_scal0 E^grad_scal0 E^kin_cmplxscal0 E^grad_cmplxscal0 E^kin_SU2matter E^grad_SU2matter "
                  "E^kin_U10 E^grad_U10 E^kin_SU2 E^grad_SU2 Vpot_term_0 Vpot_term_1 Vpot_term_2 E_tot",
}


@pytest.mark.parametrize("model", ["lphi4_1f", "lphi4", "lphi4U1", "lphi4SU2U1"])
def test_file_values_match_the_oracle_run(tmp_path, model):
    # The same main loop (lattice.run) driven once over the GPU library and once over the FP64 CPU
    # oracle: every number of every average_*.txt file within 1e-10 of its column's largest value
    # (the Gauss ratios and the rms columns within 1e-8 relative, the Friedmann ratio within 1e-12
    # absolute: these are differences of nearly equal terms), every spectra_*.txt
    # column within 1e-10 of its largest value, and the energies header in the reference's order.
    from cosmolattice_b200 import ParameterParser, run

    N = 8 if model == "lphi4SU2U1" else 16
    params = {"N": N, "kIR": 1.0, "dt": 0.01, "evolver": "VV2", "expansion": "true", "lambda": 1.0,
              "tMax": 0.3, "tOutputFreq": 0.05, "tOutputInfreq": 0.1, "kCutOff": N / 4, "fluct_amplitude": 1e-2,
              "print_headers": "true", "baseSeed": "files"}
    params.update(CASES[model])
    params["tMax"] = 30 * params["dt"]
    params["tOutputFreq"] = 5 * params["dt"]
    params["tOutputInfreq"] = 10 * params["dt"]
    gdir, cdir = tmp_path / "gpu", tmp_path / "cpu"
    _, lat = run(ParameterParser(params=params), model, outdir=str(gdir))
    lat.close()
    _, lat = run(ParameterParser(params=params), model, outdir=str(cdir), lattice_factory=_oracle_lattice_factory())
    lat.close()
    gfiles, cfiles = sorted(os.listdir(gdir)), sorted(os.listdir(cdir))
    assert gfiles == cfiles
    assert _read(gdir / "average_energies.txt")[0] == "#" + ENERGY_HEADERS[model].replace(" ", "    ")
    for name in gfiles:
        if name.startswith("average_"):
            a = np.loadtxt(gdir / name, ndmin=2)
            b = np.loadtxt(cdir / name, ndmin=2)
            assert a.shape == b.shape, name
            # the mean of |B| of SU(2) takes sqrt(B^2) per site as the reference does
            # (su2measurer.h:62); near unit links B^2 can round below zero: NaN on both sides
            assert np.array_equal(np.isnan(a), np.isnan(b)), name
            a, b = np.nan_to_num(a), np.nan_to_num(b)
            is_means = b.shape[1] == 7 and not name.startswith(("average_energ", "average_scale", "average_gauss"))
            for col in range(1, b.shape[1]):
                # the Gauss ratio and the rms columns of the means files, sqrt(<x^2> - <x>^2), are
                # differences of nearly equal terms
                tol = 1e-8 if (name.startswith("average_gauss") and col == 1) or (is_means and col >= 5) else 1e-10
                if name == "average_energy_conservation.txt" and col == 1:
                    # (LHS - RHS)/(LHS + RHS), or |1 - E/E0|: a difference of nearly equal terms
                    assert np.abs(a[:, col] - b[:, col]).max() <= 1e-12, (name, col)
                elif tol == 1e-8:
                    assert np.all(np.abs(a[:, col] - b[:, col]) <= tol * np.abs(b[:, col]) + 1e-300), (name, col)
                else:
                    scale = max(np.abs(b[:, col]).max(), 1e-300)
                    assert np.abs(a[:, col] - b[:, col]).max() <= tol * scale, (name, col)
        else:
            ga = "\n".join(_read(gdir / name)[1:]).strip().split("\n\n")
            ca = "\n".join(_read(cdir / name)[1:]).strip().split("\n\n")
            assert len(ga) == len(ca) == 3, name  # t = 0, 0.1, 0.2 (x dt units)
            for bg, bc in zip(ga, ca):
                a = np.array([list(map(float, r.split())) for r in bg.splitlines()])
                b = np.array([list(map(float, r.split())) for r in bc.splitlines()])
                assert a.shape == b.shape, name
                for col in range(b.shape[1]):
                    scale = max(np.abs(b[:, col]).max(), 1e-300)
                    assert np.abs(a[:, col] - b[:, col]).max() <= 1e-10 * scale, (name, col)
