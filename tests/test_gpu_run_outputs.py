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
