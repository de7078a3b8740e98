"""A model header that runs unchanged (B200): the reference's tanh2 model (models/tanh2.h) as a
header of the shape of cosmolattice_b200/csrc/models/model_api.h (potentialTerms, potDeriv,
potDeriv2 per Tag), compiled into the library in place of lphi4 (lib/tanh2/libclb200.so, selected
with CLB200_SCALAR_MODEL=tanh2), runs through the same sweeps and matches the oracle's
restatement of tanh2 with the scalar bars: per-site 1e-12 of each component's max after 60 steps,
a(t) and energies within 1e-10 (alpha = 0, self-consistent expansion, two fields, VV2, LF and
PV4); the FP32 form, which for a header without a fluctuation polynomial takes the potential
differences in FP64, follows FP64 to 1e-5 in the energies.

Each case runs in a child process, since one process loads one build of the library."""
import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SCRIPT = r"""
import json, sys
sys.path.insert(0, {root!r}); sys.path.insert(0, {tests!r})
import numpy as np
from cosmolattice_b200 import MODELS, Lattice, ParameterParser, RunParameters, _capi
from cosmolattice_b200.initializers import scalar_initial_state
from oracle.oracle import OracleLattice
assert _capi.LIB_PATH.endswith("tanh2/libclb200.so"), _capi.LIB_PATH
par = ParameterParser(params={{"N": 16, "kIR": 1.0, "dt": 0.01, "evolver": {ev!r}, "expansion": "true",
                              "M": 1e18, "Lambda4": 1e64, "q": 0.5, "initial_amplitudes": "5e18 1e16",
                              "initial_momenta": "0 0", "fluct_amplitude": 1e-2, "kCutOff": 4.0, "baseSeed": "tanh2"}})
rp = RunParameters(par)
m = MODELS["tanh2"](par, rp)
f, p, aI, aD = scalar_initial_state(m, rp)
sf = {{"aI": aI, "aSI": aI, "aIM": aI, "aDotI": aD, "aDotSI": aD}}
out = {{}}
for key, lat in (("gpu", Lattice(m, rp)), ("gpu32", Lattice(m, rp, precision="fp32")), ("cpu", OracleLattice(m, rp))):
    lat.set_state(f, p, sf); lat.initialize(); lat.evolve(60); lat.sync()
    mm = lat.measure(1.0); st = lat.get_state(); lat.close()
    out[key] = (st, mm)
(fg, pg, sg), mg = out["gpu"]; (fc, pc, sc), mc = out["cpu"]; mf = out["gpu32"][1]
def rel(a, b):
    a = a.reshape(2, -1); b = b.reshape(2, -1)
    return max(float(np.abs(a[c] - b[c]).max() / np.abs(b[c]).max()) for c in range(2))
res = {{"f": rel(fg, fc), "p": rel(pg, pc), "a": abs(sg["aI"] - sc["aI"]) / sc["aI"],
       "e": max(abs(x - y) / abs(y) for x, y in zip(mg["energies"], mc["energies"]) if y != 0),
       "e32": max(abs(x - y) / abs(y) for x, y in zip(mf["energies"], mg["energies"]) if y != 0),
       "a_grew": sg["aI"] / aI, "n_energies": len(mg["energies"])}}
print("RESULT " + json.dumps(res))
"""


@pytest.mark.parametrize("evolver", ["VV2", "LF", "PV4"])
def test_tanh2_header_matches_oracle(evolver):
    env = dict(os.environ, CLB200_SCALAR_MODEL="tanh2")
    code = SCRIPT.format(root=ROOT, tests=os.path.join(ROOT, "tests"), ev=evolver)
    r = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    res = json.loads([l for l in r.stdout.splitlines() if l.startswith("RESULT ")][-1][7:])
    assert res["n_energies"] == 7  # two fields' E_kin, E_grad, two potential terms, E_tot
    assert res["a_grew"] > 1.0
    assert res["f"] < 1e-12 and res["p"] < 1e-12, res
    assert res["a"] < 1e-10 and res["e"] < 1e-10, res
    assert res["e32"] < 1e-5, res
