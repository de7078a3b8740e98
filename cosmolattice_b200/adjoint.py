"""Gradients of final energy fractions of lphi4U1 through the adjoint pair of the C ABI.

dO/dtheta = (explicit dependence of the evolution on theta, from clb_backward)
          + <fields_bar, d fields_0 / d theta> + <momenta_bar, d momenta_0 / d theta>,
with the start-state tangents of the RandomWithMatter initial state
(initializers.u1_initial_state_tangent).  theta: "amp" (fluctuation amplitude), "c4" (quartic
coupling lambda_prog), "gQ" (gauge coupling times charge).  The start state goes through
clb_initialize(correct_adot=1), whose aDot correction the backward pass differentiates.
"""
from __future__ import annotations

from typing import Dict, Iterable, Sequence, Tuple

import numpy as np

from .initializers import u1_initial_state, u1_initial_state_tangent
from .lattice import Lattice
from .models import Model
from .params import RunParameters

GAUGE_FRACTION = (0.0, 0.0, 1.0, 1.0, 0.0)  # (E_el + E_mag) / E_tot


def u1_gradients(model: Model, rp: RunParameters, n_steps: int, checkpoint_every: int,
                 weights: Sequence[float] = GAUGE_FRACTION, params: Iterable[str] = ("amp", "c4", "gQ"),
                 lattice: Lattice = None) -> Tuple[float, Dict[str, float], Dict[str, object]]:
    """(O, {param: dO/dparam}, backward record) for O = sum_k w_k E_k / E_tot after n_steps."""
    lat = lattice if lattice is not None else Lattice(model, rp)
    f, p, aI, aD = u1_initial_state(model, rp)
    lat.set_state(f, p, {"aI": aI, "aSI": aI, "aIM": aI, "aDotI": aD, "aDotSI": aD})
    lat.initialize(correct_adot=True)
    O = lat.forward(n_steps, checkpoint_every, weights)
    fb, pb, g = lat.backward(through_init=True)
    out = {}
    for prm in params:
        df, dp = u1_initial_state_tangent(model, rp, prm)
        ic = float(fb @ df.ravel() + pb @ dp.ravel())
        explicit = {"amp": 0.0, "c4": g["dO_dcouplings"][0], "gQ": g["dO_dcouplings"][1]}[prm]
        out[prm] = ic + explicit
    if lattice is None:
        lat.close()
    g["fields_bar"], g["momenta_bar"] = fb, pb
    return O, out, g


def observable_from_measurement(m: Dict[str, object], weights: Sequence[float] = GAUGE_FRACTION) -> float:
    """O = sum_k w_k E_k / E_tot from a measurement dict (energies E_0..E_4, E_tot last)."""
    e = m["energies"]
    return float(sum(w * x for w, x in zip(weights, e[:-1])) / sum(e[:-1]))
