"""Gradients of final energy fractions: lphi4U1 through the adjoint pair of the C ABI, lphi4SU2U1
through its tangent-linear form.

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
                 lattice: Lattice = None, state=None, tangents=None, spectrum: Dict[str, object] = None
                 ) -> Tuple[float, Dict[str, float], Dict[str, object]]:
    """(O, {param: dO/dparam}, backward record) for O = sum_k w_k E_k / E_tot after n_steps.
    spectrum: instead O = sum_b w_b P_b, P the binned spectrum of one component at the end state,
    given as {"which", "comp", "bin_weights"} plus Lattice.spectrum's optional ps_type,
    ps_version, dk, fold.  state: u1_initial_state(model, rp) if already made; tangents:
    {param: (df, dp)} likewise.  The record holds the wall times of the forward and backward calls."""
    import time

    lat = lattice if lattice is not None else Lattice(model, rp)
    if state is None:
        state = u1_initial_state(model, rp)
    f, p, aI, aD = state
    lat.set_state(f, p, {"aI": aI, "aSI": aI, "aIM": aI, "aDotI": aD, "aDotSI": aD})
    lat.initialize(correct_adot=True)
    t0 = time.perf_counter()
    if spectrum is not None:
        sp = dict(spectrum)
        O = lat.forward_spectrum(n_steps, checkpoint_every, sp.pop("which"), sp.pop("comp"), sp.pop("bin_weights"), **sp)
    else:
        O = lat.forward(n_steps, checkpoint_every, weights)
    t1 = time.perf_counter()
    fb, pb, g = lat.backward(through_init=True)
    t2 = time.perf_counter()
    g["forward_s"], g["backward_s"] = t1 - t0, t2 - t1
    out = {}
    for prm in params:
        df, dp = tangents[prm] if tangents is not None else u1_initial_state_tangent(model, rp, prm, state)
        ic = float(fb @ df.ravel() + pb @ dp.ravel())
        explicit = {"amp": 0.0, "c4": g["dO_dcouplings"][0], "gQ": g["dO_dcouplings"][1]}[prm]
        out[prm] = ic + explicit
    if lattice is None:
        lat.close()
    g["fields_bar"], g["momenta_bar"] = fb, pb
    return O, out, g


SU2_GAUGE_FRACTION = (0.0,) * 6 + (1.0, 1.0, 1.0, 1.0, 0.0)  # (E_el + E_mag of U(1) and SU(2)) / E_tot


def su2_gradient(model: Model, rp: RunParameters, n_steps: int, param: str = "gSU2",
                 weights: Sequence[float] = SU2_GAUGE_FRACTION, lattice: Lattice = None,
                 state=None) -> Tuple[float, float]:
    """(O, dO/dparam) for O = sum_k w_k E_k / E_tot of lphi4SU2U1 after n_steps, param "gSU2" or
    "gU1", by the tangent-linear form (clb_tangent_*): the start state of su2u1_initial_state with
    its tangent, clb_initialize(correct_adot=1) and the evolution differentiated in one pass.
    E_k: E_kin and E_grad of S, phi, Phi; E_el, E_mag of U(1) and SU(2); V."""
    from .initializers import su2u1_initial_state, su2u1_initial_state_tangent

    lat = lattice if lattice is not None else Lattice(model, rp)
    if state is None:
        state = su2u1_initial_state(model, rp)
    f, p, aI, aD = state
    lat.set_state(f, p, {"aI": aI, "aSI": aI, "aIM": aI, "aDotI": aD, "aDotSI": aD})
    df, dp, cd = su2u1_initial_state_tangent(model, rp, param, (f, p))
    lat.tangent_begin(cd, df, dp)
    lat.initialize(correct_adot=True)
    lat.evolve(n_steps)
    lat.sync()
    O, dO = lat.tangent_observable(weights)
    lat.tangent_end()
    if lattice is None:
        lat.close()
    return O, dO


def su2_observable_from_measurement(m: Dict[str, object], weights: Sequence[float] = SU2_GAUGE_FRACTION) -> float:
    """O = sum_k w_k E_k / E_tot from an lphi4SU2U1 measurement dict (10 sector energies, the three
    potential terms, E_tot): V is the sum of the potential terms."""
    e = list(m["energies"])
    comps = e[:10] + [sum(e[10:13])]
    return float(sum(w * x for w, x in zip(weights, comps)) / sum(comps))


def observable_from_measurement(m: Dict[str, object], weights: Sequence[float] = GAUGE_FRACTION) -> float:
    """O = sum_k w_k E_k / E_tot from a measurement dict (energies E_0..E_4, E_tot last)."""
    e = m["energies"]
    return float(sum(w * x for w, x in zip(weights, e[:-1])) / sum(e[:-1]))
