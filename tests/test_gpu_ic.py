"""Device initial conditions (clb_generate_state) against the oracle's restatement (B200).

The random draws are integers (Philox4x64-10) and agree exactly; the mode values differ from the
oracle's only through the transcendental functions (log1p, sin/cos) and the FFTs, so the FP64
state agrees to 1e-12 of each component's largest magnitude.  The FP32 form stores each
component rounded once to FP32 (the lphi4 form about its volume mean): 1e-6 there.  The gauge
momenta satisfy the Gauss laws as the measurement reports them.
"""
import numpy as np
import pytest

from conftest import make_scalar_case, make_su2_case, make_u1_case
from oracle import ic_recipe as icr

pytestmark = pytest.mark.gpu

CASES = {
    "lphi4_1f": (icr.MODEL_LPHI4, lambda N: make_scalar_case(N=N, model="lphi4_1f")),
    "lphi4": (icr.MODEL_LPHI4, lambda N: make_scalar_case(N=N, model="lphi4")),
    "lphi4U1": (icr.MODEL_LPHI4U1, lambda N: make_u1_case(N=N)),
    "lphi4SU2U1": (icr.MODEL_LPHI4SU2U1, lambda N: make_su2_case(N=N)),
}


def generated(name, N, precision, seed=1234):
    from cosmolattice_b200 import Lattice
    from cosmolattice_b200.initializers import device_initial_state

    kind, make = CASES[name]
    par, rp, m, *_ = make(N)
    lat = Lattice(m, rp, precision=precision)
    p = device_initial_state(lat, m, rp, seed=seed)
    f, mom, sf = lat.get_state()
    F, P = icr.generate_state(kind, N, rp.dx, (m.fStar / m.omegaStar) ** 2, p, n_scalars=getattr(m, "Ns", 1))
    return lat, m, p, f.reshape(F.shape), mom.reshape(P.shape), sf, F, P


@pytest.mark.parametrize("name,N", [("lphi4_1f", 16), ("lphi4", 12), ("lphi4U1", 16), ("lphi4SU2U1", 8),
                                    ("lphi4U1", 10)])
def test_fp64_matches_oracle(name, N):
    lat, m, p, f, mom, sf, F, P = generated(name, N, "fp64")
    lat.close()
    assert sf["aI"] == p["aI"] and sf["aDotI"] == p["aDotI"]
    for got, ref in ((f, F), (mom, P)):
        for c in range(ref.shape[0]):
            scale = max(np.max(np.abs(ref[c])), 1e-300)
            assert np.max(np.abs(got[c] - ref[c])) <= 1e-12 * scale, (name, c)


@pytest.mark.parametrize("name,N", [("lphi4_1f", 16), ("lphi4U1", 12), ("lphi4SU2U1", 8)])
def test_fp32_form_matches_oracle(name, N):
    lat, m, p, f, mom, sf, F, P = generated(name, N, "fp32")
    lat.close()
    for got, ref in ((f, F), (mom, P)):
        for c in range(ref.shape[0]):
            scale = max(np.max(np.abs(ref[c])), 1e-300)
            assert np.max(np.abs(got[c] - ref[c])) <= 1e-6 * scale, (name, c)


def test_seed_changes_draws_and_repeats():
    from cosmolattice_b200 import Lattice
    from cosmolattice_b200.initializers import device_initial_state

    par, rp, m, *_ = make_scalar_case(N=16)
    lat = Lattice(m, rp)
    device_initial_state(lat, m, rp, seed=5)
    a = lat.get_state()[0]
    device_initial_state(lat, m, rp, seed=6)
    b = lat.get_state()[0]
    device_initial_state(lat, m, rp, seed=5)
    c = lat.get_state()[0]
    lat.close()
    assert np.array_equal(a, c) and not np.array_equal(a, b)


def test_generated_u1_state_satisfies_gauss():
    # the residual of the U(1) Gauss law is the dropped zero mode of the charge, a constant
    from test_oracle_u1 import gauss_field

    lat, m, p, f, mom, sf, F, P = generated("lphi4U1", 16, "fp64")
    lat.close()
    G, r = gauss_field(lat.rp, m, f.ravel(), mom.ravel())
    assert np.abs(G - G.mean()).max() <= 1e-12 * np.abs(r).max()


def test_generated_su2u1_state_satisfies_gauss():
    from test_oracle_su2 import gauss_fields

    lat, m, p, f, mom, sf, F, P = generated("lphi4SU2U1", 8, "fp64")
    lat.close()
    gu1, gsu2, rho = gauss_fields(lat.rp, m, f.ravel(), mom.ravel())
    assert np.abs(gu1 - gu1.mean()).max() <= 1e-12 * np.abs(rho).max() * lat.rp.dx
    u, v = f[3] + 1j * f[4], f[5] + 1j * f[6]
    scale = (m.fStar / m.omegaStar) ** 2 / 2 * m.gQ_S * max(np.abs(u).max(), np.abs(v).max()) * np.abs(mom[3:7]).max()
    for b in range(3):
        assert np.abs(gsu2[b] - gsu2[b].mean()).max() <= 1e-12 * scale


def test_generated_state_evolves():
    from cosmolattice_b200 import Lattice
    from cosmolattice_b200.initializers import device_initial_state

    par, rp, m, *_ = make_scalar_case(N=32)
    lat = Lattice(m, rp)
    device_initial_state(lat, m, rp, seed=9)
    lat.initialize()
    lat.evolve(20)
    lat.sync()
    meas = lat.measure(1.0)
    lat.close()
    assert np.all(np.isfinite(meas["energies"])) and abs(meas["friedmann"][0]) < 1e-4


def test_rejects_bad_parameters():
    from cosmolattice_b200 import Lattice, _capi

    par, rp, m, *_ = make_scalar_case(N=8)
    lat = Lattice(m, rp)
    with pytest.raises(_capi.ClbError):
        lat.generate_state({"seed": 1, "amplitude": float("nan"), "k_cutoff": 1.0, "adot": 0.0})
    lat.close()
