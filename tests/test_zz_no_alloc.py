"""clb_scalar_averages_noalloc: averages of caller-owned device arrays with no device allocation.

It serves callers that cannot call cudaMalloc (a host runtime owning the whole device memory
pool, embeddings that forbid device allocation after start-up).  The
caller owns the input and output buffers (allocated here by torch); the entry point's block
partials live in its fixed device array.  Its results must match what the allocating path
(clb_measure) reports for the same state, within the parity suite's 1e-10 average tolerance, on
two calls in a row -- the second on a smaller lattice, so stale rows left by the first call in
the shared array would show.  This file is named to run after every other test.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import make_scalar_case

pytestmark = pytest.mark.gpu

AVG_TOL = 1e-10


def _lib():
    from cosmolattice_b200 import _capi

    lib = _capi.load()
    fn = lib.clb_scalar_averages_noalloc
    fn.restype = C.c_int
    fn.argtypes = [C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_double, C.c_double, C.c_double,
                   C.c_void_p, C.c_void_p]
    return lib


def _expected(model_name, N, seed):
    """(state, averages) from the allocating path: clb_measure at a = 1 without expansion gives
    E_kin = <pi^2>/2, E_grad = <grad^2>/2 per field and each <V_k> (energiesmeasurer.h:56-90)."""
    from cosmolattice_b200 import Lattice

    par, rp, m, f, p, sf = make_scalar_case(N=N, evolver="VV2", expansion=False, model=model_name, seed=seed,
                                            amp=1e-2)
    lat = Lattice(m, rp)
    lat.set_state(f, p, None)
    lat.initialize()
    e = lat.measure(1.0)["energies"]
    lat.close()
    ns = m.Ns
    pi2 = 2 * sum(e[2 * i] for i in range(ns))
    g2 = 2 * sum(e[2 * i + 1] for i in range(ns))
    pot = sum(e[2 * ns:2 * ns + m.NPotTerms])
    return rp, m, f, p, np.array([pi2, g2, pot])


def test_noalloc_matches_allocating_path_two_calls():
    import torch

    lib = _lib()
    cases = [("lphi4", 48, "na-1"), ("lphi4_1f", 24, "na-2")]
    out = torch.full((3,), float("nan"), dtype=torch.float64, device="cuda")
    for model_name, N, seed in cases:
        rp, m, f, p, expect = _expected(model_name, N, seed)
        df = torch.tensor(np.ascontiguousarray(f).ravel(), dtype=torch.float64, device="cuda")
        dp = torch.tensor(np.ascontiguousarray(p).ravel(), dtype=torch.float64, device="cuda")
        out.fill_(float("nan"))
        torch.cuda.synchronize()
        rc = lib.clb_scalar_averages_noalloc(df.data_ptr(), dp.data_ptr(), N, m.Ns, rp.dx, m.c0, m.q,
                                             out.data_ptr(), None)
        assert rc == 0, lib.clb_last_error(None)
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        assert np.all(np.abs(got - expect) <= AVG_TOL * np.abs(expect)), (model_name, N, got, expect)


def test_noalloc_rejects_sizes_beyond_its_scratch():
    import torch

    lib = _lib()
    buf = torch.zeros(16, dtype=torch.float64, device="cuda")
    rc = lib.clb_scalar_averages_noalloc(buf.data_ptr(), buf.data_ptr(), 2048, 1, 0.1, 1.0, 0.0,
                                         buf.data_ptr(), None)
    assert rc == -1
    assert b"outside [2, 1024]" in lib.clb_last_error(None)
