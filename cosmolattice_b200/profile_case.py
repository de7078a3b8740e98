"""Run one evolution case through the C ABI, for profilers (ncu) and quick timing.

    python -m cosmolattice_b200.profile_case --N 256 --steps 10 --precision fp64 --path fused
    python -m cosmolattice_b200.profile_case --model lphi4U1 --N 128 --steps 5
    python -m cosmolattice_b200.profile_case --model lphi4SU2U1 --N 96 --steps 3 [--precision fp32]
    python -m cosmolattice_b200.profile_case --model batch --members 64 --steps 5 --precision fp32 [--tile 32,16,32,4]
    python -m cosmolattice_b200.profile_case --N 128 --steps 4 --gws
    python -m cosmolattice_b200.profile_case --model lphi4U1 --N 96 --steps 4 --mode adjoint
    python -m cosmolattice_b200.profile_case --model lphi4SU2U1 --N 64 --steps 2 --mode tangent

Gauge models and the batch run on seeded synthetic states (no FFT initial conditions): small
Gaussian noise about the homogeneous point, links near unity.

Workload: one real scalar, V = phi^4/4, VV2, self-consistent expansion, dt = 0.01, lattice spacing
2 pi / 64 (kIR = 64 / N), seeded small fluctuations around phi = 1.  Launch order: one
field-averages sweep (initialise), then per evolve call one kick sweep followed by one fused
sweep and one tail per step.
"""
from __future__ import annotations

import argparse
import time

import numpy as np

from . import MODELS, Lattice, ParameterParser, RunParameters, lphi4_1f


def _gauge_case(args):
    N = args.N
    rng = np.random.default_rng(99)
    if args.model == "lphi4U1":
        par = ParameterParser(params={"N": N, "kIR": 1.0, "dt": 0.005, "evolver": args.evolver, "expansion": "true",
                                      "lambda": 1.0, "cmplx_field_initial_norm": "5.6964e18", "gU1s": 0.5})
        rp = RunParameters(par)
        m = MODELS["lphi4U1"](par, rp)
        f = 1e-2 * rng.standard_normal((5, N, N, N))
        f[:2] += 2 ** -0.5
        p = 1e-2 * rng.standard_normal((5, N, N, N))
    else:
        par = ParameterParser(params={"N": N, "kIR": 1.0, "dt": 0.005, "evolver": args.evolver, "expansion": "true",
                                      "lambda": 1.0, "qG": 50, "qH": 50, "SU2Doublet_initial_norm": "5.25151e18",
                                      "gU1s": 0.35, "gSU2s": 0.6})
        rp = RunParameters(par)
        m = MODELS["lphi4SU2U1"](par, rp)
        f = 1e-2 * rng.standard_normal((22, N, N, N))
        f[3:7] += 0.5
        for i in range(3):
            f[10 + 4 * i] += 1.0
            q = f[10 + 4 * i:14 + 4 * i]
            q /= np.sqrt((q * q).sum(axis=0))
        p = 1e-2 * rng.standard_normal((19, N, N, N))
    return m, rp, f, p


def _batch(args):
    from .batch import LatticeBatch

    rng = np.random.default_rng(5)
    cases = []
    for i in range(args.members):
        N = int(rng.choice([32, 48, 64, 96]))
        par = ParameterParser(params={"N": N, "kIR": 1.0, "dt": 0.01, "evolver": "VV2", "expansion": "true",
                                      "lambda": 1.0, "initial_amplitudes": "5.6964e18"})
        rp = RunParameters(par)
        cases.append((lphi4_1f(par, rp), rp))
    bt = LatticeBatch(cases, precision=args.precision)
    if args.tile:  # a fixed sweep configuration instead of the autotuner's
        tz, ty, px, vz = (int(v) for v in args.tile.split(","))
        bt.set_tuning(tz, ty, px, vz)
    for i, (m, rp) in enumerate(cases):
        n = rp.N ** 3
        bt.set_state(i, 1.0 + 1e-3 * rng.standard_normal(n), 1e-3 * rng.standard_normal(n),
                     {"aI": 1.0, "aSI": 1.0, "aIM": 1.0, "aDotI": 0.5, "aDotSI": 0.5})
    bt.initialize()
    bt.evolve(args.steps)
    t0 = time.perf_counter()
    bt.evolve(args.steps)
    dt = time.perf_counter() - t0
    sites = sum(rp.N ** 3 for _, rp in cases)
    bt.close()
    print(f"batch of {args.members} ({sites} sites) {args.precision}: {dt * 1e3 / args.steps:.3f} ms/step")


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--N", type=int, default=256)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--precision", default="fp64", choices=["fp64", "fp32"])
    ap.add_argument("--path", default="fused", choices=["fused", "reference"])
    ap.add_argument("--evolver", default="VV2")
    ap.add_argument("--model", default="lphi4", choices=["lphi4", "lphi4U1", "lphi4SU2U1", "batch"])
    ap.add_argument("--members", type=int, default=64)
    ap.add_argument("--tile", default="", help="batch: tile_z,tile_y,planes_x,sites_per_thread (no autotuning)")
    ap.add_argument("--gws", action="store_true", help="lphi4: evolve the GW sector too")
    ap.add_argument("--mode", default="evolve", choices=["evolve", "adjoint", "tangent"],
                    help="adjoint: clb_forward + clb_backward (lphi4U1); tangent: the tangent-linear "
                         "form along g_SU2 (lphi4SU2U1)")
    args = ap.parse_args(argv)
    if args.model == "batch":
        return _batch(args)
    if args.model != "lphi4":
        m, rp, f, p = _gauge_case(args)
        lat = Lattice(m, rp, precision=args.precision)
        lat.set_state(f, p, {"aI": 1.0, "aSI": 1.0, "aIM": 1.0, "aDotI": 0.5, "aDotSI": 0.5})
        if args.mode == "tangent":
            lat.tangent_begin([0, 0, 0, 0, 1, 0])
        lat.initialize()
        t0 = time.perf_counter()
        if args.mode == "adjoint":
            lat.forward(args.steps, max(1, args.steps // 2), [0, 0, 1, 1, 0])
            lat.backward(True)
        else:
            lat.evolve(args.steps)
            if args.mode == "tangent":
                lat.tangent_observable([0] * 6 + [1] * 4)
        dt = time.perf_counter() - t0
        lat.close()
        print(f"{args.model} {args.mode} N={args.N} steps={args.steps} {args.precision}: "
              f"{dt * 1e3 / args.steps:.3f} ms/step")
        return
    N = args.N
    par = ParameterParser(params={"N": N, "kIR": 64.0 / N, "dt": 0.01, "evolver": args.evolver, "expansion": "true",
                                  "lambda": 1.0, "initial_amplitudes": "5.6964e18"})
    rp = RunParameters(par)
    model = lphi4_1f(par, rp)
    rng = np.random.default_rng(1234)
    f = 1.0 + 1e-3 * rng.standard_normal(N ** 3)
    p = 1e-3 * rng.standard_normal(N ** 3)
    lat = Lattice(model, rp, precision=args.precision, path=args.path)
    if args.gws:
        lat.gws_enable()
    lat.set_state(f, p, {"aI": 1.0, "aSI": 1.0, "aIM": 1.0, "aDotI": 0.5, "aDotSI": 0.5})
    lat.initialize()
    t0 = time.perf_counter()
    lat.evolve(args.steps)
    dt = time.perf_counter() - t0
    h = lat.history()
    lat.close()
    print(f"N={N} steps={args.steps} {args.precision} {args.path}: {dt * 1e3 / args.steps:.3f} ms/step, "
          f"a={h[-1, 0]:.9f}")


if __name__ == "__main__":
    main()
