"""Run one lphi4 evolution case through the C ABI, for profilers (ncu) and quick timing.

    python -m cosmolattice_b200.profile_case --N 256 --steps 10 --precision fp64 --path fused

Workload: one real scalar, V = phi^4/4, VV2, self-consistent expansion, dt = 0.01, lattice spacing
2 pi / 64 (kIR = 64 / N), seeded small fluctuations around phi = 1.  Launch order: one
field-averages sweep (initialise), then per evolve call one kick sweep followed by one fused
sweep and one tail per step.
"""
from __future__ import annotations

import argparse
import time

import numpy as np

from . import Lattice, ParameterParser, RunParameters, lphi4_1f


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--N", type=int, default=256)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--precision", default="fp64", choices=["fp64", "fp32"])
    ap.add_argument("--path", default="fused", choices=["fused", "reference"])
    ap.add_argument("--evolver", default="VV2")
    args = ap.parse_args(argv)
    N = args.N
    par = ParameterParser(params={"N": N, "kIR": 64.0 / N, "dt": 0.01, "evolver": args.evolver, "expansion": "true",
                                  "lambda": 1.0, "initial_amplitudes": "5.6964e18"})
    rp = RunParameters(par)
    model = lphi4_1f(par, rp)
    rng = np.random.default_rng(1234)
    f = 1.0 + 1e-3 * rng.standard_normal(N ** 3)
    p = 1e-3 * rng.standard_normal(N ** 3)
    lat = Lattice(model, rp, precision=args.precision, path=args.path)
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
