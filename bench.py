#!/usr/bin/env python
"""Throughput of the lattice time-evolution hot path on B200.

Workload (one "step" = one VV2 time step of the whole lattice): lphi4 with one real scalar,
V = phi^4/4 in program variables, N = 512 periodic, kIR = 1/8 (the 64^3 case's spacing), dt = 0.01, VV2, self-consistent
expansion, phi0 = 1 (f* = 5.6964e18 GeV, MPl = 2.435e18 GeV), Gaussian vacuum-like fluctuations
of relative amplitude 1e-3 cut at |k| <= N kIR / 4 (synthetic, seeded).

Reported:
  value            site-updates/s of the FP64 fused path (inputs resident in HBM), CUDA events
                   on the library's stream, max over ranks
  mixed            the FP32/FP64-split form on the same workload, with its Friedmann-constraint
                   and energy differences against FP64
  roofline         achieved HBM GB/s of the dominant kernel (the fused sweep) from its own
                   per-launch CUDA events, against MEASURED_PEAKS.json
  e2e              the same metric through the C ABI with host buffers: state upload from pinned
                   host memory, evolve, per-step history read back, final state download
  cpu_baseline     the FP64 CPU oracle (OpenMP, reference operation order) on a bounded sample

--impl reference times the reference's CPU implementation of this path on the host cores.  The
reference cannot be built here (its TempLat runtime is not vendored), so that arm runs the CPU
restatement of the reference's algorithm (oracle/), with all host threads.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import re
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

BYTES_PER_SITE = {"fp64": 32, "fp32": 16}  # state read once + written once per VV2 stage


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--N", type=int, default=512)
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-configs", action="store_true",
                    help="skip the shortened runs of the other workloads in the default line")
    ap.add_argument("--cpu-seconds", type=float, default=20.0)
    ap.add_argument("--config", default="lphi4", choices=["lphi4", "lphi4U1-adjoint", "batched", "lphi4SU2U1"],
                    help="lphi4: the headline 512^3 scalar workload; lphi4U1-adjoint: 128^3 VV4 gauge "
                         "run with the adjoint gradient and its finite-difference check; batched: 384 "
                         "lphi4 lattices of 32^3-96^3 in one graph-captured ensemble")
    ap.add_argument("--members", type=int, default=384)
    ap.add_argument("--seq-steps", type=int, default=200, help="steps of the one-at-a-time comparison")
    ap.add_argument("--checkpoint-every", type=int, default=50)
    return ap.parse_args()


def workload_params(N, steps):
    # The 64^3 case's lattice spacing dx = 2 pi / 64 at every N (kIR = 64 / N): at kIR = 1 a 512^3
    # lattice has dx = 2 pi / 512 and its highest mode omega_max = 2 sqrt(3) / dx gives
    # omega_max dt = 2.8 > 2, outside the stability region of velocity Verlet.  The fluctuation
    # cutoff stays at the same physical |k| <= 16 (= N kIR / 4 of the 64^3 recipe).
    kIR = 64.0 / N
    return {
        "N": N, "kIR": kIR, "dt": 0.01, "evolver": "VV2", "expansion": "true",
        "lambda": 1.0, "initial_amplitudes": "5.6964e18", "initial_momenta": "0",
        "fluct_amplitude": 1e-3, "kCutOff": 16.0, "baseSeed": "bench-512",
        "tMax": steps * 0.01,
    }


def headline_config(N, K, world):
    """The `config` object of the headline line, the same for both arms."""
    return {
        "workload": f"lphi4 1 real scalar {N}^3 VV2, self-consistent expansion, {K} steps, FP64",
        "lattice": N, "evolver": "VV2", "dt": 0.01, "kIR": 64.0 / N, "expansion": True,
        "l2": "inputs larger than L2 (state %.1f GiB)" % (2 * N ** 3 * 8 / 2 ** 30),
        "parallelism": "replicas" if world > 1 else "single GPU",
    }


def make_workload(N, steps):
    from cosmolattice_b200 import ParameterParser, RunParameters, lphi4_1f

    par = ParameterParser(params=workload_params(N, steps))
    rp = RunParameters(par)
    return rp, lphi4_1f(par, rp)


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def ncu_traffic(kernel_tag, N, precision):
    """dram bytes per launch of the fused sweep from the committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", f"ncu_{kernel_tag}.md")
    if not os.path.exists(path):
        return None
    pat = re.compile(rf"^dram_bytes_per_launch\[{precision},N={N}\]\s*[:=]\s*([0-9.eE+]+)", re.M)
    m = pat.search(open(path).read())
    return float(m.group(1)) if m else None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during a timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = os.path.join("/tmp", f"clb_clocks_{os.getpid()}_{device}.csv")

    def __enter__(self):
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", str(self.device)], stdout=self.fh, stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.fh.close()

    def summary(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        if torch.cuda.is_available():
            torch.cuda.set_device(local)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                    device_id=torch.device("cuda", local))
        else:  # the rank logic on CPU (tests): replicas need no data exchange, only barrier and max
            dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def max_over_ranks(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device="cuda" if dist.get_backend() == "nccl" else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job(units_per_rank, ms_local, world):
    """(max over ranks of the ms, whole-job units per second): every rank runs its own replica of
    units_per_rank units in ms_local; the job's time is the slowest rank's."""
    ms = max_over_ranks(ms_local, world)
    return ms, world * units_per_rank / (ms * 1e-3)


def open_form(rp, model, fields, momenta, sf, precision, warmup, device):
    """A lattice of one storage form with the start state, initialized, measured and warmed up."""
    from cosmolattice_b200 import Lattice

    lat = Lattice(model, rp, precision=precision, path="fused", device=device)
    lat.set_state(fields, momenta, sf)
    lat.initialize()
    lat.sync()
    m0 = lat.measure(1.0)
    if warmup > 0:
        lat.evolve(warmup)
    lat.set_profiling(False)
    return lat, m0


def timed_pass(lat, steps, device, world):
    """`steps` fused VV2 steps bracketed by barrier + synchronize; device ms from the events the
    library records on its stream around the evolve call (no per-kernel events)."""
    import torch

    torch.cuda.synchronize(device)
    barrier(world)
    lat.evolve(steps)
    torch.cuda.synchronize(device)
    barrier(world)
    return lat.last_evolve_ms()


def close_form(lat, m0, steps, device):
    """The same steps once more with an event pair around every launch (per-kernel durations for
    the roofline), then the final measurement and spectra."""
    import torch

    lat.reset_stats()
    lat.set_profiling(True)
    lat.evolve(steps)
    torch.cuda.synchronize(device)
    ms_prof = lat.last_evolve_ms()
    stats = lat.kernel_stats()
    lat.set_profiling(False)
    lat.sync()
    m1 = lat.measure(m0["energies"][-1])
    hist = lat.history()
    # field spectra at the end of the run: the reference's default bins and N/2 bins
    torch.cuda.synchronize(device)
    t0 = time.perf_counter()
    spec = lat.spectrum(which=0)
    torch.cuda.synchronize(device)
    spec_ms = (time.perf_counter() - t0) * 1e3
    spec_half = lat.spectrum(which=0, nbins=lat.rp.N // 2, fold=False)
    lat.close()
    return {"ms_prof": ms_prof, "stats": stats, "m0": m0, "m1": m1, "hist_rows": len(hist),
            "spec": spec, "spec_half": spec_half, "spec_ms": spec_ms}


def spectrum_error(a, b):
    """max relative difference of spectrum b to a over a's populated band (> 1e-6 of its peak)."""
    import numpy as np

    va, vb = a[1], b[1]
    band = va > 1e-6 * va.max()
    return float((np.abs(va - vb)[band] / np.abs(va)[band]).max())


def run_e2e(rp, model, fields, momenta, sf, steps, device):
    """Through the C ABI with host buffers: upload from pinned memory, evolve, read back every
    step's (a, aDot, averages) row and the final state."""
    import numpy as np
    import torch

    from cosmolattice_b200 import Lattice

    n = fields.size
    hf = torch.empty(n, dtype=torch.float64, pin_memory=True).numpy()
    hp = torch.empty(n, dtype=torch.float64, pin_memory=True).numpy()
    hf[:] = fields.ravel()
    hp[:] = momenta.ravel()
    out_f = torch.empty(n, dtype=torch.float64, pin_memory=True).numpy()
    out_p = torch.empty(n, dtype=torch.float64, pin_memory=True).numpy()
    lat = Lattice(model, rp, precision="fp64", path="fused", device=device)
    torch.cuda.synchronize(device)
    t0 = time.perf_counter()
    lat.set_state(hf, hp, sf)
    lat.initialize()
    lat.evolve(steps)
    hist = lat.history()
    import ctypes as C

    from cosmolattice_b200 import _capi

    sfo = _capi.ScaleFactor()
    lat._check(lat.lib.clb_get_state(lat.h, out_f.ctypes.data_as(C.POINTER(C.c_double)),
                                     out_p.ctypes.data_as(C.POINTER(C.c_double)), C.byref(sfo)))
    torch.cuda.synchronize(device)
    dt = time.perf_counter() - t0
    lat.close()
    assert np.isfinite(hist).all() and len(hist) == steps
    state_bytes = 2 * n * 8
    return {
        "value": rp.N ** 3 * steps / dt,
        "seconds": dt,
        "h2d_bytes_per_step": state_bytes / steps,
        "d2h_bytes_per_step": (state_bytes + hist.nbytes) / steps,
    }


def cpu_baseline(rp, model, fields, momenta, sf, budget_s, max_steps=None):
    """FP64 CPU oracle (reference operation order) timed on the host cores, bounded sample."""
    from oracle.oracle import OracleLattice, num_threads

    o = OracleLattice(model, rp)
    o.set_state(fields, momenta, sf)
    o.initialize()
    t0 = time.perf_counter()
    o.evolve(1)
    one = time.perf_counter() - t0
    steps = max(1, int(budget_s / max(one, 1e-9)) - 1)
    if max_steps is not None:
        steps = min(steps, max_steps)
    t0 = time.perf_counter()
    o.evolve(steps)
    dt = time.perf_counter() - t0
    o.close()
    return {
        "value": rp.N ** 3 * steps / dt, "unit": "site-updates/s", "cores": num_threads(), "kind": "port",
        "sample": f"{steps} VV2 steps of the {rp.N}^3 lattice after 1 untimed step ({dt:.1f} s)",
    }


def roofline(stats, N, precision, peak, peak_kind):
    st = stats["scalar_fused_sweep"]
    if not st["timed_launches"]:
        return None
    per_launch_ms = st["total_ms"] / st["timed_launches"]
    alg_bytes = BYTES_PER_SITE[precision] * N ** 3
    achieved = alg_bytes / (per_launch_ms * 1e-3) / 1e9
    return {
        "bound": "hbm", "kernel": "scalar_fused_sweep", "achieved": round(achieved, 1), "peak": peak,
        "peak_kind": peak_kind, "unit": "GB/s", "frac": round(achieved / peak, 4),
        "algorithmic_bytes_per_launch": alg_bytes, "launch_ms": round(per_launch_ms, 5),
        "traffic": ncu_traffic("scalar_fused_sweep", N, precision),
    }


def main_u1_adjoint(args):
    """128^3 lphi4U1, VV4, dt = 0.005, g = 0.5, lambda = 1, amplitude 1e-3, self-consistent
    expansion: forward + backward time of the adjoint pair, gradients of the final gauge-energy
    fraction against central differences (relative h = 1e-4) of the plain GPU path."""
    import torch

    from cosmolattice_b200 import MODELS, Lattice, ParameterParser, RunParameters
    from cosmolattice_b200.adjoint import GAUGE_FRACTION, observable_from_measurement, u1_gradients

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    N = args.N if args.N != 512 else 128
    steps = args.steps if args.steps != 2000 else 1000
    base = {"amp": 1e-3, "c4": 1.0, "gQ": 0.5}

    def setup(over=None):
        v = dict(base)
        v.update(over or {})
        par = ParameterParser(params={
            "N": N, "kIR": 1.0, "dt": 0.005, "evolver": "VV4", "expansion": "true", "lambda": 1.0,
            "lambda_prog": v["c4"], "cmplx_field_initial_norm": "5.6964e18", "cmplx_momentum_initial_norm": "0",
            "gU1s": v["gQ"], "CSU1_charges": 1, "fluct_amplitude": v["amp"], "kCutOff": N / 4.0, "baseSeed": "cfg3"})
        rp = RunParameters(par)
        return rp, MODELS["lphi4U1"](par, rp)

    def plain(over, precision="fp64"):
        from cosmolattice_b200.initializers import u1_initial_state

        rp, m = setup(over)
        f, p, aI, aD = u1_initial_state(m, rp)
        lat = Lattice(m, rp, precision=precision)
        lat.set_state(f, p, {"aI": aI, "aSI": aI, "aIM": aI, "aDotI": aD, "aDotSI": aD})
        lat.initialize()
        lat.evolve(steps)
        ms = lat.last_evolve_ms()
        o = observable_from_measurement(lat.measure(1.0))
        lat.close()
        return o, ms

    from cosmolattice_b200.initializers import u1_initial_state, u1_initial_state_tangent

    rp, m = setup()
    # start state and its tangents (host setup, outside the timed forward and backward calls)
    t0 = time.perf_counter()
    state = u1_initial_state(m, rp)
    tangents = {prm: u1_initial_state_tangent(m, rp, prm, state) for prm in ("amp", "c4", "gQ")}
    setup_s = time.perf_counter() - t0
    # one untimed gradient first (module loading, checkpoint and segment allocation), then the timed one
    lat = Lattice(m, rp)
    lat.set_profiling(False)
    u1_gradients(m, rp, steps, args.checkpoint_every, GAUGE_FRACTION, lattice=lat, state=state, tangents=tangents)
    O, grads, rec = u1_gradients(m, rp, steps, args.checkpoint_every, GAUGE_FRACTION, lattice=lat, state=state,
                                 tangents=tangents)
    t_total = rec["forward_s"] + rec["backward_s"]
    fwd_ms = lat.last_evolve_ms()
    lat.close()
    # FP32/FP64 split: FP32 state storage and stencils, FP64 increments, sums and cotangents
    lat = Lattice(m, rp, precision="fp32")
    lat.set_profiling(False)
    u1_gradients(m, rp, steps, args.checkpoint_every, GAUGE_FRACTION, lattice=lat, state=state, tangents=tangents)
    O32, grads32, rec32 = u1_gradients(m, rp, steps, args.checkpoint_every, GAUGE_FRACTION, lattice=lat,
                                       state=state, tangents=tangents)
    t_total32 = rec32["forward_s"] + rec32["backward_s"]
    fwd_ms32 = lat.last_evolve_ms()
    lat.close()
    _, plain_ms32 = plain({}, "fp32")
    fdv, plain_ms = {}, []
    for prm in ("amp", "c4", "gQ"):
        h = 1e-4 * base[prm]
        up, ms1 = plain({prm: base[prm] + h})
        dn, ms2 = plain({prm: base[prm] - h})
        plain_ms += [ms1, ms2]
        fdv[prm] = (up - dn) / (2 * h)
    sites = N ** 3
    line = {
        "metric": "adjoint gradient of the final gauge-energy fraction (forward + backward wall time, from an initialized start state)",
        "value": t_total, "unit": "s", "higher_is_better": False, "n_gpus": 1, "steps": steps,
        "dtype": "f64", "data": "synthetic (seeded RandomWithMatter initial state)",
        "config": {"workload": f"lphi4U1 {N}^3 VV4 dt=0.005 g=0.5 lambda=1 amplitude=1e-3, expansion, "
                               f"{steps} steps, checkpoint every {args.checkpoint_every}"},
        "observable": O,
        "gradient": grads,
        "finite_difference": fdv,
        "rel_diff": {k: abs(grads[k] - fdv[k]) / abs(fdv[k]) for k in grads},
        "forward_ms": fwd_ms,
        "forward_site_updates_per_s": sites * steps / (fwd_ms * 1e-3),
        "plain_evolve_ms": statistics.median(plain_ms),
        "forward_wall_s": rec["forward_s"], "backward_wall_s": rec["backward_s"],
        "backward_over_forward": rec["backward_s"] / rec["forward_s"],
        "gradient_over_plain_evolve": t_total * 1e3 / statistics.median(plain_ms),
        "start_state_and_tangents_host_s": setup_s,
        "fp32_split": {
            "value": t_total32, "unit": "s", "observable": O32, "gradient": grads32,
            "backward_over_forward": rec32["backward_s"] / rec32["forward_s"],
            "rel_diff_vs_fp64": {k: abs(grads32[k] - grads[k]) / abs(grads[k]) for k in grads},
            "rel_diff_vs_fd": {k: abs(grads32[k] - fdv[k]) / abs(fdv[k]) for k in grads},
            "forward_ms": fwd_ms32, "forward_site_updates_per_s": sites * steps / (fwd_ms32 * 1e-3),
            "plain_evolve_ms": plain_ms32,
            "plain_evolve_speedup_vs_fp64": statistics.median(plain_ms) / plain_ms32,
        },
    }
    print(json.dumps(line))


def main_batched(args):
    """384 independent lphi4 lattices, N uniform in {32, 48, 64, 96}, lambda log-uniform in
    [0.5, 2], amplitude log-uniform in [1e-4, 1e-2], one seed each, FP32/FP64 split, VV2,
    dt = 0.01, expansion: the whole ensemble as one CUDA graph per evolve call, against the same
    lattices run one at a time through the single-lattice handle."""
    import numpy as np
    import torch

    from cosmolattice_b200 import MODELS, Lattice, ParameterParser, RunParameters
    from cosmolattice_b200.batch import LatticeBatch
    from cosmolattice_b200.initializers import scalar_initial_state

    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    torch.cuda.set_device(local)
    steps = args.steps
    rng = np.random.default_rng(20261203 + rank)
    cases = []
    for i in range(args.members):
        N = int(rng.choice([32, 48, 64, 96]))
        lam = float(np.exp(rng.uniform(np.log(0.5), np.log(2.0))))
        amp = float(np.exp(rng.uniform(np.log(1e-4), np.log(1e-2))))
        par = ParameterParser(params={
            "N": N, "kIR": 1.0, "dt": 0.01, "evolver": "VV2", "expansion": "true", "lambda": 1.0,
            "lambda_prog": lam, "initial_amplitudes": "5.6964e18", "initial_momenta": "0",
            "fluct_amplitude": amp, "kCutOff": N / 4.0, "baseSeed": f"ens{rank}-{i}"})
        rp = RunParameters(par)
        m = MODELS["lphi4_1f"](par, rp)
        f, p, aI, aD = scalar_initial_state(m, rp)
        cases.append((m, rp, f, p, {"aI": aI, "aSI": aI, "aIM": aI, "aDotI": aD, "aDotSI": aD}))
    sites = sum(c[1].N ** 3 for c in cases)

    def batch_run(precision, n):
        bt = LatticeBatch([(c[0], c[1]) for c in cases], precision=precision, device=local)
        for i, c in enumerate(cases):
            bt.set_state(i, c[2], c[3], c[4])
        bt.initialize()
        bt.evolve(args.warmup)
        l0 = bt.kernel_launches()
        with ClockSampler(local) as clk:
            bt.evolve(n)
        ms = bt.last_evolve_ms()
        launches = bt.kernel_launches() - l0
        meas = [bt.measure(i) for i in range(len(cases))]
        tuning[precision] = dict(bt.tuning(), form=bt.form())
        bt.close()
        return ms, launches, meas, clk.summary()

    tuning = {}
    ms32, launches, m32, clocks = batch_run("fp32", steps)
    ms64, _, m64, _ = batch_run("fp64", steps)
    # one at a time through the single-lattice handle (FP32 split), seq_steps each
    seq_ms = 0.0
    for c in cases:
        lat = Lattice(c[0], c[1], precision="fp32", device=local)
        lat.set_state(c[2], c[3], c[4])
        lat.initialize()
        lat.evolve(args.warmup)
        lat.evolve(args.seq_steps)
        seq_ms += lat.last_evolve_ms()
        lat.close()
    value = sites * steps / (ms32 * 1e-3)
    seq_value = sites * args.seq_steps / (seq_ms * 1e-3)
    fr = [abs(a["friedmann"][0] - b["friedmann"][0]) for a, b in zip(m32, m64)]
    ar = [abs(a["aI"] - b["aI"]) / b["aI"] for a, b in zip(m32, m64)]
    er = [max(abs(x - y) / abs(y) for x, y in zip(a["energies"], b["energies"]) if y != 0) for a, b in zip(m32, m64)]
    if rank != 0:
        return
    peak, peak_kind = measured_peaks()
    achieved = sites * 16 * steps / (ms32 * 1e-3) / 1e9
    line = {
        "metric": "ensemble site-updates/s (batched FP32/FP64 split, one graph per evolve call, the faster of the per-stage and persistent forms)",
        "value": value * world, "unit": "site-updates/s", "n_gpus": world, "steps": steps, "warmup": args.warmup,
        "ms_per_step": ms32 / steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 storage, f64 reductions", "data": "synthetic (seeded Gaussian vacuum fluctuations per member)",
        "config": {"workload": f"{len(cases)} lphi4 lattices, N in {{32,48,64,96}}, VV2 dt=0.01, expansion, {steps} steps",
                   "total_sites": sites, "members_by_N": {str(n): sum(1 for c in cases if c[1].N == n) for n in (32, 48, 64, 96)},
                   "l2": "inputs larger than L2 (ensemble state %.2f GiB)" % (sites * 16 / 2 ** 30)},
        "roofline": {"bound": "hbm", "kernel": "batch sweep + tails (whole step)", "achieved": round(achieved, 1),
                     "peak": peak, "peak_kind": peak_kind, "unit": "GB/s", "frac": round(achieved / peak, 4),
                     "algorithmic_bytes_per_step": sites * 16},
        "fp64_batch": {"value": sites * steps / (ms64 * 1e-3), "ms_per_step": ms64 / steps},
        "sweep_autotuner": tuning,
        "one_at_a_time": {"value": seq_value, "steps": args.seq_steps, "path": "single-lattice handle, FP32 split",
                          "batched_speedup": value / seq_value},
        "fp32_vs_fp64": {"friedmann_abs_diff_max": max(fr), "a_rel_diff_max": max(ar), "energy_rel_diff_max": max(er)},
        "gpu_launches": launches,
        "clocks": clocks,
    }
    print(json.dumps(line))


def main_su2(args):
    """lphi4SU2U1, N^3 (default 384), dt = 0.005, VV2, self-consistent expansion, lambda = 1,
    g_SU2 = 0.6, g_U1 = 0.35, qG = qH = 50 and the homogeneous doublet of lphi4SU2U1.in, unit links,
    fluctuations of relative amplitude 1e-3 cut at N kIR / 4: FP64 site-updates/s with both Gauss
    checks, energies and a doublet spectrum at the start and the end."""
    import torch

    from cosmolattice_b200 import MODELS, Lattice, ParameterParser, RunParameters
    from cosmolattice_b200.initializers import su2u1_initial_state

    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    N = args.N if args.N != 512 else 384
    steps = args.steps if args.steps != 2000 else 1000
    par = ParameterParser(params={
        "N": N, "kIR": 1.0, "dt": 0.005, "evolver": "VV2", "expansion": "true", "lambda": 1.0, "qG": 50, "qH": 50,
        "initial_amplitudes": 0.0, "initial_momenta": 0.0, "cmplx_field_initial_norm": 0.0,
        "cmplx_momentum_initial_norm": 0.0, "SU2Doublet_initial_norm": "5.25151e18",
        "SU2Doublet_initial_momenta_norm": 0.0, "gU1s": 0.35, "gSU2s": 0.6, "fluct_amplitude": 1e-3,
        "kCutOff": N / 4.0, "baseSeed": f"cfg4-{rank}"})
    rp = RunParameters(par)
    m = MODELS["lphi4SU2U1"](par, rp)
    t0 = time.perf_counter()
    f, p, aI, aD = su2u1_initial_state(m, rp)
    ic_s = time.perf_counter() - t0
    sf = {"aI": aI, "aSI": aI, "aIM": aI, "aDotI": aD, "aDotSI": aD}

    def run(precision):
        lat = Lattice(m, rp, precision=precision, device=local)
        lat.set_state(f, p, sf)
        lat.initialize()
        lat.sync()
        m0 = lat.measure(1.0)
        lat.evolve(args.warmup)
        lat.set_profiling(True)
        lat.reset_stats()
        with ClockSampler(local) as clk:
            lat.evolve(steps)
        ms = lat.last_evolve_ms()
        stats = lat.kernel_stats()
        lat.set_profiling(False)
        lat.sync()
        m1 = lat.measure(m0["energies"][-1])
        k1, s1, _ = lat.spectrum(which=0, comp=3)
        lat.close()
        return {"ms": ms, "stats": stats, "m0": m0, "m1": m1, "spec": s1, "clocks": clk.summary()}

    r64 = run("fp64")
    r32 = run("fp32")

    # d(gauge-energy fraction)/d g_SU2 by the tangent-linear form, FP64 and FP32 storage
    from cosmolattice_b200.adjoint import SU2_GAUGE_FRACTION

    from cosmolattice_b200.initializers import su2u1_initial_state_tangent

    dfs, dps, cds = su2u1_initial_state_tangent(m, rp, "gSU2", (f, p))
    sfs = {"aI": aI, "aSI": aI, "aIM": aI, "aDotI": aD, "aDotSI": aD}

    def grad_run(precision):
        lat = Lattice(m, rp, precision=precision, device=local)
        t0 = time.perf_counter()
        lat.set_state(f, p, sfs)
        lat.tangent_begin(cds, dfs, dps)
        lat.initialize()
        lat.evolve(steps)
        lat.sync()
        O, dO = lat.tangent_observable(SU2_GAUGE_FRACTION)
        E, dE = lat.tangent_energies()
        wall = time.perf_counter() - t0
        ms = lat.last_evolve_ms()
        lat.close()
        return {"observable": O, "gradient": dO, "energies": E.tolist(), "d_energies": dE.tolist(),
                "evolve_ms": ms, "wall_s": wall}

    g64 = grad_run("fp64")
    g32 = grad_run("fp32")
    # central difference of the plain FP64 path at h = 1e-2 g_SU2: the start state is linear in
    # g_SU2 (only the Gauss-solved SU(2) momenta depend on it), so it is p + (g - g0) dp.  Smaller
    # steps are dominated by rounding in the SU(2) magnetic energy, 4/(dx^4 g^2) sum(2 - tr P),
    # which is 1e-11 of E_tot here.
    fdE = []
    h = 1e-2 * 0.6
    for g in (0.6 + h, 0.6 - h):
        par_g = ParameterParser(params=dict(par.params, gSU2s=g))
        rp_g = RunParameters(par_g)
        m_g = MODELS["lphi4SU2U1"](par_g, rp_g)
        lat = Lattice(m_g, rp_g, device=local)
        lat.set_state(f, p + (g - 0.6) * dps.reshape(p.shape), sfs)
        lat.initialize()
        lat.evolve(steps)
        lat.sync()
        e = lat.measure(1.0)["energies"]
        fdE.append(list(e[:10]) + [sum(e[10:13])])
        lat.close()
    del f, p, dfs, dps
    fd_comp = [(a - b) / (2 * h) for a, b in zip(fdE[0], fdE[1])]
    Ow = [sum(w * x for w, x in zip(SU2_GAUGE_FRACTION, E)) / sum(E) for E in fdE]
    fd = (Ow[0] - Ow[1]) / (2 * h)
    names = ["Ekin_S", "Egrad_S", "Ekin_phi", "Egrad_phi", "Ekin_Phi", "Egrad_Phi", "Eel_U1", "Emag_U1",
             "Eel_SU2", "Emag_SU2", "V"]
    comp_diff = {nm: abs(t - d) / abs(d) if d else None for nm, t, d in zip(names, g64["d_energies"], fd_comp)}
    if rank != 0:
        return
    sites = N ** 3
    peak, peak_kind = measured_peaks()

    def roof(r, esz):
        # one kick sweep of all five sectors = its parts' launches together; the timed call runs
        # the call's first kick and then one merged sweep per VV2 step
        kick = r["stats"].get("gauge_kick_sweep", {})
        sweeps = steps + 1
        kms = kick["total_ms"] / sweeps if kick.get("timed_launches") else None
        byts = sites * esz * (22 + 2 * 19)
        return {"bound": "hbm", "kernel": "kick sweep (all five sectors, its parts together)", "launch_ms": kms,
                "parts_per_sweep": kick.get("launches", 0) / sweeps,
                "algorithmic_bytes_per_launch": byts, "achieved": byts / (kms * 1e-3) / 1e9 if kms else None,
                "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
                "frac": (byts / (kms * 1e-3) / 1e9) / peak if kms else None}

    m64, m32 = r64["m1"], r32["m1"]
    line = {
        "metric": "site-updates/s (lphi4SU2U1)", "value": sites * steps / (r64["ms"] * 1e-3), "unit": "site-updates/s",
        "n_gpus": 1, "steps": steps, "warmup": args.warmup, "ms_per_step": r64["ms"] / steps, "higher_is_better": True,
        "dtype": "f64", "data": "synthetic (seeded doublet, complex-scalar and scalar fluctuations; unit links)",
        "config": {"workload": f"lphi4SU2U1 {N}^3 VV2 dt=0.005 gSU2=0.6 gU1=0.35 lambda=1 qG=qH=50, expansion, {steps} steps"},
        "roofline": roof(r64, 8),
        "fp32": {"value": sites * steps / (r32["ms"] * 1e-3), "ms_per_step": r32["ms"] / steps,
                 "speedup_vs_fp64": r64["ms"] / r32["ms"], "roofline": roof(r32, 4),
                 "unitarize_every": 10,
                 "a_rel_diff": abs(m32["aI"] - m64["aI"]) / m64["aI"],
                 # per component, on the scale of E_tot (the magnetic energies sit at roundoff here)
                 "energy_diff_over_etot": max(abs(x - y) for x, y in zip(m32["energies"], m64["energies"])) / abs(m64["energies"][-1]),
                 "gauss_su2_end": m32["gauss_su2"], "gauss_u1_end": m32["gauss_u1"],
                 "spectrum_rel_diff": float(abs(r32["spec"] - r64["spec"]).max() / abs(r64["spec"]).max())},
        "gauss_su2": {"start": r64["m0"]["gauss_su2"], "end": m64["gauss_su2"]},
        "gauss_u1": {"start": r64["m0"]["gauss_u1"], "end": m64["gauss_u1"]},
        "energies_start": r64["m0"]["energies"], "energies_end": m64["energies"],
        "friedmann_end": m64["friedmann"], "a_end": m64["aI"],
        "doublet_spectrum_bins": len(r64["spec"]), "doublet_spectrum_end_head": [float(x) for x in r64["spec"][:8]],
        "initial_state_s": ic_s,
        "kernel_launches": {k: v["launches"] for k, v in r64["stats"].items() if v["launches"]},
        "gradient_gSU2": {
            "observable": "(E_el + E_mag of U(1) and SU(2)) / E_tot at the end",
            "method": "tangent-linear (forward-mode) evolution, one pass, no checkpoints",
            "fp64": g64, "fp32": g32,
            "finite_difference": fd, "fd_step": "h = 1e-2 g_SU2 (central)",
            "rel_diff_fp64_vs_fd": abs(g64["gradient"] - fd) / abs(fd),
            "rel_diff_fp32_vs_fd": abs(g32["gradient"] - fd) / abs(fd),
            "rel_diff_fp32_vs_fp64": abs(g32["gradient"] - g64["gradient"]) / abs(g64["gradient"]),
            "d_energies_fd": fd_comp, "d_energies_rel_diff_fp64_vs_fd": comp_diff,
            "cost_vs_plain_fp64": g64["evolve_ms"] / r64["ms"], "cost_fp32_vs_plain_fp32": g32["evolve_ms"] / r32["ms"],
        },
        "clocks": r64["clocks"], "clocks_fp32": r32["clocks"],
    }
    print(json.dumps(line))


def run_configs(local, cpu_cores_ok=True):
    """Shortened but full-size runs of the other workloads, each with its throughput, its roofline
    on the algorithmic bytes per site-update (state read once and written once per stage) and its
    clocks, for the default bench line:
      lphi4_64     lphi4 64^3 kIR = 1 VV2, all 5000 steps on the GPU (FP64, FP32 split) and on the
                   CPU oracle, with the GPU-vs-CPU differences at the end;
      batched      384 lphi4 lattices of 32^3-96^3, 200 steps, batched (FP32, FP64) against the same
                   members one at a time;
      lphi4U1      128^3 VV4 dt = 0.005 g = 0.5: 100 plain steps (FP64, FP32) and one adjoint
                   gradient over them with checkpoints every 10 steps, its cost over the forward;
      lphi4SU2U1   384^3 VV2 dt = 0.005: 20 steps FP64 and FP32 from a device-drawn start state,
                   with the Gauss ratios at the start and end."""
    import numpy as np
    import torch

    from cosmolattice_b200 import MODELS, Lattice, ParameterParser, RunParameters
    from cosmolattice_b200.initializers import device_initial_state, scalar_initial_state, u1_initial_state

    peak, peak_kind = measured_peaks()
    out = {}

    def roof(bytes_per_step, ms_per_step, what):
        ach = bytes_per_step / (ms_per_step * 1e-3) / 1e9
        return {"bound": "hbm", "basis": what, "achieved": round(ach, 1), "peak": peak, "peak_kind": peak_kind,
                "unit": "GB/s", "frac": round(ach / peak, 4)}

    def sf_of(aI, aD):
        return {"aI": aI, "aSI": aI, "aIM": aI, "aDotI": aD, "aDotSI": aD}

    # ---- lphi4 64^3, 5000 steps ----
    t0 = time.perf_counter()
    par = ParameterParser(params={"N": 64, "kIR": 1.0, "dt": 0.01, "evolver": "VV2", "expansion": "true",
                                  "lambda": 1.0, "initial_amplitudes": "5.6964e18", "initial_momenta": "0",
                                  "fluct_amplitude": 1e-3, "kCutOff": 16.0, "baseSeed": "cfg0"})
    rp = RunParameters(par)
    m = MODELS["lphi4_1f"](par, rp)
    f, p, aI, aD = scalar_initial_state(m, rp)
    K0 = 5000
    res = {}
    for prec in ("fp64", "fp32"):
        lat = Lattice(m, rp, precision=prec, device=local)
        lat.set_state(f, p, sf_of(aI, aD))
        lat.initialize()
        lat.sync()
        e0 = lat.measure(1.0)["energies"][-1]
        with ClockSampler(local) as clk:
            lat.evolve(K0)
        ms = lat.last_evolve_ms()
        lat.sync()
        res[prec] = (ms, lat.measure(e0), lat.get_state(), clk.summary())
        lat.close()
    from oracle.oracle import OracleLattice, num_threads

    o = OracleLattice(m, rp)
    o.set_state(f, p, sf_of(aI, aD))
    o.initialize()
    o.sync()
    e0c = o.measure(1.0)["energies"][-1]
    tc = time.perf_counter()
    o.evolve(K0)
    cpu_s = time.perf_counter() - tc
    o.sync()
    mc, sc = o.measure(e0c), o.get_state()
    o.close()
    sites = 64 ** 3
    ms64, m64, s64, clk64 = res["fp64"]
    ms32, m32 = res["fp32"][0], res["fp32"][1]
    fl = float(np.abs(s64[0] - sc[0]).max() / np.abs(sc[0] - sc[0].mean()).max())
    out["lphi4_64"] = {
        "workload": "lphi4 64^3 kIR=1 dt=0.01 VV2, expansion, amplitude 1e-3, 5000 steps",
        "fp64": {"value": sites * K0 / (ms64 * 1e-3), "ms_per_step": ms64 / K0,
                 "roofline": roof(32 * sites, ms64 / K0, "32 B/site/step FP64 (state in L2: above HBM is possible)")},
        "fp32": {"value": sites * K0 / (ms32 * 1e-3), "ms_per_step": ms32 / K0},
        "cpu": {"value": sites * K0 / cpu_s, "seconds": cpu_s, "cores": num_threads(), "kind": "port"},
        "gpu_over_cpu": (sites * K0 / (ms64 * 1e-3)) / (sites * K0 / cpu_s),
        "gpu_vs_cpu_after_5000_steps": {
            "a_rel": abs(s64[2]["aI"] - sc[2]["aI"]) / sc[2]["aI"],
            "friedmann_abs": abs(m64["friedmann"][0] - mc["friedmann"][0]),
            "energy_rel": max(abs(x - y) / abs(y) for x, y in zip(m64["energies"], mc["energies"]) if y != 0),
            "field_rel_to_fluctuations": fl},
        "fp32_vs_fp64": {"friedmann_abs": abs(m32["friedmann"][0] - m64["friedmann"][0]),
                         "energy_rel": max(abs(x - y) / abs(y) for x, y in zip(m32["energies"], m64["energies"]) if y != 0)},
        "clocks": clk64, "seconds": time.perf_counter() - t0}

    # ---- batched ensemble: 384 members, 200 steps ----
    from cosmolattice_b200.batch import LatticeBatch

    t0 = time.perf_counter()
    rng = np.random.default_rng(20261203)
    cases = []
    for i in range(384):
        N = int(rng.choice([32, 48, 64, 96]))
        lam = float(np.exp(rng.uniform(np.log(0.5), np.log(2.0))))
        amp = float(np.exp(rng.uniform(np.log(1e-4), np.log(1e-2))))
        par = ParameterParser(params={
            "N": N, "kIR": 1.0, "dt": 0.01, "evolver": "VV2", "expansion": "true", "lambda": 1.0,
            "lambda_prog": lam, "initial_amplitudes": "5.6964e18", "initial_momenta": "0",
            "fluct_amplitude": amp, "kCutOff": N / 4.0, "baseSeed": f"ens-{i}"})
        rpi = RunParameters(par)
        mi = MODELS["lphi4_1f"](par, rpi)
        fi, pi_, a_, d_ = scalar_initial_state(mi, rpi)
        cases.append((mi, rpi, fi, pi_, sf_of(a_, d_)))
    bsites = sum(c[1].N ** 3 for c in cases)
    KB = 200
    bres = {}
    for prec in ("fp32", "fp64"):
        bt = LatticeBatch([(c[0], c[1]) for c in cases], precision=prec, device=local)
        for i, c in enumerate(cases):
            bt.set_state(i, c[2], c[3], c[4])
        bt.initialize()
        bt.evolve(5)
        with ClockSampler(local) as clk:
            bt.evolve(KB)
        bres[prec] = (bt.last_evolve_ms(), clk.summary(), bt.tuning(), bt.form())
        bt.close()
    seq_ms = 0.0
    by_n = {}  # N -> [members, summed ms over KB steps]
    for c in cases:
        lat = Lattice(c[0], c[1], precision="fp32", device=local)
        lat.set_state(c[2], c[3], c[4])
        lat.initialize()
        lat.evolve(3)
        lat.evolve(KB)
        ms = lat.last_evolve_ms()
        seq_ms += ms
        by_n.setdefault(c[1].N, [0, 0.0])
        by_n[c[1].N][0] += 1
        by_n[c[1].N][1] += ms
        lat.close()
    # per member size: the single-lattice handle's ms per step and its fraction of the HBM roofline
    # on 16 B/site/step, to tell the handle's small-lattice overhead from the batch sweep's quality
    one_by_n = {}
    for n_, (cnt, ms) in sorted(by_n.items()):
        per = ms / cnt / KB
        one_by_n[str(n_)] = {"members": cnt, "ms_per_step": per,
                             "roofline": roof(16 * n_ ** 3, per, "16 B/site/step FP32 storage, one lattice")}
    b32, b64 = bres["fp32"][0], bres["fp64"][0]
    out["batched"] = {
        "workload": "384 lphi4 lattices, N in {32,48,64,96}, lambda log-uniform [0.5,2], amplitude log-uniform "
                    "[1e-4,1e-2], VV2 dt=0.01, expansion, 200 steps",
        "total_sites": bsites,
        "fp32": {"value": bsites * KB / (b32 * 1e-3), "ms_per_step": b32 / KB,
                 "roofline": roof(16 * bsites, b32 / KB, "16 B/site/step FP32 storage, whole step")},
        "fp64": {"value": bsites * KB / (b64 * 1e-3), "ms_per_step": b64 / KB,
                 "roofline": roof(32 * bsites, b64 / KB, "32 B/site/step FP64, whole step")},
        "one_at_a_time_fp32": {"value": bsites * KB / (seq_ms * 1e-3), "ms_per_step": seq_ms / KB,
                               "by_N": one_by_n},
        "batched_speedup": seq_ms / b32,
        "tuning": bres["fp32"][2], "form": {"fp32": bres["fp32"][3], "fp64": bres["fp64"][3]},
        "clocks": bres["fp32"][1], "seconds": time.perf_counter() - t0}
    del cases

    # ---- lphi4U1 128^3 VV4: 100 steps and one gradient (K = 10) ----
    from cosmolattice_b200.adjoint import GAUGE_FRACTION, u1_gradients

    t0 = time.perf_counter()
    par = ParameterParser(params={
        "N": 128, "kIR": 1.0, "dt": 0.005, "evolver": "VV4", "expansion": "true", "lambda": 1.0, "lambda_prog": 1.0,
        "cmplx_field_initial_norm": "5.6964e18", "cmplx_momentum_initial_norm": "0", "gU1s": 0.5,
        "CSU1_charges": 1, "fluct_amplitude": 1e-3, "kCutOff": 32.0, "baseSeed": "cfg3"})
    rp = RunParameters(par)
    m = MODELS["lphi4U1"](par, rp)
    state = u1_initial_state(m, rp)
    f, p, aI, aD = state
    K3 = 100
    ures = {}
    for prec in ("fp64", "fp32"):
        lat = Lattice(m, rp, precision=prec, device=local)
        lat.set_state(f, p, sf_of(aI, aD))
        lat.initialize()
        lat.evolve(3)
        with ClockSampler(local) as clk:
            lat.evolve(K3)
        ures[prec] = (lat.last_evolve_ms(), clk.summary())
        lat.close()
    lat = Lattice(m, rp, device=local)
    u1_gradients(m, rp, K3, 10, GAUGE_FRACTION, params=(), lattice=lat, state=state)  # warm
    O, _, rec = u1_gradients(m, rp, K3, 10, GAUGE_FRACTION, params=(), lattice=lat, state=state)
    lat.close()
    sites = 128 ** 3
    u64, u32 = ures["fp64"][0], ures["fp32"][0]
    grad_s = rec["forward_s"] + rec["backward_s"]
    out["lphi4U1"] = {
        "workload": "lphi4U1 128^3 VV4 dt=0.005 g=0.5 lambda=1 amplitude 1e-3, expansion, 100 steps; "
                    "gradient of the final gauge-energy fraction, checkpoints every 10 steps",
        "fp64": {"value": sites * K3 / (u64 * 1e-3), "ms_per_step": u64 / K3,
                 "roofline": roof(3 * 160 * sites, u64 / K3, "160 B/site/stage FP64, 3 stages")},
        "fp32": {"value": sites * K3 / (u32 * 1e-3), "ms_per_step": u32 / K3, "speedup_vs_fp64": u64 / u32,
                 "roofline": roof(3 * 80 * sites, u32 / K3, "80 B/site/stage FP32 storage, 3 stages")},
        "gradient": {"observable": O, "forward_s": rec["forward_s"], "backward_s": rec["backward_s"],
                     "gradient_over_plain_forward": grad_s * 1e3 / u64},
        "clocks": ures["fp64"][1], "seconds": time.perf_counter() - t0}
    del state, f, p

    # ---- lphi4SU2U1 384^3 VV2, 20 steps ----
    t0 = time.perf_counter()
    par = ParameterParser(params={
        "N": 384, "kIR": 1.0, "dt": 0.005, "evolver": "VV2", "expansion": "true", "lambda": 1.0, "qG": 50, "qH": 50,
        "initial_amplitudes": 0.0, "initial_momenta": 0.0, "cmplx_field_initial_norm": 0.0,
        "cmplx_momentum_initial_norm": 0.0, "SU2Doublet_initial_norm": "5.25151e18",
        "SU2Doublet_initial_momenta_norm": 0.0, "gU1s": 0.35, "gSU2s": 0.6, "fluct_amplitude": 1e-3,
        "kCutOff": 96.0, "baseSeed": "cfg4"})
    rp = RunParameters(par)
    m = MODELS["lphi4SU2U1"](par, rp)
    K4 = 20
    sres = {}
    for prec in ("fp64", "fp32"):
        lat = Lattice(m, rp, precision=prec, device=local)
        device_initial_state(lat, m, rp, seed=4)
        lat.initialize()
        lat.sync()
        m0 = lat.measure(1.0)
        lat.evolve(2)
        with ClockSampler(local) as clk:
            lat.evolve(K4)
        ms = lat.last_evolve_ms()
        lat.sync()
        m1 = lat.measure(m0["energies"][-1])
        sres[prec] = (ms, m0, m1, clk.summary())
        lat.close()
    torch.cuda.empty_cache()
    sites = 384 ** 3
    s64, s32 = sres["fp64"], sres["fp32"]
    out["lphi4SU2U1"] = {
        "workload": "lphi4SU2U1 384^3 VV2 dt=0.005 gSU2=0.6 gU1=0.35 lambda=1 qG=qH=50, expansion, 20 steps "
                    "(device-drawn start state)",
        "fp64": {"value": sites * K4 / (s64[0] * 1e-3), "ms_per_step": s64[0] / K4,
                 "roofline": roof(656 * sites, s64[0] / K4, "656 B/site/step FP64 (41 reals read and written)")},
        "fp32": {"value": sites * K4 / (s32[0] * 1e-3), "ms_per_step": s32[0] / K4, "speedup_vs_fp64": s64[0] / s32[0],
                 "roofline": roof(328 * sites, s32[0] / K4, "328 B/site/step FP32 storage")},
        "gauss_su2": {"fp64": [s64[1]["gauss_su2"][0], s64[2]["gauss_su2"][0]],
                      "fp32": [s32[1]["gauss_su2"][0], s32[2]["gauss_su2"][0]], "order": "start, end"},
        "gauss_u1": {"fp64": [s64[1]["gauss_u1"][0], s64[2]["gauss_u1"][0]],
                     "fp32": [s32[1]["gauss_u1"][0], s32[2]["gauss_u1"][0]], "order": "start, end"},
        "fp32_vs_fp64": {"a_rel": abs(s32[2]["aI"] - s64[2]["aI"]) / s64[2]["aI"],
                         "energy_diff_over_etot": max(abs(x - y) for x, y in zip(s32[2]["energies"], s64[2]["energies"]))
                         / abs(s64[2]["energies"][-1])},
        "clocks": s64[3], "seconds": time.perf_counter() - t0}
    return out


def main():
    args = parse_args()
    if args.config == "lphi4SU2U1":
        return main_su2(args)
    if args.config == "batched":
        return main_batched(args)
    if args.config == "lphi4U1-adjoint":
        return main_u1_adjoint(args)
    if args.impl == "reference":
        return main_reference(args)
    world, rank, local = dist_setup(args)
    import torch

    torch.cuda.set_device(local)
    from cosmolattice_b200.initializers import scalar_initial_state

    N, K, W = args.N, args.steps, args.warmup
    rp, model = make_workload(N, K)
    fields, momenta, aI, aDot = scalar_initial_state(model, rp)
    sf = {"aI": aI, "aSI": aI, "aIM": aI, "aDotI": aDot, "aDotSI": aDot}

    # Both forms resident; timed passes in the order FP64, FP32, FP32, FP64, so that the power-cap
    # clock drift over the run weighs on both alike.  value: the first FP64 pass; the FP32/FP64
    # ratio: the means of the two passes of each form.
    lat64, m064 = open_form(rp, model, fields, momenta, sf, "fp64", W, local)
    lat32, m032 = open_form(rp, model, fields, momenta, sf, "fp32", W, local)
    with ClockSampler(local) as clk:
        t64a = timed_pass(lat64, K, local, world)
        t32a = timed_pass(lat32, K, local, world)
        t32b = timed_pass(lat32, K, local, world)
        t64b = timed_pass(lat64, K, local, world)
    r64 = close_form(lat64, m064, K, local)
    r32 = close_form(lat32, m032, K, local)
    r64["clocks"] = r32["clocks"] = clk.summary()
    # the FP64 path in the reference's own operation order (separate kick, drift and reduction
    # sweeps), for the FP32/FP64 ratio against it too: a 200-step sample after warm-up
    from cosmolattice_b200 import Lattice

    lref = Lattice(model, rp, precision="fp64", path="reference", device=local)
    lref.set_state(fields, momenta, sf)
    lref.initialize()
    lref.evolve(3)
    kref = min(K, 200)
    tref = timed_pass(lref, kref, local, world) / kref
    lref.close()
    sites = N ** 3
    ms64, value64 = whole_job(sites * K, t64a, world)
    ms32 = max_over_ranks(t32a, world)
    ms64_mean = max_over_ranks(0.5 * (t64a + t64b), world)
    ms32_mean, value32 = whole_job(sites * K, 0.5 * (t32a + t32b), world)
    e2e = run_e2e(rp, model, fields, momenta, sf, K, local)
    e2e_val = max_over_ranks(1.0 / e2e["value"], world)
    cpu = None
    if rank == 0 and not args.no_cpu:
        cpu = cpu_baseline(rp, model, fields, momenta, sf, args.cpu_seconds)
    if rank != 0:
        return
    configs = None
    if world == 1 and not args.no_configs:
        del fields, momenta
        configs = run_configs(local)
    peak, peak_kind = measured_peaks()
    f64, f32 = r64["m1"], r32["m1"]
    launches = sum(v["launches"] for v in r64["stats"].values())
    line = {
        "metric": "site-updates/s, mixed vs FP64 GPU at equal constraint error; HBM % of peak",
        "value": value64,
        "unit": "site-updates/s",
        "n_gpus": world,
        "steps": K,
        "warmup": W,
        "ms_per_step": ms64 / K,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (seeded Gaussian vacuum fluctuations, BASELINE recipe)",
        "config": headline_config(N, K, world),
        "roofline": roofline(r64["stats"], N, "fp64", peak, peak_kind),
        "ms_per_step_kernel_events_pass": r64["ms_prof"] / K,
        "fp64_reference_order": {"ms_per_step": tref, "value": world * sites / (tref * 1e-3),
                                 "path": "kick, drift and reduction sweeps in the reference's order (200-step sample)"},
        "timed_passes_ms_per_step": {"fp64": [t64a / K, t64b / K], "fp32": [t32a / K, t32b / K],
                                     "order": "fp64, fp32, fp32, fp64"},
        "kernel_ms_per_launch": {form: {k: v["total_ms"] / v["timed_launches"] for k, v in r["stats"].items()
                                        if v["timed_launches"]} for form, r in (("fp64", r64), ("fp32", r32))},
        "mixed": {
            "value": value32, "ms_per_step": ms32_mean / K, "speedup_vs_fp64": ms64_mean / ms32_mean,
            "speedup_vs_fp64_reference_order": tref / (ms32_mean / K),
            "ms_per_step_kernel_events_pass": r32["ms_prof"] / K,
            "roofline": roofline(r32["stats"], N, "fp32", peak, peak_kind),
            "friedmann_fp32": f32["friedmann"][0], "friedmann_fp64": f64["friedmann"][0],
            "friedmann_abs_diff": abs(f32["friedmann"][0] - f64["friedmann"][0]),
            "energy_rel_diff": max(abs(a - b) / abs(b) for a, b in zip(f32["energies"], f64["energies"]) if b != 0),
            "a_rel_diff": abs(f32["aI"] - f64["aI"]) / f64["aI"],
            "spectrum_rel_diff": spectrum_error(r64["spec"], r32["spec"]),
            "spectrum_rel_diff_half_bins": spectrum_error(r64["spec_half"], r32["spec_half"]),
            "spectrum_bins": [len(r64["spec"][1]), len(r64["spec_half"][1])],
            "mode_counts_equal": bool((r64["spec"][2] == r32["spec"][2]).all()),
        },
        "spectrum_ms": r64["spec_ms"],
        "e2e": {"value": 1.0 / e2e_val if world > 1 else e2e["value"], "unit": "site-updates/s",
                "h2d_bytes_per_step": e2e["h2d_bytes_per_step"], "d2h_bytes_per_step": e2e["d2h_bytes_per_step"],
                "seconds": e2e["seconds"], "timer": "host wall clock around the C-ABI calls"},
        "gpu_launches": launches,
        "kernel_launches": {k: v["launches"] for k, v in r64["stats"].items() if v["launches"]},
        "clocks": r64["clocks"],
        "clocks_mixed": r32["clocks"],
        "cpu_baseline": cpu,
        "history_rows": r64["hist_rows"],
        "configs": configs,
    }
    print(json.dumps(line))


def main_reference(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from cosmolattice_b200.initializers import scalar_initial_state

    N, K, W = args.N, args.steps, args.warmup
    rp, model = make_workload(N, K)
    fields, momenta, aI, aDot = scalar_initial_state(model, rp)
    sf = {"aI": aI, "aSI": aI, "aIM": aI, "aDotI": aDot, "aDotSI": aDot}
    # the reference's CPU path on all host threads, bounded to a few minutes for K steps
    budget = min(120.0, max(10.0, 2.0 * args.cpu_seconds))
    cpu = cpu_baseline(rp, model, fields, momenta, sf, budget, max_steps=K)
    line = {
        "metric": "site-updates/s, mixed vs FP64 GPU at equal constraint error; HBM % of peak",
        "value": cpu["value"], "unit": "site-updates/s", "n_gpus": world, "steps": K, "warmup": W,
        "ms_per_step": N ** 3 / cpu["value"] * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded Gaussian vacuum fluctuations, BASELINE recipe)",
        "config": headline_config(N, K, world),
        "impl": "reference",
        "cpu_baseline": cpu,
        "e2e": {"value": cpu["value"], "unit": "site-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "the reference needs its un-vendored TempLat runtime (CMake FetchContent), so its CPU "
                "algorithm runs as the FP64 restatement in oracle/ (reference operation order, OpenMP)",
    }
    print(json.dumps(line))


if __name__ == "__main__":
    main()
