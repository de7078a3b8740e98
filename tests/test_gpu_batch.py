"""Batched lphi4 ensemble (clb_batch_*) against single-lattice runs (B200).

FP64 batch: every member matches the CPU oracle run on its own, per site within 1e-12 after the
run (same kernels' rounding as the single path; only the volume-sum order differs), a(t) and
energies within 1e-10.  FP32/FP64-split batch: each member within the bounds of the
single-lattice FP32 split test (fields 1e-6 of max |phi|, fluctuations 1e-3, a(t) 1e-7,
Friedmann 1e-6 absolute) of its FP64 run.  Sizes are ragged and differ per member.
"""
import numpy as np
import pytest

from conftest import make_scalar_case

pytestmark = pytest.mark.gpu

MEMBERS = [(8, 1.0, 1e-3, "a"), (12, 0.5, 1e-2, "b"), (16, 2.0, 3e-3, "c"), (13, 1.3, 1e-4, "d"), (33, 0.8, 5e-3, "e")]


def members(evolver="VV2", expansion=True, dt=0.01):
    out = []
    for N, lam, amp, seed in MEMBERS:
        out.append(make_scalar_case(N=N, evolver=evolver, expansion=expansion, dt=dt, seed=seed, amp=amp,
                                    extra={"lambda_prog": lam}))
    return out


def rel(a, b):
    return np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-300)


def run_batch(cases, precision, steps, chunks=1, tuning=None):
    from cosmolattice_b200.batch import LatticeBatch

    bt = LatticeBatch([(c[2], c[1]) for c in cases], precision=precision)
    if tuning is not None:
        bt.set_tuning(*tuning)
    for i, c in enumerate(cases):
        bt.set_state(i, c[3], c[4], c[5])
    bt.initialize()
    m0 = [bt.measure(i) for i in range(len(cases))]
    for _ in range(chunks):
        bt.evolve(steps // chunks)
    out = [bt.get_state(i) for i in range(len(cases))]
    m1 = [bt.measure(i, m0[i]["energies"][-1]) for i in range(len(cases))]
    bt.close()
    return out, m0, m1


def run_oracle(c, steps):
    from oracle.oracle import OracleLattice

    o = OracleLattice(c[2], c[1])
    o.set_state(c[3], c[4], c[5])
    o.initialize()
    m0 = o.measure(1.0)
    o.evolve(steps)
    st = o.get_state()
    m1 = o.measure(m0["energies"][-1])
    o.close()
    return st, m0, m1


@pytest.mark.parametrize("evolver,expansion", [("VV2", True), ("VV4", True), ("VV2", False)])
def test_fp64_batch_matches_oracle_per_member(evolver, expansion):
    cases = members(evolver, expansion)
    out, m0, m1 = run_batch(cases, "fp64", 40, chunks=2)
    for i, c in enumerate(cases):
        (fo, po, so), mo0, mo1 = run_oracle(c, 40)
        fg, pg, sg = out[i]
        assert rel(fg, fo) < 1e-12 and rel(pg, po) < 1e-12, (i, rel(fg, fo), rel(pg, po))
        assert abs(sg["aI"] - so["aI"]) <= 1e-10 * so["aI"]
        for a, b in zip(m1[i]["energies"], mo1["energies"]):
            assert abs(a - b) <= 1e-10 * abs(b) + 1e-300


def test_fp32_batch_tracks_fp64():
    cases = members("VV2", True)
    g32, _, m32 = run_batch(cases, "fp32", 100)
    g64, _, m64 = run_batch(cases, "fp64", 100)
    for i in range(len(cases)):
        (fa, pa, sa), (fb, pb, sb) = g32[i], g64[i]
        assert rel(fa, fb) < 1e-6
        assert rel(fa - fa.mean(), fb - fb.mean()) < 1e-3, (i, rel(fa - fa.mean(), fb - fb.mean()))
        assert abs(sa["aI"] - sb["aI"]) / sb["aI"] < 1e-7
        assert abs(m32[i]["friedmann"][0] - m64[i]["friedmann"][0]) < 1e-6


def test_batch_equals_single_lattice_fp64_and_graph_replay():
    # the batch member and the single-lattice handle run the same arithmetic; replaying a cached
    # graph (same step count twice) continues the run correctly
    from cosmolattice_b200 import Lattice
    from cosmolattice_b200.batch import LatticeBatch

    cases = members("VV2", True)[:3]
    bt = LatticeBatch([(c[2], c[1]) for c in cases], precision="fp64")
    singles = []
    for i, c in enumerate(cases):
        bt.set_state(i, c[3], c[4], c[5])
        s = Lattice(c[2], c[1], precision="fp64")
        s.set_state(c[3], c[4], c[5])
        s.initialize()
        singles.append(s)
    bt.initialize()
    for _ in range(3):
        bt.evolve(7)
        for s in singles:
            s.evolve(7)
    n_launch = bt.kernel_launches()
    assert n_launch > 0
    for i, s in enumerate(singles):
        fb, pb, sb = bt.get_state(i)
        fs, ps, ss = s.get_state()
        assert rel(fb, fs) < 1e-12 and rel(pb, ps) < 1e-12
        assert abs(sb["aI"] - ss["aI"]) <= 1e-12 * ss["aI"]
        s.close()
    bt.close()


def test_batch_rejects_mixed_members():
    from cosmolattice_b200 import _capi
    from cosmolattice_b200.batch import LatticeBatch

    a = make_scalar_case(N=8, dt=0.01)
    b = make_scalar_case(N=8, dt=0.02)
    with pytest.raises(_capi.ClbError) as e:
        LatticeBatch([(a[2], a[1]), (b[2], b[1])])
    assert e.value.code == _capi.CLB_EINVAL
    c = make_scalar_case(N=8, model="lphi4")
    with pytest.raises(_capi.ClbError) as e:
        LatticeBatch([(c[2], c[1])])
    assert e.value.code == _capi.CLB_EUNSUPPORTED


# members whose N are multiples of 4, so that the vector-site tiles apply too
MEMBERS4 = [(8, 1.0, 1e-3, "a"), (12, 0.5, 1e-2, "b"), (16, 2.0, 3e-3, "c"), (20, 1.3, 1e-4, "d"), (32, 0.8, 5e-3, "e")]


def members4(evolver="VV4", expansion=True, dt=0.01):
    return [make_scalar_case(N=N, evolver=evolver, expansion=expansion, dt=dt, seed=seed, amp=amp,
                             extra={"lambda_prog": lam}) for N, lam, amp, seed in MEMBERS4]


# (tile z sites, tile y, x-planes, z sites per thread)
@pytest.mark.parametrize("tile", [(32, 4, 8, 1), (32, 8, 32, 1), (32, 16, 5, 1), (64, 4, 1024, 1), (32, 4, 1, 1),
                                  (32, 8, 7, 2), (64, 8, 16, 2), (32, 16, 3, 4), (64, 16, 64, 4), (32, 32, 1024, 4)])
def test_every_sweep_configuration_matches_oracle(tile):
    # every block shape kind, with x-runs shorter than, equal to and longer than the members
    cases = members("VV4", True) if tile[3] == 1 else members4()
    out, m0, m1 = run_batch(cases, "fp64", 20, tuning=tile)
    for i, c in enumerate(cases):
        st, o0, o1 = run_oracle(c, 20)
        assert rel(out[i][0], st[0]) < 1e-12 and rel(out[i][1], st[1]) < 1e-12, (tile, i)
        assert abs(m1[i]["aI"] - o1["aI"]) <= 1e-10 * abs(o1["aI"])


def test_autotuner_picks_a_timed_configuration():
    from cosmolattice_b200.batch import LatticeBatch

    cases = members()
    bt = LatticeBatch([(c[2], c[1]) for c in cases], precision="fp32")
    for i, c in enumerate(cases):
        bt.set_state(i, c[3], c[4], c[5])
    bt.initialize()
    assert bt.tuning()["candidates"] == 0
    t = bt.autotune(3)
    print("autotune", t)
    assert t["candidates"] >= 8 and t["ms_per_sweep"] > 0 and t["ms_default"] > 0
    assert t["ms_per_sweep"] <= t["ms_default"]
    assert (t["tile_z"], t["tile_y"], t["sites_per_thread"]) in {(32, 4, 1), (32, 8, 1), (32, 16, 1), (64, 4, 1)}
    assert t["planes_x"] >= 8  # the members' odd N allow one site per thread only
    assert bt.tuning() == t
    f0 = [bt.get_state(i) for i in range(len(cases))]
    bt.evolve(10)
    # the timing sweeps left the state alone: a second handle without tuning runs the same steps
    bt2 = LatticeBatch([(c[2], c[1]) for c in cases], precision="fp32")
    bt2.set_tuning(t["tile_z"], t["tile_y"], t["planes_x"], t["sites_per_thread"])
    f = bt.form()
    if f["persistent"]:  # the autotuner kept the persistent form: the second handle takes it too
        bt2.set_persistent(f["tile_z"], f["tile_y"], f["planes_x"], f["sites_per_thread"])
    for i, c in enumerate(cases):
        bt2.set_state(i, c[3], c[4], c[5])
    bt2.initialize()
    assert all(np.array_equal(a[0], b[0]) for a, b in zip(f0, [bt2.get_state(i) for i in range(len(cases))]))
    bt2.evolve(10)
    for i in range(len(cases)):
        a, b = bt.get_state(i), bt2.get_state(i)
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    with pytest.raises(Exception):
        bt.set_tuning(16, 16, 8)
    with pytest.raises(Exception):
        bt.set_tuning(32, 8, 8, 2)  # N = 13 and 33 are not multiples of 2
    bt.close()
    bt2.close()


def test_fp32_vector_tiles_track_fp64():
    # the FP32 split form with vector sites: every member within the FP32 bounds of its FP64 run
    cases = members4("VV2")
    g32, _, m32 = run_batch(cases, "fp32", 60, tuning=(64, 16, 16, 4))
    g64, _, m64 = run_batch(cases, "fp64", 60, tuning=(32, 8, 32, 1))
    for i in range(len(cases)):
        (fa, pa, sa), (fb, pb, sb) = g32[i], g64[i]
        assert rel(fa, fb) < 1e-6
        assert abs(sa["aI"] - sb["aI"]) / sb["aI"] < 1e-7
        assert abs(m32[i]["friedmann"][0] - m64[i]["friedmann"][0]) < 1e-6


# ---- persistent form: the whole evolve call as one launch of thread-block clusters ----------------
def run_persistent(cases, precision, steps, shape, chunks=1):
    from cosmolattice_b200.batch import LatticeBatch

    bt = LatticeBatch([(c[2], c[1]) for c in cases], precision=precision)
    bt.set_persistent(*shape)
    for i, c in enumerate(cases):
        bt.set_state(i, c[3], c[4], c[5])
    bt.initialize()
    m0 = [bt.measure(i) for i in range(len(cases))]
    form = bt.form()
    launches = []
    for _ in range(chunks):
        l0 = bt.kernel_launches()
        bt.evolve(steps // chunks)
        launches.append(bt.kernel_launches() - l0)
    out = [bt.get_state(i) for i in range(len(cases))]
    m1 = [bt.measure(i, m0[i]["energies"][-1]) for i in range(len(cases))]
    bt.close()
    return out, m0, m1, form, launches


# (tile z sites, tile y, x-planes, z sites per thread): every compiled shape, x-runs shorter than,
# equal to and longer than the members
PERSIST_SHAPES = [(32, 8, 8, 1), (32, 4, 3, 1), (32, 8, 64, 1), (32, 8, 16, 2), (64, 8, 8, 4)]


@pytest.mark.parametrize("shape", PERSIST_SHAPES)
@pytest.mark.parametrize("evolver,expansion", [("VV2", True), ("VV4", True), ("VV2", False)])
def test_persistent_form_matches_oracle_per_member(shape, evolver, expansion):
    # FP64: every member within 1e-12 per site of the oracle run on its own, over two evolve calls
    # (the second starts from the other buffer parity), each call one kernel launch
    cases = members(evolver, expansion) if shape[3] == 1 else members4(evolver, expansion)
    out, m0, m1, form, launches = run_persistent(cases, "fp64", 30, shape, chunks=2)
    assert form["persistent"] == 1 and form["clusters"] == len(cases) and form["cluster_blocks"] == 8
    assert (form["tile_z"], form["tile_y"], form["planes_x"], form["sites_per_thread"]) == shape
    assert launches == [1, 1]
    for i, c in enumerate(cases):
        (fo, po, so), mo0, mo1 = run_oracle(c, 30)
        fg, pg, sg = out[i]
        assert rel(fg, fo) < 1e-12 and rel(pg, po) < 1e-12, (shape, i, rel(fg, fo), rel(pg, po))
        assert abs(sg["aI"] - so["aI"]) <= 1e-10 * so["aI"]
        assert abs(sg["aDotI"] - so["aDotI"]) <= 1e-10 * abs(so["aDotI"]) + 1e-300
        for a, b in zip(m1[i]["energies"], mo1["energies"]):
            assert abs(a - b) <= 1e-10 * abs(b) + 1e-300


def test_persistent_form_many_members_per_cluster():
    # more members than the device holds clusters at once: each cluster takes several members in
    # turn; every member within 1e-12 of the per-stage form (FP64)
    from cosmolattice_b200.batch import LatticeBatch

    rng = np.random.default_rng(3)
    specs = [(int(rng.choice([8, 12, 16, 20])), float(np.exp(rng.uniform(np.log(0.5), np.log(2.0)))),
              float(np.exp(rng.uniform(np.log(1e-4), np.log(1e-2)))), f"m{k}") for k in range(400)]
    cases = [make_scalar_case(N=N, evolver="VV2", expansion=True, dt=0.01, seed=s, amp=a, extra={"lambda_prog": l})
             for N, l, a, s in specs]
    ref, _, _ = run_batch(cases, "fp64", 12, tuning=(32, 8, 32, 1))
    out, _, m1, form, launches = run_persistent(cases, "fp64", 12, (32, 8, 8, 1))
    print("form", form)
    assert form["clusters"] < len(cases) and launches == [1]
    for i in range(len(cases)):
        assert rel(out[i][0], ref[i][0]) < 1e-13 and rel(out[i][1], ref[i][1]) < 1e-13, i
        assert abs(out[i][2]["aI"] - ref[i][2]["aI"]) <= 1e-13 * ref[i][2]["aI"]
    # spot-check members against the oracle
    for i in (0, 199, 399):
        st, _, _ = run_oracle(cases[i], 12)
        assert rel(out[i][0], st[0]) < 1e-12 and rel(out[i][1], st[1]) < 1e-12


def test_persistent_fp32_tracks_fp64():
    # the FP32 split form in the persistent launch: every member within the FP32 bounds of its FP64
    # run, and equal to the per-stage FP32 form up to the order of the volume sums
    cases = members4("VV2")
    g32, _, m32, _, _ = run_persistent(cases, "fp32", 60, (64, 8, 8, 4))
    g64, _, m64 = run_batch(cases, "fp64", 60, tuning=(32, 8, 32, 1))
    s32, _, _ = run_batch(cases, "fp32", 60, tuning=(64, 16, 16, 4))
    for i in range(len(cases)):
        (fa, pa, sa), (fb, pb, sb) = g32[i], g64[i]
        assert rel(fa, fb) < 1e-6
        assert rel(fa - fa.mean(), fb - fb.mean()) < 1e-3
        assert abs(sa["aI"] - sb["aI"]) <= 1e-7 * sb["aI"]
        assert abs(m32[i]["friedmann"][0] - m64[i]["friedmann"][0]) <= 1e-6
        assert rel(fa, s32[i][0]) < 1e-6 and rel(pa, s32[i][1]) < 1e-5


def test_autotuner_times_both_forms_and_leaves_the_state():
    from cosmolattice_b200.batch import LatticeBatch

    cases = members4("VV2")
    bt = LatticeBatch([(c[2], c[1]) for c in cases], precision="fp32")
    for i, c in enumerate(cases):
        bt.set_state(i, c[3], c[4], c[5])
    bt.initialize()
    f0 = [bt.get_state(i) for i in range(len(cases))]
    bt.autotune(2)
    f = bt.form()
    print("form", f)
    assert f["candidates"] >= 4 and f["ms_graph"] > 0 and f["ms_persistent"] > 0
    assert f["persistent"] == (1 if f["ms_persistent"] < f["ms_graph"] else 0)
    f1 = [bt.get_state(i) for i in range(len(cases))]
    for a, b in zip(f0, f1):
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]) and a[2] == b[2]
    l0 = bt.kernel_launches()
    bt.evolve(5)
    # per-stage form: the first half kick (tail, sweep, tail), then a sweep and a tail per step
    assert bt.kernel_launches() - l0 == (1 if f["persistent"] else 3 + 2 * 5)
    bt.close()
