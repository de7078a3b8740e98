"""Host-side parameter handling and the couplings manager (no GPU)."""
import math

import pytest

from cosmolattice_b200 import CouplingsManager, ParameterParser, RunParameters
from cosmolattice_b200.params import NotAnEvolverType, RunParametersInconsistent, RunParametersMissing, parse_evolver


def rp_of(**kw):
    base = {"N": 32, "dt": 0.01}
    base.update(kw)
    return RunParameters(ParameterParser(params=base))


def test_lattice_size_from_kir_lside_dx():
    # runparameters.h:155-186: lSide = 2 pi / kIR = N dx
    a = rp_of(kIR=1.0)
    assert math.isclose(a.lSide, 2 * math.pi) and math.isclose(a.dx, 2 * math.pi / 32)
    b = rp_of(lSide=2 * math.pi)
    assert math.isclose(b.kIR, 1.0)
    c = rp_of(dx=2 * math.pi / 32)
    assert math.isclose(c.kIR, 1.0)
    d = rp_of(kIR=1.0, lSide=2 * math.pi, dx=2 * math.pi / 32)
    assert math.isclose(d.dx, a.dx)


def test_lattice_size_errors():
    with pytest.raises(RunParametersMissing):
        rp_of()
    with pytest.raises(RunParametersInconsistent):
        rp_of(kIR=1.0, lSide=3.0)
    with pytest.raises(RunParametersInconsistent):
        rp_of(kIR=1.0, dx=0.5)


def test_run_parameter_checks():
    with pytest.raises(RunParametersInconsistent):
        rp_of(kIR=1.0, dt=0.0)
    with pytest.raises(RunParametersInconsistent):
        rp_of(kIR=1.0, tMax=-1.0)
    with pytest.raises(RunParametersInconsistent):
        rp_of(kIR=1.0, tOutputFreq=0.001)
    with pytest.raises(RunParametersInconsistent):
        rp_of(kIR=1.0, appendToFiles="true", overwriteFiles="true")
    with pytest.raises(RunParametersInconsistent):
        rp_of(kIR=1.0, PS_type=3)


def test_defaults_and_bins():
    r = rp_of(kIR=0.7)
    assert r.nBinsSpectra == math.floor(math.sqrt(3) / 2 * 32)  # runparameters.h:98
    assert r.eType == 0 and r.expansion  # LF and expansion by default
    kUV = math.sqrt(3) * math.pi / r.dx
    assert math.isclose(r.kCutoff, 2 * kUV)  # no cutoff -> 2 kUV (runparameters.h:198-200)


def test_evolver_names_and_numbers():
    # evolvertype.h:37-82: names or integers
    for i, name in enumerate(["LF", "VV2", "VV4", "VV6", "VV8", "VV10", "VV6_2"]):
        assert parse_evolver(name) == i
        assert parse_evolver(str(i)) == i
    with pytest.raises(NotAnEvolverType):
        parse_evolver("RK2")
    with pytest.raises(NotAnEvolverType):
        parse_evolver("banana")


def test_parameter_file_syntax(tmp_path):
    f = tmp_path / "p.in"
    f.write_text("#Lattice\nN = 64\ndt = 0.01 # comment\nkIR = .7\ninitial_amplitudes = 5.6964e18 0  # GeV\n")
    par = ParameterParser(filename=str(f), overrides=["N=32"])
    assert par.get_int("N") == 32
    assert par.get_floats("initial_amplitudes", 2) == [5.6964e18, 0.0]
    assert math.isclose(par.get_float("kIR"), 0.7)


def test_couplings_manager_golden():
    # Golden values of the reference's only numeric test, tests/CosmoInterface/couplingsmanager.cpp:18-64:
    # CouplingsManager<2, 4, true, false, true, false, true, true, true, false>
    cm = CouplingsManager([[True, False, True, False], [True, True, True, False]])
    assert cm.couples(0, 0) and not cm.couples(0, 1) and cm.couples(0, 2) and not cm.couples(0, 3)
    assert cm.couples(1, 0) and cm.couples(1, 1) and cm.couples(1, 2) and not cm.couples(1, 3)
    assert cm.how_many_couples() == 5
    cm.set_effective_charges([1, 2, 3, 4, 5], [1, 2, 3, 4])
    assert cm(0, 0) == 1
    assert cm(0, 2) == 6
    assert cm(1, 0) == 3
    assert cm(1, 1) == 8
    assert cm(1, 2) == 15
    assert cm(0, 1) == 0 and cm(1, 3) == 0
    assert cm.coupling(0) == 1 and cm.coupling(3) == 4
    with pytest.raises(CouplingsManager.NotEnoughCharges):
        cm.set_effective_charges([1, 1, 2, 3, 4, 5], [1, 2, 3, 4])
    with pytest.raises(CouplingsManager.NotEnoughCouplings):
        cm.set_effective_charges([1, 2, 3, 4, 5], [1, 3, 4])


def test_output_cadence_rounds_halves_away_from_zero():
    """measurer.h:48-53 counts output steps with C's round(): 2.5 steps -> 3, not Python's 2."""
    from cosmolattice_b200.lattice import c_round

    assert [c_round(x) for x in (2.5, 3.5, 0.5, 2.49, 10.000000000000002, -2.5)] == [3, 4, 1, 2, 10, -3]
    assert round(2.5) == 2  # the rounding this replaces


def test_restart_file_round_trip(tmp_path):
    # save_sim / load_sim over a stand-in lattice (no GPU): every array, the six scale-factor
    # values and the time come back bitwise, in the reference's sector order, and a file of
    # another model or size is refused
    import numpy as np

    from conftest import make_su2_case
    from cosmolattice_b200 import restart

    par, rp, m, f, p, sf = make_su2_case(N=4)
    sf = dict(sf, aDotSIM=0.25)

    class Stand:
        def __init__(self):
            self.rp = rp
            self.state = None
            self.mode = None

        def get_state(self):
            return f.ravel(), p.ravel(), dict(sf)

        def set_state(self, F, P, s):
            self.state = (F.copy(), P.copy(), dict(s))

        def initialize(self, restart=False):
            self.mode = restart

    path = str(tmp_path / "run.clb")
    restart.save_sim(path, Stand(), m, 1.5, {"N": 4, "dt": 0.005})
    st = Stand()
    t, text = restart.load_sim(path, st, m)
    F, P, s = st.state
    assert t == 1.5 and "dt = 0.005" in text and st.mode is True
    assert np.array_equal(F.ravel(), f.ravel()) and np.array_equal(P.ravel(), p.ravel())
    assert all(s[k] == sf[k] for k in restart.SCALARS)
    # sector order on disk: S field, S momentum, phi fields, phi momenta, ...
    raw = np.fromfile(path, dtype="<f8", offset=80, count=2 * 64)
    assert np.array_equal(raw[:64], f.reshape(22, -1)[0]) and np.array_equal(raw[64:], p.reshape(19, -1)[0])
    par2, rp2, m2, *_ = make_su2_case(N=6)
    st2 = Stand()
    st2.rp = rp2
    with pytest.raises(ValueError):
        restart.load_sim(path, st2, m2)


def test_gw_parameters():
    # withGWs, doLFforGWs and GWprojectorType (runparameters.h:120-123): the GWs run as the
    # reference's default leapfrog over the matter evolver
    base = {"N": 8, "kIR": 1.0, "dt": 0.01, "withGWs": "true"}
    rp = RunParameters(ParameterParser(params=base))
    assert rp.withGWs and rp.doLFforGWs and rp.GWprojectorType == 2
    with pytest.raises(RunParametersInconsistent):
        RunParameters(ParameterParser(params=dict(base, doLFforGWs="false")))
    with pytest.raises(RunParametersInconsistent):
        RunParameters(ParameterParser(params=dict(base, GWprojectorType=4)))


def test_restart_file_carries_the_gws(tmp_path):
    # with GWs the five field/momentum pairs sit right after the scalar singlets (for lphi4SU2U1,
    # after S; simulationmanager.h:112-114) and come back bitwise; a lattice without GWs steps
    # over them
    import numpy as np

    from conftest import make_su2_case
    from cosmolattice_b200 import restart

    par, rp, m, f, p, sf = make_su2_case(N=4)
    sf = dict(sf, aDotSIM=0.25)
    n3 = rp.N ** 3
    rng = np.random.default_rng(3)
    gu, gp = rng.standard_normal(5 * n3), rng.standard_normal(5 * n3)

    class Stand:
        def __init__(self, gws):
            self.rp = rp
            self.gws_on = gws
            self.state = self.gw = None

        def get_state(self):
            return f.ravel(), p.ravel(), dict(sf)

        def gws_get_state(self):
            return gu, gp

        def set_state(self, F, P, s):
            self.state = (F.copy(), P.copy(), dict(s))

        def gws_set_state(self, u, pi):
            self.gw = (u.copy(), pi.copy())

        def initialize(self, restart=False):
            pass

    path = str(tmp_path / "gw.clb")
    restart.save_sim(path, Stand(True), m, 2.0)
    raw = np.fromfile(path, dtype="<f8", count=(16 + 64) // 8 + 2 * n3 + 10 * n3)
    body = raw[(16 + 64) // 8:]
    F, P = f.reshape(22, n3), p.reshape(19, n3)
    assert np.array_equal(body[:n3], F[0]) and np.array_equal(body[n3:2 * n3], P[0])  # S, pi_S
    pairs = body[2 * n3:].reshape(5, 2, n3)
    assert np.array_equal(pairs[:, 0].ravel(), gu) and np.array_equal(pairs[:, 1].ravel(), gp)
    st = Stand(True)
    t, _ = restart.load_sim(path, st, m)
    assert t == 2.0 and np.array_equal(st.gw[0], gu) and np.array_equal(st.gw[1], gp)
    assert np.array_equal(st.state[0], F) and np.array_equal(st.state[1], P)
    plain = Stand(False)
    restart.load_sim(path, plain, m)
    assert plain.gw is None and np.array_equal(plain.state[0], F) and np.array_equal(plain.state[1], P)
    path2 = str(tmp_path / "nogw.clb")
    restart.save_sim(path2, Stand(False), m, 2.0)
    with pytest.raises(ValueError):
        restart.load_sim(path2, Stand(True), m)
