"""Host-side model descriptions in the reference's model API vocabulary.

A model declares its field content, the program-unit rescaling (alpha, fStar, omegaStar), its
potential terms and derivatives, and reads its couplings from the parameter file with the
reference's keys.  ``desc()`` turns it into the C-ABI model descriptor; the per-site potential
itself is compiled into the CUDA library (models/lphi4.h:154-226 restated in
csrc/clb_scalar.cuh), the host copy below serves the homogeneous quantities (pot0, masses)
that the reference computes in AbstractModel::setInitialPotentialAndMassesFromPotential
(abstractmodel.h:220-248).
"""
from __future__ import annotations

import math
from typing import List, Sequence

from . import _capi
from .params import ParameterParser, RunParameters

# Reduced Planck mass in GeV.  TempLat's Constants::reducedMPlanck is not vendored with the
# reference (scalefactorbase.h:18 uses it); this is the standard value, overridable with MPl=.
REDUCED_MPLANCK_GEV = 2.435e18


class CouplingsManager:
    """Effective charges g*Q of matter fields under gauge fields (couplingsmanager.h:29-218).

    ``pattern[m][g]`` says whether matter field m couples to gauge field g.  Charges are consumed
    in order over the coupled pairs (row-major), couplings are picked by gauge index.
    """

    class NotEnoughCharges(ValueError):
        """NotEnoughChargesForThisCouplingsManager"""

    class NotEnoughCouplings(ValueError):
        """NotEnoughCouplingsForThisCouplingsManager"""

    def __init__(self, pattern: Sequence[Sequence[bool]]):
        self.pattern = [list(map(bool, row)) for row in pattern]
        self.n_matter = len(self.pattern)
        self.n_gauge = len(self.pattern[0]) if self.pattern else 0
        self._q = [[0.0] * self.n_gauge for _ in range(self.n_matter)]
        self._g = [0.0] * self.n_gauge

    def couples(self, m: int, g: int) -> bool:
        return self.pattern[m][g]

    def how_many_couples(self) -> int:
        return sum(sum(r) for r in self.pattern)

    def set_effective_charges(self, charges: Sequence[float], couplings: Sequence[float]) -> None:
        if len(charges) != self.how_many_couples():
            raise CouplingsManager.NotEnoughCharges(
                f"{len(charges)} charges for {self.how_many_couples()} coupled pairs")
        if len(couplings) != self.n_gauge:
            raise CouplingsManager.NotEnoughCouplings(f"{len(couplings)} couplings for {self.n_gauge} gauge fields")
        it = iter(charges)
        for m in range(self.n_matter):
            for g in range(self.n_gauge):
                self._q[m][g] = next(it) * couplings[g] if self.pattern[m][g] else 0.0
        self._g = list(couplings)

    def __call__(self, m: int, g: int) -> float:
        return self._q[m][g]

    def coupling(self, g: int) -> float:
        return self._g[g]


class Model:
    """Base of host model descriptions (the reference's AbstractModel, abstractmodel.h:84-318)."""

    name = "model"
    kind = 0
    Ns = 0
    NPotTerms = 1

    def __init__(self, par: ParameterParser, rp: RunParameters):
        self.rp = rp
        self.alpha = 1.0
        self.fStar = 1.0
        self.omegaStar = 1.0
        self.MPl = par.get_float("MPl", REDUCED_MPLANCK_GEV)
        self.dx = rp.dx
        self.kIR = rp.kIR
        self.dt = rp.dt
        self.fldS0: List[float] = [0.0] * self.Ns
        self.piS0: List[float] = [0.0] * self.Ns
        self.masses2S: List[float] = [0.0] * self.Ns
        self.pot0 = 0.0
        # fluctuation amplitude replacing omegaStar/fStar in the initial-spectrum norm
        # (fluctuationsgenerator.h:64); the reference value when not given
        self.fluct_amplitude = None

    # ---- potential API on homogeneous program-unit values (numpy or float) ----
    def potential_terms(self, k: int, phi):
        raise NotImplementedError

    def pot_deriv(self, n: int, phi):
        raise NotImplementedError

    def pot_deriv2(self, n: int, phi):
        raise NotImplementedError

    def potential(self, phi):
        return sum(self.potential_terms(k, phi) for k in range(self.NPotTerms))

    def couplings(self) -> List[float]:
        raise NotImplementedError

    def set_initial_potential_and_masses_from_potential(self) -> None:
        """abstractmodel.h:220-248: pot0 and masses^2 at the homogeneous point phi0 / fStar."""
        phi = [v / self.fStar for v in self.fldS0]
        self.pot0 = self.potential(phi)
        self.masses2S = [self.pot_deriv2(n, phi) for n in range(self.Ns)]

    def desc(self) -> _capi.ModelDesc:
        d = _capi.ModelDesc()
        d.kind = self.kind
        d.n_scalars = self.Ns
        d.alpha = self.alpha
        d.fStar = self.fStar
        d.omegaStar = self.omegaStar
        d.MPl = self.MPl
        c = self.couplings()
        for i, v in enumerate(c):
            d.couplings[i] = v
        return d


class lphi4(Model):
    """models/lphi4.h: two real scalars, V = phi^4/4 + q/2 phi^2 chi^2 in program variables.

    Keys: lambda, q, initial_amplitudes (2 values, GeV), initial_momenta (2 values, GeV^2).
    Rescaling (lphi4.h:125-127): alpha = 1, fStar = phi0, omegaStar = sqrt(lambda) fStar.
    ``lambda_prog`` (default 1) multiplies the quartic term in program units, so a lattice can run
    at a coupling other than the one that fixed omegaStar.
    """

    name = "lphi4"
    kind = _capi.MODEL_LPHI4
    Ns = 2
    NPotTerms = 2

    def __init__(self, par: ParameterParser, rp: RunParameters):
        super().__init__(par, rp)
        self.lam = par.get_float("lambda")
        self.q = par.get_float("q", 0.0) if self.Ns == 2 else 0.0
        self.c0 = par.get_float("lambda_prog", 1.0)
        self.fldS0 = par.get_floats("initial_amplitudes", self.Ns)
        self.piS0 = par.get_floats("initial_momenta", self.Ns, [0.0] * self.Ns)
        self.alpha = 1.0
        self.fStar = self.fldS0[0]
        self.omegaStar = math.sqrt(self.lam) * self.fStar
        if par.has("fluct_amplitude"):
            self.fluct_amplitude = par.get_float("fluct_amplitude")
        self.set_initial_potential_and_masses_from_potential()

    def potential_terms(self, k, phi):
        if k == 0:
            return 0.25 * self.c0 * phi[0] ** 4
        return 0.5 * self.q * (phi[0] * phi[1]) ** 2

    def pot_deriv(self, n, phi):
        if self.Ns == 1:
            return self.c0 * phi[0] ** 3
        if n == 0:
            return self.c0 * phi[0] ** 3 + self.q * phi[0] * phi[1] ** 2
        return self.q * phi[1] * phi[0] ** 2

    def pot_deriv2(self, n, phi):
        if self.Ns == 1:
            return 3 * self.c0 * phi[0] ** 2
        if n == 0:
            return 3 * self.c0 * phi[0] ** 2 + self.q * phi[1] ** 2
        return self.q * phi[0] ** 2

    def couplings(self):
        return [self.c0, self.q]


class lphi4_1f(lphi4):
    """One real scalar with V = lambda_prog/4 phi^4: the reference lphi4 header with its
    daughter field removed (same keys; initial_amplitudes / initial_momenta take one value)."""

    name = "lphi4_1f"
    Ns = 1
    NPotTerms = 1


class tanh2(Model):
    """models/tanh2.h: an inflaton phi with a T-model potential and a daughter field chi,
    V = (M/phi_i)^2 tanh^2(phi phi_i/M) / 2 + q/2 phi^2 chi^2 in program variables.

    Keys: M, Lambda4, q, initial_amplitudes (2 values, GeV), initial_momenta (2 values).
    Rescaling (tanh2.h constructor): alpha = 0, fStar = phi_i = initial_amplitudes[0],
    omegaStar = sqrt(Lambda4 / M^2).  The device kernels take the potential from the tanh2 model
    header (cosmolattice_b200/csrc/models/tanh2.h): the library built with it
    (lib/tanh2/libclb200.so) runs this model, selected by CLB200_SCALAR_MODEL=tanh2.
    """

    name = "tanh2"
    scalar_header = "tanh2"
    kind = _capi.MODEL_LPHI4  # the scalar-singlet kind: the header the library is built with
    Ns = 2
    NPotTerms = 2

    def __init__(self, par: ParameterParser, rp: RunParameters):
        super().__init__(par, rp)
        self.M = par.get_float("M")
        self.Lambda4 = par.get_float("Lambda4")
        self.q = par.get_float("q")
        self.fldS0 = par.get_floats("initial_amplitudes", self.Ns)
        self.piS0 = par.get_floats("initial_momenta", self.Ns, [0.0] * self.Ns)
        phii = self.fldS0[0]
        self.alpha = 0.0
        self.fStar = phii
        self.omegaStar = math.sqrt(self.Lambda4 / self.M ** 2)
        self.mu = self.M / phii
        if par.has("fluct_amplitude"):
            self.fluct_amplitude = par.get_float("fluct_amplitude")
        self.set_initial_potential_and_masses_from_potential()

    def potential_terms(self, k, phi):
        if k == 0:
            return self.mu ** 2 * math.tanh(phi[0] / self.mu) ** 2 / 2
        return 0.5 * self.q * phi[0] ** 2 * phi[1] ** 2

    def pot_deriv(self, n, phi):
        if n == 0:
            x = phi[0] / self.mu
            return 2 * self.mu * math.tanh(x) ** 2 / math.sinh(2 * x) + self.q * phi[0] * phi[1] ** 2
        return self.q * phi[1] * phi[0] ** 2

    def pot_deriv2(self, n, phi):
        if n == 0:
            x = phi[0] / self.mu
            return (4 * (2 - math.cosh(2 * x)) * math.tanh(x) ** 2 / math.sinh(2 * x) ** 2
                    + self.q * phi[1] ** 2)
        return self.q * phi[0] ** 2

    def couplings(self):
        return [self.mu, self.q]


class lphi4U1(Model):
    """models/lphi4U1.h: one complex scalar charged under one U(1), V = |phi|^4 in program variables.

    Keys: lambda, cmplx_field_initial_norm (GeV), cmplx_momentum_initial_norm (GeV^2, default 0),
    gU1s (default 1) and CSU1_charges (default 1) (complexscalarbase.h:71-72), lambda_prog (default
    1, multiplies the quartic term in program units).  Rescaling (lphi4U1.h:95-97): alpha = 1,
    fStar = |phi_0|, omegaStar = sqrt(lambda) |phi_0|.  The homogeneous norm is split equally over
    the two components (lphi4U1.h:75-76).  Components on the device: Re phi, Im phi, A_x, A_y, A_z.
    """

    name = "lphi4U1"
    kind = _capi.MODEL_LPHI4U1
    Ns = 0
    NCs = 1
    NU1 = 1
    NPotTerms = 1
    n_components = 5

    def __init__(self, par: ParameterParser, rp: RunParameters):
        super().__init__(par, rp)
        self.lam = par.get_float("lambda")
        self.c4 = par.get_float("lambda_prog", 1.0)
        n0 = par.get_float("cmplx_field_initial_norm")
        np0 = par.get_float("cmplx_momentum_initial_norm", 0.0)
        self.fldCS0 = [n0 / math.sqrt(2.0), n0 / math.sqrt(2.0)]
        self.piCS0 = [np0 / math.sqrt(2.0), np0 / math.sqrt(2.0)]
        self.cm = CouplingsManager([[True]])
        g = par.get_floats("gU1s", 1, [1.0])
        q = par.get_floats("CSU1_charges", 1, [1.0])
        self.cm.set_effective_charges(q, g)
        self.gQ = self.cm(0, 0)
        self.alpha = 1.0
        self.fStar = n0
        self.omegaStar = math.sqrt(self.lam) * n0
        if par.has("fluct_amplitude"):
            self.fluct_amplitude = par.get_float("fluct_amplitude")
        self.set_initial_potential_and_masses_from_potential()

    def potential_terms(self, k, phi):
        return self.c4 * (phi[0] ** 2 + phi[1] ** 2) ** 2

    def pot_deriv_norm(self, nrm):
        return self.c4 * 4 * nrm ** 3

    def pot_deriv2_norm(self, nrm):
        return self.c4 * 12 * nrm ** 2

    def set_initial_potential_and_masses_from_potential(self) -> None:
        """abstractmodel.h:220-248 with deriv2ComponentFromNorm (potential.h:36-42); a zero
        condensate is evaluated at |phi| = 1e-14 (abstractmodel.h:282)."""
        phi = [v / self.fStar for v in self.fldCS0]
        if phi[0] == 0 and phi[1] == 0:
            phi = [1e-14 * 0.70710678118654752] * 2
        n2 = phi[0] ** 2 + phi[1] ** 2
        n = math.sqrt(n2)
        nd, nd2 = self.pot_deriv_norm(n), self.pot_deriv2_norm(n)
        self.pot0 = self.potential_terms(0, [v / self.fStar for v in self.fldCS0])
        self.masses2CS = [1.0 / n2 * nd2 * c ** 2 + nd / n * (1 - c ** 2 / n2) for c in phi]

    def couplings(self):
        return [self.c4, self.gQ]


def _deriv2_component(nd, nd2, comps, c):
    """deriv2ComponentFromNorm (potential.h:36-42) at a homogeneous point."""
    n2 = sum(v * v for v in comps)
    n = math.sqrt(n2)
    return 1.0 / n2 * nd2 * comps[c] ** 2 + nd / n * (1 - comps[c] ** 2 / n2)


class lphi4SU2U1(Model):
    """models/lphi4SU2U1.h: real scalar S, complex scalar phi (U(1) charge), SU(2) doublet Phi
    (U(1) and SU(2) charges), one U(1) and one SU(2) gauge field.

    V = c4 |Phi|^4 + qG (|Phi| S)^2 + 2 qH (|Phi| |phi|)^2 in program units (lphi4SU2U1.h:147-160;
    c4 = lambda_prog, 1 in the header).  Keys: lambda, qG, qH, initial_amplitudes,
    initial_momenta, cmplx_field_initial_norm, cmplx_momentum_initial_norm,
    SU2Doublet_initial_norm, SU2Doublet_initial_momenta_norm, gU1s, gSU2s, CSU1_charges,
    SU2DoubletU1_charges, SU2DoubletSU2_charges (defaults 1; complexscalarbase.h:71-72,
    su2doubletbase.h:74-80).  Rescaling (lphi4SU2U1.h:118-121): alpha = 1, fStar = |Phi_0|,
    omegaStar = sqrt(lambda) |Phi_0|.  Device components: fields S, phi (2), Phi (4), A (3), SU(2)
    links (3 x 4 quaternion components); momenta S, phi (2), Phi (4), A (3), SU(2) (3 x 3).
    """

    name = "lphi4SU2U1"
    kind = _capi.MODEL_LPHI4SU2U1
    Ns = 1
    NCs = 1
    NU1 = 1
    NSU2Doublet = 1
    NSU2 = 1
    NPotTerms = 3
    n_components = 22
    n_momentum_components = 19

    def __init__(self, par: ParameterParser, rp: RunParameters):
        super().__init__(par, rp)
        self.lam = par.get_float("lambda")
        self.c4 = par.get_float("lambda_prog", 1.0)
        self.qG = par.get_float("qG")
        self.qH = par.get_float("qH")
        self.fldS0 = [par.get_float("initial_amplitudes", 0.0)]
        self.piS0 = [par.get_float("initial_momenta", 0.0)]
        nC = par.get_float("cmplx_field_initial_norm", 0.0)
        npC = par.get_float("cmplx_momentum_initial_norm", 0.0)
        self.fldCS0 = [nC / math.sqrt(2.0)] * 2
        self.piCS0 = [npC / math.sqrt(2.0)] * 2
        nD = par.get_float("SU2Doublet_initial_norm")
        npD = par.get_float("SU2Doublet_initial_momenta_norm", 0.0)
        self.fldD0 = [nD / 2] * 4
        self.piD0 = [npD / 2] * 4
        gU1 = par.get_floats("gU1s", 1, [1.0])
        gSU2 = par.get_floats("gSU2s", 1, [1.0])
        cs_u1 = CouplingsManager([[True]])
        cs_u1.set_effective_charges(par.get_floats("CSU1_charges", 1, [1.0]), gU1)
        d_u1 = CouplingsManager([[True]])
        d_u1.set_effective_charges(par.get_floats("SU2DoubletU1_charges", 1, [1.0]), gU1)
        d_su2 = CouplingsManager([[True]])
        d_su2.set_effective_charges(par.get_floats("SU2DoubletSU2_charges", 1, [1.0]), gSU2)
        self.gQ_C, self.gQ_D, self.gQ_S = cs_u1(0, 0), d_u1(0, 0), d_su2(0, 0)
        # charges: d(gQ)/d(g) of the three effective couplings
        self.Q_C = par.get_floats("CSU1_charges", 1, [1.0])[0]
        self.Q_D = par.get_floats("SU2DoubletU1_charges", 1, [1.0])[0]
        self.Q_S = par.get_floats("SU2DoubletSU2_charges", 1, [1.0])[0]
        self.alpha = 1.0
        self.fStar = nD
        self.omegaStar = math.sqrt(self.lam) * nD
        if par.has("fluct_amplitude"):
            self.fluct_amplitude = par.get_float("fluct_amplitude")
        self.set_initial_potential_and_masses_from_potential()

    def _norms(self, S, C, D):
        return math.sqrt(sum(v * v for v in D)), math.sqrt(sum(v * v for v in C)), S

    def set_initial_potential_and_masses_from_potential(self) -> None:
        """abstractmodel.h:220-248 with the zero-condensate floor 1e-14 (abstractmodel.h:282)."""
        S = self.fldS0[0] / self.fStar
        C = [v / self.fStar for v in self.fldCS0]
        D = [v / self.fStar for v in self.fldD0]
        if C[0] == 0 and C[1] == 0:
            C = [1e-14 * 0.70710678118654752] * 2
        if all(v == 0 for v in D):
            D = [1e-14 / 2] * 4
        nD, nC, _ = self._norms(S, C, D)
        self.pot0 = self.c4 * nD ** 4 + self.qG * (nD * S) ** 2 + 2 * self.qH * (nD * nC) ** 2
        self.masses2S = [2 * self.qG * nD ** 2]
        ndC, nd2C = 4 * self.qH * nD ** 2 * nC, 4 * self.qH
        self.masses2CS = [_deriv2_component(ndC, nd2C, C, c) for c in range(2)]
        ndD = 4 * self.c4 * nD ** 3 + nD * (2 * self.qG * S ** 2 + 4 * self.qH * nC ** 2)
        nd2D = 12 * self.c4 * nD ** 2 + 2 * self.qG * S ** 2 + 4 * self.qH * nC ** 2
        self.masses2D = [_deriv2_component(ndD, nd2D, D, c) for c in range(4)]

    def couplings(self):
        return [self.qG, self.qH, self.gQ_C, self.gQ_D, self.gQ_S, self.c4]


MODELS = {"lphi4": lphi4, "lphi4_1f": lphi4_1f, "lphi4U1": lphi4U1, "lphi4SU2U1": lphi4SU2U1, "tanh2": tanh2}
