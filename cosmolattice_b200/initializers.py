"""Initial conditions for scalar singlets and the scale factor (host, numpy FFT).

Restates the reference recipe:
* ScaleFactorInitializer::initializeScaleFactor (initializers/scalefactorinitializer.h:30-65):
  a = a0, aDot = (fStar / MPl) sqrt(rho / 3) with rho from the homogeneous kinetic energy and pot0.
* FluctuationsGenerator::getFluctuationsNorm / conjugateGaussianFluctuations
  (initializers/fluctuationsgenerator.h:39-71, 130-150): per mode, left and right movers f_L, f_R
  with Gaussian real and imaginary parts of rms
      H(kCut - k) (omega*/f*) (L/dx^2)^(3/2) (2 omega_k)^(-1/2) / sqrt(2),
  omega_k = sqrt(k^2 + max(m^2, 0)); phi_k = (f_L + f_R)/sqrt(2),
  pi_k = i omega_k (f_L - f_R)/sqrt(2) - aDot phi_k; zero modes set to 0.
* ScalarSingletInitializer::initializeScalars (scalarsingletinitializer.h:41-77): homogeneous
  phi0/f* and pi0/(f* omega*) added afterwards.

The random streams are numpy PCG64 streams seeded from (baseSeed, label, field); the reference's
TempLat streams are not reproducible outside TempLat.  The configuration-space field is the
normalised inverse real FFT (scipy.fft.irfftn, 1/N^3), consistent with the norm above giving the
continuum vacuum variance.  ``fluct_amplitude`` (a model parameter) replaces omega*/f* when set.
"""
from __future__ import annotations

import hashlib
import math

import numpy as np
import scipy.fft as sfft

from .models import Model
from .params import RunParameters


def _rng(base_seed: str, label: str) -> np.random.Generator:
    h = hashlib.sha256(f"{base_seed}|{label}".encode()).digest()
    return np.random.Generator(np.random.PCG64(int.from_bytes(h[:16], "little")))


def wave_numbers(N: int):
    """Integer lattice wave numbers of the rfftn half spectrum, shape (N, N, N//2+1)."""
    nx = np.fft.fftfreq(N, 1.0 / N)
    nz = np.fft.rfftfreq(N, 1.0 / N)
    return nx[:, None, None], nx[None, :, None], nz[None, None, :]


def initial_scale_factor(model: Model, rp: RunParameters):
    """(aI, aDotI) before fluctuations (scalefactorinitializer.h:37-65); a fixed background starts
    at a = 1, aDot = H0 (in program units)."""
    if not rp.expansion:
        return 1.0, 0.0
    if getattr(rp, "fixedBackground", False):
        return 1.0, rp.H0 / model.omegaStar
    kin = 0.0
    for i in range(model.Ns):
        # Energies::kineticS with the default a = 1 in force at that point
        kin += 0.5 * (model.piS0[i] / model.fStar / model.omegaStar) ** 2
    for c in getattr(model, "piCS0", []) if getattr(model, "NCs", 0) else []:
        # Energies::kineticCS: |pi|^2 with no 1/2 (energies.h:47-50)
        kin += (c / model.fStar / model.omegaStar) ** 2
    for c in getattr(model, "piD0", []):
        # Energies::kineticSU2Doublet: |pi|^2 with no 1/2 (energies.h:57-60)
        kin += (c / model.fStar / model.omegaStar) ** 2
    rho = kin + model.pot0
    return rp.a0, model.fStar / model.MPl * math.sqrt(rho / 3.0)


def scalar_fluctuations(model: Model, rp: RunParameters, field: int, aDot: float, dtype=np.float64):
    """phi and pi fluctuations of scalar ``field`` in configuration space (no homogeneous part)."""
    N = rp.N
    nx, ny, nz = wave_numbers(N)
    k = np.sqrt(nx * nx + ny * ny + nz * nz) * rp.kIR
    m2 = model.masses2S[field]
    omega = np.sqrt(k * k + (m2 if m2 > 0 else 0.0))
    amp = model.omegaStar / model.fStar if model.fluct_amplitude is None else model.fluct_amplitude
    with np.errstate(divide="ignore", invalid="ignore"):
        norm = np.where(k <= rp.kCutoff, amp * (rp.lSide / rp.dx ** 2) ** 1.5 * (2 * omega) ** -0.5 / math.sqrt(2.0), 0.0)
    norm[0, 0, 0] = 0.0
    shape = norm.shape
    name = f"scalar_{field}"

    def gauss(label):
        g = _rng(rp.baseSeed, f"{label}{name}")
        return g.standard_normal(shape) + 1j * g.standard_normal(shape)

    fL = norm * gauss("Random left")
    fR = norm * gauss("Random right")
    phik = (fL + fR) / math.sqrt(2.0)
    phik[0, 0, 0] = 0.0
    pik = 1j * omega * (fL - fR) / math.sqrt(2.0) - aDot * phik
    pik[0, 0, 0] = 0.0
    phi = sfft.irfftn(phik, s=(N, N, N), axes=(0, 1, 2), workers=-1)
    pi = sfft.irfftn(pik, s=(N, N, N), axes=(0, 1, 2), workers=-1)
    return phi.astype(dtype, copy=False), pi.astype(dtype, copy=False)


def scalar_initial_state(model: Model, rp: RunParameters):
    """Field and momentum arrays (Ns x N^3 each, float64) and the initial (aI, aDotI)."""
    aI, aDot = initial_scale_factor(model, rp)
    N = rp.N
    fields = np.empty((model.Ns, N, N, N), dtype=np.float64)
    momenta = np.empty_like(fields)
    for f in range(model.Ns):
        phi, pi = scalar_fluctuations(model, rp, f, aDot)
        fields[f] = phi + model.fldS0[f] / model.fStar
        momenta[f] = pi + model.piS0[f] / model.fStar / model.omegaStar
    return fields, momenta, aI, aDot


def _fluct_norm(model: Model, rp: RunParameters, k, m2):
    """FluctuationsGenerator::getFluctuationsNorm in 3-D (fluctuationsgenerator.h:39-65)."""
    omega = np.sqrt(k * k + (m2 if m2 > 0 else 0.0))
    amp = model.omegaStar / model.fStar if model.fluct_amplitude is None else model.fluct_amplitude
    with np.errstate(divide="ignore", invalid="ignore"):
        norm = np.where(k <= rp.kCutoff, amp * (rp.lSide / rp.dx ** 2) ** 1.5 * (2 * omega) ** -0.5 / math.sqrt(2.0), 0.0)
    norm[0, 0, 0] = 0.0
    return norm, omega


def _homogeneous_adot_tangent(model: Model, rp: RunParameters, param: str) -> float:
    """d aDot / d param of initial_scale_factor (only pot0 = c4 |phi_0/f*|^4 depends on c4)."""
    if not rp.expansion or param != "c4":
        return 0.0
    aI, aDot = initial_scale_factor(model, rp)
    if aDot == 0.0:
        return 0.0
    rho3 = (aDot * model.MPl / model.fStar) ** 2  # rho / 3
    return model.fStar / model.MPl * 0.5 / math.sqrt(rho3) * (model.pot0 / model.c4) / 3.0


def complex_scalar_fluctuations(model: Model, rp: RunParameters, aDot: float, tangent: str = None,
                                daDot: float = 0.0):
    """U1Initializer::addFluctuationsCScalarFromPhases (u1initializer.h:157-230): per component
    Rayleigh amplitudes a_c, three uniform phases and the fourth fixed by
    e11 = e01 e10 conj(e00) so the initial charge density follows from the amplitudes; modes
    phi_c = a_c (e_c0 + e_c1)/2, pi_c = -i omega a_c (e_c0 - e_c1)/2 - aDot phi_c, zero modes 0.

    With ``tangent`` ("amp" or "c4") the same draws give d phi_c, d pi_c with respect to the
    fluctuation amplitude or the quartic coupling (through m^2 = masses2CS and aDot)."""
    N = rp.N
    nx, ny, nz = wave_numbers(N)
    k = np.sqrt(nx * nx + ny * ny + nz * nz) * rp.kIR
    out_f, out_p = [], []
    norms = [_fluct_norm(model, rp, k, model.masses2CS[c]) for c in range(2)]
    omega0 = norms[0][1]
    shape = norms[0][0].shape

    def rayleigh(label):
        g = _rng(rp.baseSeed, label)
        return np.sqrt(-2.0 * np.log1p(-g.random(shape)))

    def phase(label):
        g = _rng(rp.baseSeed, label)
        return np.exp(2j * np.pi * g.random(shape))

    amp = model.omegaStar / model.fStar if model.fluct_amplitude is None else model.fluct_amplitude
    m2 = model.masses2CS[0]
    domega0 = np.zeros_like(omega0)
    if tangent == "c4" and m2 > 0:
        with np.errstate(divide="ignore", invalid="ignore"):
            domega0 = np.where(omega0 > 0, (m2 / model.c4) / (2 * omega0), 0.0)
    e00, e01, e10 = phase("phase00cmplx_0_0"), phase("phase01cmplx_0_0"), phase("phase10cmplx_0_1")
    e11 = e01 * e10 * np.conj(e00)
    for c, (ea, eb) in enumerate(((e00, e01), (e10, e11))):
        norm, om = norms[c]
        a = norm * rayleigh(f"norm{c}cmplx_0_{c}")
        fk = a * (ea + eb) / 2.0
        fk[0, 0, 0] = 0.0
        if tangent is None:
            pk = -1j * omega0 * a * (ea - eb) / 2.0 - aDot * fk
        else:
            if tangent == "amp":
                da = a / amp
            elif tangent == "c4" and model.masses2CS[c] > 0:
                with np.errstate(divide="ignore", invalid="ignore"):
                    dom = np.where(om > 0, (model.masses2CS[c] / model.c4) / (2 * om), 0.0)
                    da = np.where(om > 0, -0.5 * a * dom / om, 0.0)
            else:
                da = np.zeros_like(a)
            dfk = da * (ea + eb) / 2.0
            dfk[0, 0, 0] = 0.0
            pk = -1j * (domega0 * a + omega0 * da) * (ea - eb) / 2.0 - daDot * fk - aDot * dfk
            fk = dfk
        pk[0, 0, 0] = 0.0
        out_f.append(sfft.irfftn(fk, s=(N, N, N), axes=(0, 1, 2), workers=-1))
        out_p.append(sfft.irfftn(pk, s=(N, N, N), axes=(0, 1, 2), workers=-1))
    return out_f, out_p


def gauss_solve_u1(rp: RunParameters, rho):
    """pi_i(k) = conj(1 - e^{-2 pi i n_i/N}) / sum_j |1 - e^{-2 pi i n_j/N}|^2 j0(k), j0 = -dx^2 rho,
    zero mode 0 (u1initializer.h:90-114)."""
    N = rp.N
    j0 = sfft.rfftn(-rp.dx ** 2 * rho, axes=(0, 1, 2), workers=-1)
    nx, ny, nz = wave_numbers(N)
    keff = [1.0 - np.exp(-2j * np.pi * n / N) for n in (nx, ny, nz)]
    k2 = sum(np.abs(q) ** 2 for q in keff)
    k2 = np.broadcast_to(k2, j0.shape).copy()
    k2[0, 0, 0] = 1.0
    out = []
    for q in keff:
        pk = np.conj(q) / k2 * j0
        pk[0, 0, 0] = 0.0
        out.append(sfft.irfftn(pk, s=(N, N, N), axes=(0, 1, 2), workers=-1))
    return out


def charge_density_u1(model: Model, rp: RunParameters, phi, pi, gQ=None):
    """rho = 2/dx (fStar/omegaStar)^2 gQ Im(conj(pi_phi) phi) (mattercurrents.h:27-48)."""
    g = model.gQ if gQ is None else gQ
    return 2.0 / rp.dx * (model.fStar / model.omegaStar) ** 2 * g * (pi[0] * phi[1] - pi[1] * phi[0])


def gauss_momenta_u1(model: Model, rp: RunParameters, phi, pi):
    """pi_A from the Gauss constraint in momentum space with A = 0 (u1initializer.h:90-114)."""
    return gauss_solve_u1(rp, charge_density_u1(model, rp, phi, pi))


def u1_initial_state(model: Model, rp: RunParameters):
    """lphi4U1 state (5 x N^3 fields and momenta: Re phi, Im phi, A_x, A_y, A_z) by the
    RandomWithMatter recipe (u1initializer.h:77-117) and the initial (aI, aDotI)."""
    aI, aDot = initial_scale_factor(model, rp)
    N = rp.N
    fields = np.zeros((5, N, N, N), dtype=np.float64)
    momenta = np.zeros_like(fields)
    fl, pl = complex_scalar_fluctuations(model, rp, aDot)
    for c in range(2):
        fields[c] = fl[c] + model.fldCS0[c] / model.fStar
        momenta[c] = pl[c] + model.piCS0[c] / model.fStar / model.omegaStar
    pa = gauss_momenta_u1(model, rp, fields[:2], momenta[:2])
    for i in range(3):
        momenta[2 + i] = pa[i]
    return fields, momenta, aI, aDot


def doublet_fluctuations(model: Model, rp: RunParameters, aDot: float):
    """SU2Initializer::addFluctuationsSU2DoubletFromPhases (su2initializer.h:115-186): per component
    Rayleigh amplitudes a_c and left phases l_c, one right phase r_0 and r_c = r_0 l_c conj(l_0);
    Phi_c = a_c (l_c + r_c)/2, pi_c = -i omega_0 a_c (l_c - r_c)/2 - aDot Phi_c / sqrt(2) (the
    reference's extra 1/sqrt(2) on the aDot term is kept), zero modes 0."""
    N = rp.N
    nx, ny, nz = wave_numbers(N)
    k = np.sqrt(nx * nx + ny * ny + nz * nz) * rp.kIR
    norms = [_fluct_norm(model, rp, k, model.masses2D[c]) for c in range(4)]
    omega0 = norms[0][1]
    shape = norms[0][0].shape

    def rayleigh(label):
        g = _rng(rp.baseSeed, label)
        return np.sqrt(-2.0 * np.log1p(-g.random(shape)))

    def phase(label):
        g = _rng(rp.baseSeed, label)
        return np.exp(2j * np.pi * g.random(shape))

    amps = [norms[c][0] * rayleigh(f"normSU2Doublet_0_{c}") for c in range(4)]
    left = [phase(f"phaseLeftSU2Doublet_0_{c}") for c in range(4)]
    r0 = phase("phaseRightSU2Doublet_0_0")
    right = [r0 * left[c] * np.conj(left[0]) for c in range(4)]
    out_f, out_p = [], []
    for c in range(4):
        fk = amps[c] * (left[c] + right[c]) / 2.0
        fk[0, 0, 0] = 0.0
        pk = -1j * omega0 * amps[c] * (left[c] - right[c]) / 2.0 - aDot * fk / math.sqrt(2.0)
        pk[0, 0, 0] = 0.0
        out_f.append(sfft.irfftn(fk, s=(N, N, N), axes=(0, 1, 2), workers=-1))
        out_p.append(sfft.irfftn(pk, s=(N, N, N), axes=(0, 1, 2), workers=-1))
    return out_f, out_p


def su2u1_initial_state(model: Model, rp: RunParameters):
    """lphi4SU2U1 state: ModelInitializer order (modelinitializer.h:51-66) - scale factor, scalar
    singlet, SU(2) doublet with pi_SU2 from the SU(2) Gauss law and unit links
    (su2initializer.h:39-88), complex scalar with pi_A from the U(1) Gauss law whose charge
    includes the doublet (u1initializer.h:77-117, mattercurrents.h:27-48)."""
    aI, aDot = initial_scale_factor(model, rp)
    N = rp.N
    fields = np.zeros((22, N, N, N))
    momenta = np.zeros((19, N, N, N))
    phi, pi = scalar_fluctuations(model, rp, 0, aDot)
    fields[0] = phi + model.fldS0[0] / model.fStar
    momenta[0] = pi + model.piS0[0] / model.fStar / model.omegaStar
    fl, pl = doublet_fluctuations(model, rp, aDot)
    for c in range(4):
        fields[3 + c] = fl[c] + model.fldD0[c] / model.fStar
        momenta[3 + c] = pl[c] + model.piD0[c] / model.fStar / model.omegaStar
    # SU(2) charge density rho_b = (fStar/omegaStar)^2 / 2 g Re((i s_b Phi)^+ pi_Phi)
    u = fields[3] + 1j * fields[4]
    v = fields[5] + 1j * fields[6]
    pu = momenta[3] + 1j * momenta[4]
    pv = momenta[5] + 1j * momenta[6]
    isig = [(1j * v, 1j * u), (v, -u), (1j * u, -1j * v)]
    r2 = (model.fStar / model.omegaStar) ** 2
    for b in range(3):
        a, c = isig[b]
        rho = r2 / 2 * (model.gQ_S * np.real(np.conj(a) * pu + np.conj(c) * pv))
        pa = gauss_solve_u1(rp, rho / rp.dx)  # j0 = -dx rho (gauss_solve_u1 applies -dx^2)
        for i in range(3):
            momenta[10 + 3 * i + b] = pa[i]
    for i in range(3):
        fields[10 + 4 * i] = 1.0
    fl, pl = complex_scalar_fluctuations(model, rp, aDot)
    for c in range(2):
        fields[1 + c] = fl[c] + model.fldCS0[c] / model.fStar
        momenta[1 + c] = pl[c] + model.piCS0[c] / model.fStar / model.omegaStar
    rho = 2.0 / rp.dx * r2 * (model.gQ_C * (momenta[1] * fields[2] - momenta[2] * fields[1])
                              + model.gQ_D * np.imag(np.conj(pu) * u + np.conj(pv) * v))
    pa = gauss_solve_u1(rp, rho)
    for i in range(3):
        momenta[7 + i] = pa[i]
    return fields, momenta, aI, aDot


def su2u1_initial_state_tangent(model: Model, rp: RunParameters, param: str, state=None):
    """(fields_dot, momenta_dot, couplings_dot) of su2u1_initial_state along param: "gSU2" (the
    SU(2) coupling: only the SU(2) momenta, solved from the doublet charge, depend on it) or "gU1"
    (the U(1) coupling: only the U(1) momenta).  Both enter linearly through the Gauss solves.
    state: (fields, momenta) of su2u1_initial_state, if already made."""
    fields, momenta = state if state is not None else su2u1_initial_state(model, rp)[:2]
    df = np.zeros_like(fields)
    dp = np.zeros_like(momenta)
    cd = np.zeros(6)
    r2 = (model.fStar / model.omegaStar) ** 2
    u = fields[3] + 1j * fields[4]
    v = fields[5] + 1j * fields[6]
    pu = momenta[3] + 1j * momenta[4]
    pv = momenta[5] + 1j * momenta[6]
    if param == "gSU2":
        cd[4] = model.Q_S
        isig = [(1j * v, 1j * u), (v, -u), (1j * u, -1j * v)]
        for b in range(3):
            a, c = isig[b]
            rho = r2 / 2 * (model.Q_S * np.real(np.conj(a) * pu + np.conj(c) * pv))
            pa = gauss_solve_u1(rp, rho / rp.dx)
            for i in range(3):
                dp[10 + 3 * i + b] = pa[i]
    elif param == "gU1":
        cd[2], cd[3] = model.Q_C, model.Q_D
        rho = 2.0 / rp.dx * r2 * (model.Q_C * (momenta[1] * fields[2] - momenta[2] * fields[1])
                                  + model.Q_D * np.imag(np.conj(pu) * u + np.conj(pv) * v))
        pa = gauss_solve_u1(rp, rho)
        for i in range(3):
            dp[7 + i] = pa[i]
    else:
        raise ValueError(f"unknown parameter {param!r}")
    return df, dp, cd


def initial_state(model: Model, rp: RunParameters):
    """Initial state of any supported model (ModelInitializer::initialize, modelinitializer.h:47-81)."""
    if getattr(model, "NSU2", 0):
        return su2u1_initial_state(model, rp)
    if getattr(model, "NU1", 0):
        return u1_initial_state(model, rp)
    return scalar_initial_state(model, rp)


def u1_initial_state_tangent(model: Model, rp: RunParameters, param: str, state=None):
    """d(fields, momenta)/d param of u1_initial_state for param in ("amp", "c4", "gQ"): the
    fluctuation amplitude, the quartic coupling (lambda_prog) and the gauge coupling g Q.
    state: (fields, momenta, aI, aDot) of u1_initial_state, if already made."""
    fields, momenta, aI, aDot = state if state is not None else u1_initial_state(model, rp)
    N = rp.N
    df = np.zeros_like(fields)
    dp = np.zeros_like(momenta)
    if param in ("amp", "c4"):
        fl, pl = complex_scalar_fluctuations(model, rp, aDot, tangent=param,
                                             daDot=_homogeneous_adot_tangent(model, rp, param))
        for c in range(2):
            df[c] = fl[c]
            dp[c] = pl[c]
        drho = 2.0 / rp.dx * (model.fStar / model.omegaStar) ** 2 * model.gQ * (
            dp[0] * fields[1] + momenta[0] * df[1] - dp[1] * fields[0] - momenta[1] * df[0])
        pa = gauss_solve_u1(rp, drho)
    elif param == "gQ":
        pa = gauss_solve_u1(rp, charge_density_u1(model, rp, fields[:2], momenta[:2], gQ=1.0))
    else:
        raise ValueError(f"unknown parameter {param!r}")
    for i in range(3):
        dp[2 + i] = pa[i]
    return df, dp


def device_ic_params(model: Model, rp: RunParameters, seed: int = None) -> dict:
    """clb_ic_params for model (matter components in the model's field order) and the initial
    (aI, aDotI) of initial_scale_factor, as ({...}, aI, aDot).  seed defaults to 64 bits of
    sha256(baseSeed)."""
    aI, aDot = initial_scale_factor(model, rp)
    if seed is None:
        seed = int.from_bytes(hashlib.sha256(f"{rp.baseSeed}|device".encode()).digest()[:8], "little")
    fs, ws = model.fStar, model.omegaStar
    amp = ws / fs if model.fluct_amplitude is None else model.fluct_amplitude
    if getattr(model, "NSU2", 0):
        m2 = [model.masses2S[0]] + list(model.masses2CS[:2]) + list(model.masses2D[:4])
        f0 = [model.fldS0[0] / fs] + [c / fs for c in model.fldCS0[:2]] + [c / fs for c in model.fldD0[:4]]
        p0 = [model.piS0[0] / fs / ws] + [c / fs / ws for c in model.piCS0[:2]] + [c / fs / ws for c in model.piD0[:4]]
        charge = [model.gQ_S, model.gQ_C, model.gQ_D, 0.0]
    elif getattr(model, "NU1", 0):
        m2 = list(model.masses2CS[:2])
        f0 = [c / fs for c in model.fldCS0[:2]]
        p0 = [c / fs / ws for c in model.piCS0[:2]]
        charge = [model.gQ, 0.0, 0.0, 0.0]
    else:
        m2 = list(model.masses2S)
        f0 = [v / fs for v in model.fldS0]
        p0 = [v / fs / ws for v in model.piS0]
        charge = [0.0] * 4
    return ({"seed": int(seed), "amplitude": amp, "k_cutoff": rp.kCutoff, "adot": aDot,
             "mass2": m2, "fld0": f0, "pi0": p0, "charge": charge}, aI, aDot)


def device_initial_state(lattice, model: Model, rp: RunParameters, seed: int = None) -> dict:
    """Generate the initial state on the device (clb_generate_state) into lattice; returns the
    parameters used (device_ic_params) with aI and aDotI added."""
    p, aI, aDot = device_ic_params(model, rp, seed)
    lattice.generate_state(p, {"aI": aI, "aSI": aI, "aIM": aI, "aDotI": aDot, "aDotSI": aDot})
    p.update(aI=aI, aDotI=aDot)
    return p
