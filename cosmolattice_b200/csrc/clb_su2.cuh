// clb_su2.cuh - sm_100a kernels of lphi4SU2U1: real scalar S, complex scalar phi, SU(2) doublet
// Phi, one U(1) and one SU(2) gauge field (models/lphi4SU2U1.h).
//
// Restates, in the reference's operation order (this unit is compiled without FMA contraction so
// plain expressions round where the reference's expression templates round):
//   ScalarSingletKernels::get     evolvers/kernels/scalarsingletkernels.h:30-40
//   ComplexScalarKernels::get     evolvers/kernels/complexscalarkernels.h:28-35
//   SU2DoubletKernels::get        evolvers/kernels/su2doubletkernels.h:28-33
//   U1Kernels::get                evolvers/kernels/u1kernels.h:31-52
//   SU2Kernels::get               evolvers/kernels/su2kernels.h:30-54
//   covariant Laplacians, links   definitions/gaugederivatives.h:48-115
//   currents, charge densities    definitions/mattercurrents.h:27-119
//   averages                      definitions/fieldfunctionals.h:52-223
//   Gauss laws                    definitions/gausslaws.h:34-80
//   energies, scale factor        definitions/energies.h:37-239, scalefactorkernels.h:27-80
// SU(2) representation: a link is a unit quaternion (q0, q) = q0 + i q.sigma; an algebra element
// (pi_1, pi_2, pi_3) = i pi_a sigma_a; exp(i p.sigma) = cos|p| + i sin|p| p/|p|; plaq(U, i, j) =
// U_i(x) U_j(x+i) U_i(x+j)^+ U_j(x)^+; plaqBack(U, i, j) = [U_i(x) U_j(x+i-j)^+ U_i(x-j)^+ U_j(x-j)]^+,
// so sum_j (plaq - plaqBack) is the force of the Wilson term of fieldfunctionals.h:201-209; a
// doublet is (Phi_0 + i Phi_1, Phi_2 + i Phi_3) and scalar_prod(A, B) = A^+ B.
//
// Layout: 22 field and 19 momentum arrays of N^3 sites (x slowest), FP64 or FP32 (FP32 links are
// re-unitarised every few steps by the host schedule; all volume sums stay FP64).  Fields: S | phi (2) |
// Phi (4) | A_x..A_z | links U_i (4 each, i = x, y, z).  Momenta: S | phi (2) | Phi (4) | A (3) |
// pi_SU2 (3 per direction).

#pragma once

#include "clb_internal.cuh"
#include "clb_scalar.cuh"
#include "clb_tangent.cuh"

namespace clb {
namespace su2d {

constexpr int NF = 22, NP = 19;
constexpr int kRed = 16;  // kick-sweep partial slots
constexpr int kMeas = 64; // measurement partial slots

struct Params {
  int N;
  size_t n3;
  double dx, dx2, inv_dx2, inv_dx;
  double qG, qH, gC, gD, gS, c4;
  double rfo2, rof2; // (fStar/omegaStar)^2 and its inverse
  double alpha, fm2, dt, inv_n3;
  int order; // site order of the kick sweeps (for_sites)
};

// Scale factor, the cached averages of the five sectors (S, phi, Phi, A, SU(2)) and the sweep
// coefficients derived from a and aS; T = double, or Tan<double> in the tangent-linear form.
template <class T> struct StateT {
  T aI, aSI, aIM, aDotI, aDotSI, aDotSIM;
  T pi2[5], pi2SI[5], pi2SIM[5];
  T g2S, g2C, g2D, b2A, b2G, potI;
  T g2S_SI, g2C_SI, g2D_SI, b2A_SI, b2G_SI, potSI; // position Verlet: half-step field averages
  T kA, kB, kB2, kG; // pow(aI, 1+alpha), pow(aI, 3+alpha), /2, pow(aI, -1+alpha)
  T p3, p1;          // pow(aSI, alpha-3), pow(aSI, alpha-1); position Verlet: of aI
  int32_t status, pad;
};
using State = StateT<double>;
using TState = StateT<Tan<double>>;

// Applies fn(x.m, y.m) to every floating member m of two scalar states.
template <class A, class B, class Fn> inline void zip_state(StateT<A> &x, const StateT<B> &y, Fn fn)
{
  fn(x.aI, y.aI);
  fn(x.aSI, y.aSI);
  fn(x.aIM, y.aIM);
  fn(x.aDotI, y.aDotI);
  fn(x.aDotSI, y.aDotSI);
  fn(x.aDotSIM, y.aDotSIM);
  for (int g = 0; g < 5; ++g) {
    fn(x.pi2[g], y.pi2[g]);
    fn(x.pi2SI[g], y.pi2SI[g]);
    fn(x.pi2SIM[g], y.pi2SIM[g]);
  }
  fn(x.g2S, y.g2S);
  fn(x.g2C, y.g2C);
  fn(x.g2D, y.g2D);
  fn(x.b2A, y.b2A);
  fn(x.b2G, y.b2G);
  fn(x.potI, y.potI);
  fn(x.g2S_SI, y.g2S_SI);
  fn(x.g2C_SI, y.g2C_SI);
  fn(x.g2D_SI, y.g2D_SI);
  fn(x.b2A_SI, y.b2A_SI);
  fn(x.b2G_SI, y.b2G_SI);
  fn(x.potSI, y.potSI);
  fn(x.kA, y.kA);
  fn(x.kB, y.kB);
  fn(x.kB2, y.kB2);
  fn(x.kG, y.kG);
  fn(x.p3, y.p3);
  fn(x.p1, y.p1);
}

struct Kick {
  double h[2][5]; // kick factors of up to two kicks: S, phi, Phi, A, SU(2)
};

template <class T> __device__ __host__ inline T ipw_h(T x, int n)
{
  if (n < 0) return 1.0 / ipw_h(x, -n);
  T r = x;
  for (int i = 1; i < n; ++i) r = r * x;
  return n == 0 ? T(1.0) : r;
}

// ---- tail: volume sums and the scale-factor update --------------------------------------------
template <class T> struct EnT {
  T ks, gs, kc, gc, kd, gd, ea, ba, eg, bg;
};
using En = EnT<double>;
template <class T> __device__ __host__ inline EnT<T> energies_of(const StateT<T> &s, const Params &p)
{
  const T a6 = ipw_h(s.aI, -6), a2 = ipw_h(s.aI, -2), e4 = 0.5 * p.rof2 * ipw_h(s.aI, -4);
  return EnT<T>{0.5 * s.pi2[0] * a6, 0.5 * s.g2S * a2, s.pi2[1] * a6, s.g2C * a2, s.pi2[2] * a6, s.g2D * a2,
                e4 * s.pi2[3] * 1.0, e4 * s.b2A / 1.0, e4 * s.pi2[4], e4 * s.b2G};
}
template <class T> __device__ __forceinline__ T sf_kernel(const StateT<T> &s, const Params &p)
{
  const double al = p.alpha;
  const EnT<T> E = energies_of(s, p);
  return pow(s.aI, 2 * al + 1) / 3.0 * p.fm2 *
         ((((al - 2) * ((E.ks + E.kc) + E.kd) + al * ((E.gs + E.gc) + E.gd)) +
           (al - 1) * ((1.0 * (E.ea + E.ba) + E.eg) + E.bg)) +
          (al + 1) * s.potI);
}
template <class T> __device__ __host__ inline T rho_of(const StateT<T> &s, const Params &p)
{
  const EnT<T> E = energies_of(s, p);
  return ((((((((((E.ks + E.kc) + E.kd) + E.gs) + E.gc) + E.gd) + E.ea) + E.ba) + E.eg) + E.bg) + 0.0) + s.potI;
}

// One-thread tail.  T = double: partials [block][kRed]; T = Tan<double>: [block][2 kRed], the
// values then their tangents.
template <class T>
__global__ void __launch_bounds__(256)
    k_tail(const double *__restrict__ partials, TailOp op, StateT<T> *__restrict__ stp, Params p)
{
  constexpr int W = TanTraits<T>::is ? 2 : 1;
  __shared__ double smem[(256 / 32) * kRed * W];
  double r[kRed * W];
  for (int k = 0; k < kRed * W; ++k) r[k] = 0;
  if (op.nblocks > 0) {
    for (int b = threadIdx.x; b < op.nblocks; b += blockDim.x)
      for (int k = 0; k < kRed * W; ++k) r[k] += partials[(size_t)b * kRed * W + k];
    block_reduce<kRed * W, 256>(r, smem);
  }
  if (threadIdx.x != 0) return;
  StateT<T> s = *stp;
  T v[kRed];
  for (int k = 0; k < kRed; ++k) {
    if constexpr (TanTraits<T>::is)
      v[k] = T(r[k], r[kRed + k]);
    else
      v[k] = r[k];
    v[k] = v[k] * p.inv_n3;
  }
  const double dt = p.dt;
  const uint32_t fl = op.flags;
  auto store_fields = [&]() {
    s.g2S = v[5];
    s.g2C = v[6];
    s.g2D = v[7];
    s.b2A = v[8];
    s.b2G = v[9];
    s.potI = v[10];
  };
  if (fl & T_STORE_ALL) {
    store_fields();
    for (int g = 0; g < 5; ++g) s.pi2[g] = s.pi2SI[g] = v[g];
  }
  auto write_hist = [&]() {
    double *h = op.hist + op.hist_row * kHistCols;
    h[0] = val(s.aI);
    h[1] = val(s.aDotI);
    h[2] = val(s.pi2[2]);
    h[3] = val(s.g2D);
    h[4] = val(s.potI);
  };
  const bool hist = op.hist != nullptr && op.hist_row >= 0;
  if (fl & T_STORE_FIELDS) store_fields();
  if (hist && (fl & T_HIST_EARLY)) write_hist();
  if (fl & T_STORE_PI2_I)
    for (int g = 0; g < 5; ++g) s.pi2[g] = v[g];
  if (fl & T_STORE_PI2_LF)
    for (int g = 0; g < 5; ++g) {
      s.pi2SIM[g] = s.pi2SI[g];
      s.pi2SI[g] = v[g];
      s.pi2[g] = 0.5 * (s.pi2SIM[g] + s.pi2SI[g]);
    }
  if (fl & T_CORRECT_ADOT) s.aDotI = sqrt(pow(s.aI, 2 * p.alpha + 2) / 3. * p.fm2 * rho_of(s, p));
  if (fl & T_VV_KICK_ONE) s.aDotI = s.aDotSI + (dt / 2) * sf_kernel(s, p) * op.w;
  if (hist && !(fl & T_HIST_EARLY)) write_hist();
  if (fl & T_LF_SYNC) s.aDotI = s.aDotSI + dt / 2.0 * sf_kernel(s, p);
  if (fl & T_LF_CTOR) s.aDotSI = s.aDotI - dt / 2.0 * sf_kernel(s, p);
  if (fl & T_LF_KICK) {
    s.aDotSIM = s.aDotSI;
    s.aDotSI += dt * sf_kernel(s, p);
    s.aDotI = (s.aDotSIM + s.aDotSI) / 2.0;
  }
  if (fl & T_LF_DRIFT) {
    s.aIM = s.aI;
    s.aI += dt * s.aDotSI;
    s.aSI = (s.aIM + s.aI) / 2.0;
  }
  if (fl & T_VV_KICK_HALF) s.aDotSI = s.aDotI + (dt / 2) * sf_kernel(s, p) * op.w2;
  if (fl & T_STORE_PI2_B)
    for (int g = 0; g < 5; ++g) s.pi2[g] = v[11 + g];
  if (fl & T_VV_DRIFT) {
    s.aIM = s.aI;
    s.aI += dt * s.aDotSI * op.w2;
    s.aSI = (s.aIM + s.aI) / 2.0;
  }
  // PositionVerlet (positionverlet.h:160-163, 207-276), as in the scalar tail; getSI is the
  // scale-factor kernel of the half-step averages at aI
  if (fl & T_PV_STORE_SI) {
    s.g2S_SI = v[5];
    s.g2C_SI = v[6];
    s.g2D_SI = v[7];
    s.b2A_SI = v[8];
    s.b2G_SI = v[9];
    s.potSI = v[10];
  }
  if (fl & T_PV_STORE_PI2)
    for (int g = 0; g < 5; ++g) {
      s.pi2SIM[g] = s.pi2[g]; // pi2AvIM
      s.pi2[g] = v[g];
      s.pi2SI[g] = 0.5 * (s.pi2[g] + s.pi2SIM[g]);
    }
  if (fl & T_PV_KICK) {
    StateT<T> si = s;
    for (int g = 0; g < 5; ++g) si.pi2[g] = s.pi2SI[g];
    si.g2S = s.g2S_SI;
    si.g2C = s.g2C_SI;
    si.g2D = s.g2D_SI;
    si.b2A = s.b2A_SI;
    si.b2G = s.b2G_SI;
    si.potI = s.potSI;
    s.aDotI += dt * sf_kernel(si, p) * op.w;
  }
  if (fl & T_PV_DRIFT_A2) {
    s.aI += dt / 2.0 * s.aDotI * op.w;
    s.aSI = (s.aIM + s.aI) / 2.0;
  }
  if (fl & T_PV_DRIFT_A1) {
    s.aIM = s.aI;
    s.aI += dt / 2.0 * s.aDotI * op.w2;
    s.aSI = s.aI;
  }
  // fixed background: the host's closed-form values (fixedbackgroundexpansion.h:37-45)
  if (fl & T_FB_AIM) s.aIM = s.aI;
  if (fl & T_FB_AI) s.aI = T(op.fa);
  if (fl & T_FB_ASI) s.aSI = T(op.fb);
  if (fl & T_FB_PV_HALF) {
    s.aIM = s.aI;
    s.aI = T(op.fb);
    s.aSI = s.aI;
  }
  if (fl & T_FB_ADOT) s.aDotI = T(op.fb);
  s.kA = pow(s.aI, 1 + p.alpha);
  s.kB = pow(s.aI, 3 + p.alpha);
  s.kB2 = pow(s.aI, 3 + p.alpha) / 2;
  s.kG = pow(s.aI, -1 + p.alpha);
  const T ad = (fl & T_PV_MODE) ? ((fl & (T_PV_DRIFT_A1 | T_FB_PV_HALF)) ? s.aIM : s.aI) : s.aSI;
  s.p3 = pow(ad, p.alpha - 3);
  s.p1 = pow(ad, p.alpha - 1);
  bool ok = finite_(s.aI) && finite_(s.aDotI) && finite_(s.aDotSI) && finite_(s.potI);
  for (int g = 0; g < 5; ++g) ok = ok && finite_(s.pi2[g]);
  if (!ok) s.status = 1;
  *stp = s;
}

} // namespace su2d
} // namespace clb

#include "clb_su2_body.cuh"
