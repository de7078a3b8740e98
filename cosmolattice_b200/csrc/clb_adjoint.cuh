// clb_adjoint.cuh - reverse-mode (adjoint) sweeps of the lphi4U1 velocity-Verlet stage.
//
// The forward map of one VV stage with weight w (velocityverlet.h:51-114, 140-210) is
//   1  aDotS = aDot0 + dt/2 w F(a0, <.>(q0, p0))
//   2  p1 = p0 + h K(q0; a0)                       h = dt/2 w (scalar), dt w / 2 (U(1))
//   3  a1 = a0 + dt w aDotS,  aS = (a0 + a1) / 2
//   4  q1 = q0 + dt w D(aS) p1                     D = aS^(alpha-3) (scalar), aS^(alpha-1) (U(1))
//   5  p2 = p1 + h K(q1; a1)
//   6  aDot1 = aDotS + dt/2 w F(a1, <.>(q1, p2))
// with q = (Re phi, Im phi, A_x, A_y, A_z), p the momenta and <.> the five volume averages
// <|pi_phi|^2>, <sum_i |D_i phi|^2>, <sum_i pi_i^2>, <B^2>, <V> that enter F
// (scalefactorkernels.h:73-77).
//
// The kernel is a metric gradient: K = -M^{-1} dU/dq with
//   U = a^{1+alpha} U_D + a^{3+alpha}/2 sum V + m_A a^{alpha-1} U_B,  M = diag(1, 1, m_A, m_A, m_A),
//   U_D = 1/(2 dx^2) sum |U_i phi(x+i) - phi(x)|^2,  U_B = 1/2 sum_{i<j} F_ij^2,  m_A = 1/(2 (fStar/omegaStar)^2),
// which reproduces complexscalarkernels.h:33-34 and u1kernels.h:44-50 term by term.  Its Jacobian
// J = dK/dq is therefore M^{-1}-symmetric and the transposed kick J^T lambda equals M J (M^{-1} lambda):
// a Jacobian-vector product, evaluated here with dual numbers over the same stencil.  The gradients
// of the averages are read off the same pieces: d<|D phi|^2>/dphi = -2/N^3 covLap,
// d<|D phi|^2>/dA_i = 1/N^3 (2 gQ/dx) Im(conj(U_i phi(x+i)) phi), d<B^2>/dA = -2/N^3 curl curl A,
// d<V>/dphi = 1/N^3 dV/dphi.
//
// Two sweeps per stage run backwards: k_u1_adj<1> at the stage output (steps 6, 5 and 4) and
// k_u1_adj<0> at the stage input (steps 2 and 1); the scalar steps (F, a, aDot) are formed on the
// host between them from the per-site dot products these sweeps reduce.

#pragma once

#include "clb_internal.cuh"
#include "clb_u1.cuh"

namespace clb {

// Value plus two derivative directions: [0] the state direction mu, [1] d/dgQ.
struct Dual2 {
  double v, d0, d1;
};
__device__ __forceinline__ Dual2 dl(double v) { return Dual2{v, 0.0, 0.0}; }
__device__ __forceinline__ Dual2 operator+(Dual2 a, Dual2 b) { return Dual2{a.v + b.v, a.d0 + b.d0, a.d1 + b.d1}; }
__device__ __forceinline__ Dual2 operator-(Dual2 a, Dual2 b) { return Dual2{a.v - b.v, a.d0 - b.d0, a.d1 - b.d1}; }
__device__ __forceinline__ Dual2 operator*(Dual2 a, Dual2 b)
{
  return Dual2{a.v * b.v, a.d0 * b.v + a.v * b.d0, a.d1 * b.v + a.v * b.d1};
}
__device__ __forceinline__ Dual2 operator*(double s, Dual2 a) { return Dual2{s * a.v, s * a.d0, s * a.d1}; }
__device__ __forceinline__ Dual2 operator*(Dual2 a, double s) { return Dual2{s * a.v, s * a.d0, s * a.d1}; }
__device__ __forceinline__ Dual2 operator/(Dual2 a, double s) { return Dual2{a.v / s, a.d0 / s, a.d1 / s}; }
__device__ __forceinline__ void sincos_d(Dual2 t, Dual2 &s, Dual2 &c)
{
  double sv, cv;
  sincos(t.v, &sv, &cv);
  s = Dual2{sv, cv * t.d0, cv * t.d1};
  c = Dual2{cv, -sv * t.d0, -sv * t.d1};
}

// Stencil pieces of the lphi4U1 kernel at one site, in dual numbers.
struct U1Pieces {
  Dual2 cl[2];  // covariant Laplacian of phi
  Dual2 dv[2];  // dV/dphi_c = 4 c4 |phi|^2 phi_c
  Dual2 cc[3];  // lapl A_i - sum_j backDiff_j forwDiff_i A_j
  Dual2 im[3];  // Im(conj(U_i phi(x+i)) phi(x))
  Dual2 d2;     // sum_i |D_i phi|^2
  double vn[2]; // |phi|^2 phi_c (d dV/dphi_c / d c4 / 4)
  double n4;    // |phi|^4 (dV / d c4)
};

// ld(c, site) returns component c at a site as a dual number (value, direction, 0).
template <class LD>
__device__ __forceinline__ void u1_pieces(LD ld, const U1Params &a, size_t s, const long long (&op)[3],
                                          const long long (&om)[3], U1Pieces &o)
{
  const Dual2 g = Dual2{a.gQ, 0.0, 1.0};
  const double ndx = -a.dx;
  const Dual2 fr = ld(0, s), fi = ld(1, s);
  Dual2 pr = dl(0), pim = dl(0), mr = dl(0), mim = dl(0), d2 = dl(0);
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const size_t sp = s + op[d], sm = s + om[d];
    Dual2 ur, ui, vr, vi;
    sincos_d(ndx * (g * ld(2 + d, s)), ui, ur);
    const Dual2 gr = ld(0, sp), gi = ld(1, sp);
    const Dual2 wr = ur * gr - ui * gi, wi = ur * gi + ui * gr;
    sincos_d(ndx * (g * ld(2 + d, sm)), vi, vr);
    const Dual2 hr = ld(0, sm), hi = ld(1, sm);
    pr = pr + wr;
    pim = pim + wi;
    mr = mr + (vr * hr + vi * hi);
    mim = mim + (vr * hi - vi * hr);
    o.im[d] = wr * fi - wi * fr;
    const Dual2 er = wr - fr, ei = wi - fi;
    d2 = d2 + (er * er + ei * ei);
  }
  o.cl[0] = (pr + mr - 6.0 * fr) / a.dx2;
  o.cl[1] = (pim + mim - 6.0 * fi) / a.dx2;
  const Dual2 n2 = fr * fr + fi * fi;
  o.dv[0] = (4.0 * a.c4) * (n2 * fr);
  o.dv[1] = (4.0 * a.c4) * (n2 * fi);
  o.vn[0] = n2.v * fr.v;
  o.vn[1] = n2.v * fi.v;
  o.n4 = n2.v * n2.v;
  o.d2 = d2 / a.dx2;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    const Dual2 c = ld(2 + i, s);
    Dual2 acc = dl(0);
#pragma unroll
    for (int d = 0; d < 3; ++d) acc = acc + (ld(2 + i, s + op[d]) + ld(2 + i, s + om[d]) - 2.0 * c);
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      const size_t sij = i == j ? s : s + op[i] + om[j];
      acc = acc - ((ld(2 + j, s + op[i]) - ld(2 + j, s)) - (ld(2 + j, sij) - ld(2 + j, s + om[j])));
    }
    o.cc[i] = acc / a.dx2;
  }
}

struct U1AdjArgs {
  // cotangents of the five averages at this sweep's state: <|pi_phi|^2>, <sum pi_A^2> act on the
  // momenta, <|D phi|^2>, <B^2>, <V> on the fields
  double Api, AE, AD, AB, AV;
  double kA, kB2, kG;    // kick coefficients at this sweep's a
  double dkA, dkB2, dkG; // their a-derivatives
  double hc, hu;         // kick factors of the transposed kick (0: none)
  double cdf, cda;       // dt w D(aS) per group: transposed drift (stage-output sweep only)
  double J0;             // 2/dx (fStar/omegaStar)^2
  double r2;             // 2 (fStar/omegaStar)^2 = 1/m_A
  double inv_n3;
};

// d/da (phi, A), d/dgQ (phi, A), d/dc4, d<|D phi|^2>/dgQ, drift (phi, A), d<V>/dc4
constexpr int kAdjSlots = 9;

// PRE = 1: sweep at the stage output (q1, p2): momentum-average gradients enter before the
// transposed kick, and the transposed drift follows; writes qbar = qbar0 and pbar_out = pbar1.
// PRE = 0: sweep at the stage input (q0, p0): transposed kick of pbar_in = pbar1, then the
// average gradients; writes qbar and pbar_out = pbar0.  With hc = hu = 0 it applies only the
// average gradients (observable seed, initial aDot correction).
// S is the storage type of the forward state (f, p); the cotangents are FP64 in either form.
template <int PRE, class S>
__global__ void __launch_bounds__(256)
    k_u1_adj(const S *__restrict__ f, const S *__restrict__ p, const double *__restrict__ pbar_in,
             double *__restrict__ qbar, double *__restrict__ pbar_out, U1Params a, U1AdjArgs g,
             double *__restrict__ partials)
{
  __shared__ double smem[(256 / 32) * kAdjSlots];
  const size_t n3 = a.n3;
  double acc[kAdjSlots];
#pragma unroll
  for (int k = 0; k < kAdjSlots; ++k) acc[k] = 0;
  const double two_n3 = 2.0 * g.inv_n3;
  // cotangent of the kick output at a site (PRE adds the momentum-average gradients)
  auto lam = [&](int c, size_t y) -> double {
    double l = pbar_in[c * n3 + y];
    if (PRE) l += (c < 2 ? g.Api : g.AE) * two_n3 * (double)p[c * n3 + y];
    return l;
  };
  for (size_t s = (size_t)blockIdx.x * blockDim.x + threadIdx.x; s < n3; s += (size_t)gridDim.x * blockDim.x) {
    long long op[3], om[3];
    u1_offsets(a.N, s, op, om);
    U1Pieces o;
    auto ld = [&](int c, size_t y) -> Dual2 {
      const double mu = c < 2 ? lam(c, y) : g.r2 * lam(c, y);
      return Dual2{(double)f[c * n3 + y], mu, 0.0};
    };
    u1_pieces(ld, a, s, op, om, o);
    // kernel values and derivatives (complexscalarkernels.h:33-34, u1kernels.h:50)
    Dual2 K[5];
    K[0] = g.kA * o.cl[0] - g.kB2 * o.dv[0];
    K[1] = g.kA * o.cl[1] - g.kB2 * o.dv[1];
    const Dual2 gq = Dual2{a.gQ, 0.0, 1.0};
#pragma unroll
    for (int i = 0; i < 3; ++i) K[2 + i] = g.kG * o.cc[i] - (g.kA * g.J0) * (gq * o.im[i]);
    double l[5], qb[5];
#pragma unroll
    for (int c = 0; c < 5; ++c) {
      l[c] = lam(c, s);
      qb[c] = qbar[c * n3 + s];
    }
    // transposed kick: qbar += h M J (M^{-1} lambda)
    qb[0] += g.hc * K[0].d0;
    qb[1] += g.hc * K[1].d0;
#pragma unroll
    for (int i = 0; i < 3; ++i) qb[2 + i] += g.hu * K[2 + i].d0 / g.r2;
    // gradients of the field averages
#pragma unroll
    for (int c = 0; c < 2; ++c) qb[c] += g.AD * (-two_n3) * o.cl[c].v + g.AV * g.inv_n3 * o.dv[c].v;
#pragma unroll
    for (int i = 0; i < 3; ++i)
      qb[2 + i] += g.AD * g.inv_n3 * (2.0 * a.gQ / a.dx) * o.im[i].v + g.AB * (-two_n3) * o.cc[i].v;
    // parameter and scale-factor dot products of the transposed kick
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      acc[0] += l[c] * (g.dkA * o.cl[c].v - g.dkB2 * o.dv[c].v);
      acc[2] += l[c] * K[c].d1;
      acc[4] += l[c] * (-g.kB2 * 4.0 * o.vn[c]);
    }
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      acc[1] += l[2 + i] * (g.dkG * o.cc[i].v - g.dkA * g.J0 * a.gQ * o.im[i].v);
      acc[3] += l[2 + i] * K[2 + i].d1;
    }
    acc[5] += o.d2.d1;
    acc[8] += o.n4;
    double pb[5];
    if (PRE) {
      // transposed drift: pbar1 = lambda + dt w D qbar1; the drift's aS dot uses p1 = p2 - h K(q1)
#pragma unroll
      for (int c = 0; c < 5; ++c) {
        const bool phi = c < 2;
        const double p1 = (double)p[c * n3 + s] - (phi ? g.hc : g.hu) * K[c].v;
        pb[c] = l[c] + (phi ? g.cdf : g.cda) * qb[c];
        acc[phi ? 6 : 7] += p1 * qb[c];
      }
    } else {
#pragma unroll
      for (int c = 0; c < 5; ++c) pb[c] = l[c] + (c < 2 ? g.Api : g.AE) * two_n3 * (double)p[c * n3 + s];
    }
#pragma unroll
    for (int c = 0; c < 5; ++c) {
      qbar[c * n3 + s] = qb[c];
      pbar_out[c * n3 + s] = pb[c];
    }
  }
  block_reduce<kAdjSlots, 256>(acc, smem);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < kAdjSlots; ++k) partials[(size_t)blockIdx.x * kAdjSlots + k] = acc[k];
  }
}

// Copies the U(1) scalar state into row r of the per-boundary record (adjoint recompute).
__global__ void k_u1_record(const U1State *__restrict__ st, U1State *__restrict__ rec, int64_t r) { rec[r] = *st; }

} // namespace clb
