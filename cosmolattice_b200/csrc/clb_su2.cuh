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
// Layout: 22 field and 19 momentum FP64 arrays of N^3 sites (x slowest).  Fields: S | phi (2) |
// Phi (4) | A_x..A_z | links U_i (4 each, i = x, y, z).  Momenta: S | phi (2) | Phi (4) | A (3) |
// pi_SU2 (3 per direction).

#pragma once

#include "clb_internal.cuh"
#include "clb_scalar.cuh"

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
};

// Scale factor, the cached averages of the five sectors (S, phi, Phi, A, SU(2)) and the sweep
// coefficients derived from a and aS.
struct State {
  double aI, aSI, aIM, aDotI, aDotSI, aDotSIM;
  double pi2[5], pi2SI[5], pi2SIM[5];
  double g2S, g2C, g2D, b2A, b2G, potI;
  double kA, kB, kB2, kG; // pow(aI, 1+alpha), pow(aI, 3+alpha), /2, pow(aI, -1+alpha)
  double p3, p1;          // pow(aSI, alpha-3), pow(aSI, alpha-1)
  int32_t status, pad;
};

struct Kick {
  double h[2][5]; // kick factors of up to two kicks: S, phi, Phi, A, SU(2)
};

struct C2 {
  double re, im;
};
__device__ __forceinline__ C2 cmul(C2 a, C2 b) { return C2{a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
__device__ __forceinline__ C2 cadd(C2 a, C2 b) { return C2{a.re + b.re, a.im + b.im}; }
__device__ __forceinline__ C2 csub(C2 a, C2 b) { return C2{a.re - b.re, a.im - b.im}; }
__device__ __forceinline__ C2 conj_(C2 a) { return C2{a.re, -a.im}; }
struct Q4 {
  double w, x, y, z;
};
__device__ __forceinline__ Q4 qmul(const Q4 &a, const Q4 &b)
{
  return Q4{a.w * b.w - (a.x * b.x + a.y * b.y + a.z * b.z), a.w * b.x + b.w * a.x - (a.y * b.z - a.z * b.y),
            a.w * b.y + b.w * a.y - (a.z * b.x - a.x * b.z), a.w * b.z + b.w * a.z - (a.x * b.y - a.y * b.x)};
}
__device__ __forceinline__ Q4 qdag(const Q4 &a) { return Q4{a.w, -a.x, -a.y, -a.z}; }
struct D2 {
  C2 u, v;
};
__device__ __forceinline__ D2 qapply(const Q4 &q, const D2 &d)
{
  return D2{cadd(cmul(C2{q.w, q.z}, d.u), cmul(C2{q.y, q.x}, d.v)),
            cadd(cmul(C2{-q.y, q.x}, d.u), cmul(C2{q.w, -q.z}, d.v))};
}
__device__ __forceinline__ D2 dscale(C2 c, const D2 &d) { return D2{cmul(c, d.u), cmul(c, d.v)}; }
__device__ __forceinline__ C2 sprod(const D2 &a, const D2 &b) { return cadd(cmul(conj_(a.u), b.u), cmul(conj_(a.v), b.v)); }
__device__ __forceinline__ D2 isig(int b, const D2 &d)
{
  const C2 I{0, 1};
  if (b == 0) return D2{cmul(I, d.v), cmul(I, d.u)};
  if (b == 1) return D2{d.v, C2{-d.u.re, -d.u.im}};
  return D2{cmul(I, d.u), cmul(C2{0, -1}, d.v)};
}
__device__ __host__ inline double ipw_h(double x, int n)
{
  if (n < 0) return 1.0 / ipw_h(x, -n);
  double r = x;
  for (int i = 1; i < n; ++i) r = r * x;
  return n == 0 ? 1.0 : r;
}
__device__ __forceinline__ double ipw(double x, int n)
{
  if (n < 0) return 1.0 / ipw(x, -n);
  double r = x;
  for (int i = 1; i < n; ++i) r = r * x;
  return n == 0 ? 1.0 : r;
}

// Read-only view of one state at one site, with the oracle's accessor names.
struct Site {
  const double *f;
  const Params *a;
  size_t s;
  long long op[3], om[3];
  __device__ __forceinline__ double F(int c, size_t t) const { return f[(size_t)c * a->n3 + t]; }
  __device__ __forceinline__ Q4 link(int i, size_t t) const
  {
    const int b = 10 + 4 * i;
    return Q4{F(b, t), F(b + 1, t), F(b + 2, t), F(b + 3, t)};
  }
  __device__ __forceinline__ D2 dbl(size_t t) const { return D2{C2{F(3, t), F(4, t)}, C2{F(5, t), F(6, t)}}; }
  __device__ __forceinline__ C2 cs(size_t t) const { return C2{F(1, t), F(2, t)}; }
  __device__ __forceinline__ C2 phase(double g, int i, size_t t) const
  {
    const double th = (-a->dx * g) * F(7 + i, t);
    return C2{cos(th), sin(th)};
  }
  __device__ __forceinline__ double normD(size_t t) const
  {
    double q = 0;
    for (int c = 0; c < 4; ++c) q = c == 0 ? F(3, t) * F(3, t) : q + F(3 + c, t) * F(3 + c, t);
    return sqrt(q);
  }
  __device__ __forceinline__ double normC(size_t t) const { return sqrt(F(1, t) * F(1, t) + F(2, t) * F(2, t)); }
  __device__ __forceinline__ double potTerm(int k) const
  {
    const double nD = normD(s);
    if (k == 0) return a->c4 * ipw(nD, 4);
    if (k == 1) return a->qG * ipw(nD * F(0, s), 2);
    return 2 * a->qH * ipw(nD * normC(s), 2);
  }
  __device__ __forceinline__ double pot() const { return (potTerm(0) + potTerm(1)) + potTerm(2); }
  __device__ __forceinline__ size_t pl(int i) const { return s + op[i]; }
  __device__ __forceinline__ size_t mi(int i) const { return s + om[i]; }
  __device__ __forceinline__ size_t plmi(int i, int j) const { return i == j ? s : s + op[i] + om[j]; }
  __device__ __forceinline__ D2 wD(int i) const { return dscale(phase(a->gD, i, s), qapply(link(i, s), dbl(pl(i)))); }
  __device__ __forceinline__ C2 wC(int i) const { return cmul(phase(a->gC, i, s), cs(pl(i))); }
  __device__ __forceinline__ double lapl(int comp) const
  {
    const double c = F(comp, s);
    double t[3];
    for (int d = 0; d < 3; ++d) t[d] = (F(comp, pl(d)) + F(comp, mi(d))) - 2 * c;
    return (1.0 / (a->dx * a->dx)) * ((t[0] + t[1]) + t[2]);
  }
  __device__ __forceinline__ double fd(int comp, size_t t0, size_t t1) const { return (F(comp, t1) - F(comp, t0)) / a->dx; }
  __device__ __forceinline__ Q4 plaq(int i, int j) const
  {
    return qmul(qmul(qmul(link(i, s), link(j, pl(i))), qdag(link(i, pl(j)))), qdag(link(j, s)));
  }
  __device__ __forceinline__ Q4 plaqBack(int i, int j) const
  {
    const size_t sm = mi(j);
    return qdag(qmul(qmul(qmul(link(i, s), qdag(link(j, plmi(i, j)))), qdag(link(i, sm))), link(j, sm)));
  }
};

__device__ __forceinline__ Site make_site(const double *f, const Params &a, size_t s)
{
  Site v;
  v.f = f;
  v.a = &a;
  v.s = s;
  u1_offsets(a.N, s, v.op, v.om);
  return v;
}

// ---- momentum kernels at one site (momentum-component order) ----------------------------------
__device__ __forceinline__ C2 covLapC(const Site &v)
{
  C2 plus{0, 0}, minus{0, 0};
  for (int d = 0; d < 3; ++d) {
    const C2 w = cmul(v.phase(v.a->gC, d, v.s), v.cs(v.pl(d)));
    const C2 m = cmul(conj_(v.phase(v.a->gC, d, v.mi(d))), v.cs(v.mi(d)));
    plus = d == 0 ? w : cadd(plus, w);
    minus = d == 0 ? m : cadd(minus, m);
  }
  const double dx2 = v.a->dx * v.a->dx;
  const C2 c = v.cs(v.s);
  return C2{((plus.re + minus.re) - 6 * c.re) / dx2, ((plus.im + minus.im) - 6 * c.im) / dx2};
}

__device__ __forceinline__ void covLapD(const Site &v, double out[4])
{
  D2 plus{}, minus{};
  for (int d = 0; d < 3; ++d) {
    const D2 w = qapply(v.link(d, v.s), dscale(v.phase(v.a->gD, d, v.s), v.dbl(v.pl(d))));
    const size_t sm = v.mi(d);
    const D2 m = qapply(qdag(v.link(d, sm)), dscale(conj_(v.phase(v.a->gD, d, sm)), v.dbl(sm)));
    if (d == 0) {
      plus = w;
      minus = m;
    } else {
      plus = D2{cadd(plus.u, w.u), cadd(plus.v, w.v)};
      minus = D2{cadd(minus.u, m.u), cadd(minus.v, m.v)};
    }
  }
  const double dx2 = v.a->dx * v.a->dx;
  const D2 c = v.dbl(v.s);
  out[0] = ((plus.u.re + minus.u.re) - 6 * c.u.re) / dx2;
  out[1] = ((plus.u.im + minus.u.im) - 6 * c.u.im) / dx2;
  out[2] = ((plus.v.re + minus.v.re) - 6 * c.v.re) / dx2;
  out[3] = ((plus.v.im + minus.v.im) - 6 * c.v.im) / dx2;
}

__device__ __forceinline__ void kernels(const Site &v, const State &st, double K[NP])
{
  const Params &a = *v.a;
  const size_t s = v.s;
  const double A = st.kA, B = st.kB, B2 = st.kB2;
  const double nD = v.normD(s), nC = v.normC(s), S = v.F(0, s);
  K[0] = A * v.lapl(0) - B * (2 * a.qG * ipw(nD, 2) * S);
  const C2 cl = covLapC(v);
  const double ndC = 4 * a.qH * ipw(nD, 2) * nC;
  K[1] = A * cl.re - B2 * (ndC / nC * v.F(1, s));
  K[2] = A * cl.im - B2 * (ndC / nC * v.F(2, s));
  double dl[4];
  covLapD(v, dl);
  const double ndD = a.c4 * (4 * ipw(nD, 3)) + nD * (2 * a.qG * ipw(S, 2) + 4 * a.qH * ipw(nC, 2));
  for (int c = 0; c < 4; ++c) K[3 + c] = A * dl[c] - B2 * (ndD / nD * v.F(3 + c, s));
  const D2 D0 = v.dbl(s);
  const C2 C0 = v.cs(s);
  for (int i = 0; i < 3; ++i) {
    const double lap = v.lapl(7 + i);
    double grad = 0;
    for (int j = 0; j < 3; ++j) {
      const double g0 = v.fd(7 + j, s, v.pl(i));
      const double g1 = v.fd(7 + j, v.mi(j), v.plmi(i, j));
      const double t = (g0 - g1) / a.dx;
      grad = j == 0 ? t : grad + t;
    }
    const double Jc = a.gC * cmul(conj_(v.wC(i)), C0).im;
    const double Jd = a.gD * sprod(v.wD(i), D0).im;
    const double J = 2.0 / a.dx * a.rfo2 * (Jc + Jd);
    K[7 + i] = st.kG * (lap - grad) - A * J;
  }
  const double normGrad = ipw(1 / a.dx, 3) / a.gS * st.kG;
  const double normSrc = (1 / a.dx) * A;
  for (int i = 0; i < 3; ++i) {
    double gr[3] = {0, 0, 0}, gb[3] = {0, 0, 0};
    bool first = true;
    for (int j = 0; j < 3; ++j) {
      if (j == i) continue;
      const Q4 P = v.plaq(i, j), Pb = v.plaqBack(i, j);
      const double pv[3] = {P.x, P.y, P.z}, bv[3] = {Pb.x, Pb.y, Pb.z};
      for (int c = 0; c < 3; ++c) {
        gr[c] = first ? pv[c] : gr[c] + pv[c];
        gb[c] = first ? bv[c] : gb[c] + bv[c];
      }
      first = false;
    }
    const D2 W = v.wD(i);
    for (int c = 0; c < 3; ++c) {
      const double J = a.rfo2 / 2 * (a.gS * sprod(W, isig(c, D0)).re);
      K[10 + 3 * i + c] = -normGrad * (gr[c] - gb[c]) - normSrc * J;
    }
  }
}

// ---- per-site averages (fieldfunctionals.h) -------------------------------------------------------
__device__ __forceinline__ double sGrad2(const Site &v)
{
  double acc = 0;
  for (int j = 0; j < 3; ++j) {
    const double g = v.fd(0, v.s, v.pl(j));
    acc = j == 0 ? g * g : acc + g * g;
  }
  return acc;
}
__device__ __forceinline__ double cGrad2(const Site &v)
{
  const C2 c = v.cs(v.s);
  double acc = 0;
  for (int j = 0; j < 3; ++j) {
    const C2 d0 = csub(v.wC(j), c);
    const C2 d{d0.re / v.a->dx, d0.im / v.a->dx};
    const double n2 = d.re * d.re + d.im * d.im;
    acc = j == 0 ? n2 : acc + n2;
  }
  return acc;
}
__device__ __forceinline__ double dGrad2(const Site &v)
{
  const D2 c = v.dbl(v.s);
  double acc = 0;
  for (int j = 0; j < 3; ++j) {
    const D2 w = qapply(v.link(j, v.s), dscale(v.phase(v.a->gD, j, v.s), v.dbl(v.pl(j))));
    const C2 du0 = csub(w.u, c.u), dv0 = csub(w.v, c.v);
    const C2 du{du0.re / v.a->dx, du0.im / v.a->dx}, dv{dv0.re / v.a->dx, dv0.im / v.a->dx};
    const double n2 = (du.re * du.re + du.im * du.im) + (dv.re * dv.re + dv.im * dv.im);
    acc = j == 0 ? n2 : acc + n2;
  }
  return acc;
}
__device__ __forceinline__ double Fij(const Site &v, int i, int j)
{
  return v.fd(7 + j, v.s, v.pl(i)) - v.fd(7 + i, v.s, v.pl(j));
}
__device__ __forceinline__ double aB2(const Site &v)
{
  const double f21 = Fij(v, 1, 0), f31 = Fij(v, 2, 0), f32 = Fij(v, 2, 1);
  return f21 * f21 + (f31 * f31 + f32 * f32);
}
__device__ __forceinline__ double gB2(const Site &v)
{
  const double c = 4.0 / (ipw(v.a->dx, 4) * ipw(v.a->gS, 2));
  const double t10 = 2 - 2 * v.plaq(1, 0).w, t20 = 2 - 2 * v.plaq(2, 0).w, t21 = 2 - 2 * v.plaq(2, 1).w;
  return c * (t10 + (t20 + t21));
}
// momentum sums of the five sectors from momentum values q[19]
__device__ __forceinline__ void pi2s(const double *q, double out[5])
{
  out[0] = q[0] * q[0];
  out[1] = q[1] * q[1] + q[2] * q[2];
  out[2] = ((q[3] * q[3] + q[4] * q[4]) + q[5] * q[5]) + q[6] * q[6];
  out[3] = (q[7] * q[7] + q[8] * q[8]) + q[9] * q[9];
  double acc = 0;
  for (int i = 0; i < 3; ++i) {
    double ai = 0;
    for (int b = 0; b < 3; ++b) {
      const double e = q[10 + 3 * i + b];
      ai = b == 0 ? 4 * (e * e) : ai + 4 * (e * e);
    }
    acc = i == 0 ? ai : acc + ai;
  }
  out[4] = acc;
}

__device__ __forceinline__ int sector(int c) { return c == 0 ? 0 : c < 3 ? 1 : c < 7 ? 2 : c < 10 ? 3 : 4; }

// Kick sweep: NK (0..2) in-place kicks with the kernel at the current fields; partials [0..4]
// momentum sums after the first kick (or as they are, NK = 0), [5..10] <grad^2> S, phi, Phi,
// <B^2> U(1), SU(2), <V>; [11..15] momentum sums after the second kick.
template <int NK, bool RF, bool RP>
__global__ void __launch_bounds__(128)
    k_kick(const double *__restrict__ f, double *__restrict__ p, Params a, Kick kc, const State *__restrict__ stp,
           double *__restrict__ partials)
{
  __shared__ double smem[(128 / 32) * kRed];
  const State st = *stp;
  double acc[kRed];
  for (int k = 0; k < kRed; ++k) acc[k] = 0;
  for (size_t s = (size_t)blockIdx.x * blockDim.x + threadIdx.x; s < a.n3; s += (size_t)gridDim.x * blockDim.x) {
    const Site v = make_site(f, a, s);
    double q[NP];
    for (int c = 0; c < NP; ++c) q[c] = p[(size_t)c * a.n3 + s];
    if (NK > 0) {
      double K[NP];
      kernels(v, st, K);
      for (int k = 0; k < NK; ++k) {
        for (int c = 0; c < NP; ++c) q[c] = q[c] + kc.h[k][sector(c)] * K[c];
        if (RP) {
          double t[5];
          pi2s(q, t);
          for (int g = 0; g < 5; ++g) acc[(k == 0 ? 0 : 11) + g] += t[g];
        }
      }
      for (int c = 0; c < NP; ++c) p[(size_t)c * a.n3 + s] = q[c];
    } else if (RP) {
      double t[5];
      pi2s(q, t);
      for (int g = 0; g < 5; ++g) acc[g] += t[g];
    }
    if (RF) {
      acc[5] += sGrad2(v);
      acc[6] += cGrad2(v);
      acc[7] += dGrad2(v);
      acc[8] += aB2(v);
      acc[9] += gB2(v);
      acc[10] += v.pot();
    }
  }
  if (RF || RP) {
    block_reduce<kRed, 128>(acc, smem);
    if (threadIdx.x == 0)
      for (int k = 0; k < kRed; ++k) partials[(size_t)blockIdx.x * kRed + k] = acc[k];
  }
}

// Drifts (velocityverlet.h:181-222; the leapfrog's forms leapfrog.h:203-236 have lf = 1).
__device__ __forceinline__ Q4 qexp(double p1, double p2, double p3)
{
  const double n = sqrt(p1 * p1 + p2 * p2 + p3 * p3);
  if (n == 0) return Q4{1, 0, 0, 0};
  const double sn = sin(n) / n;
  return Q4{cos(n), sn * p1, sn * p2, sn * p3};
}
static __global__ void __launch_bounds__(256)
    k_drift(double *__restrict__ f, const double *__restrict__ p, Params a, double w, int lf,
            const State *__restrict__ stp)
{
  const double dt = a.dt, p3 = stp->p3, p1 = stp->p1;
  const double cC = lf ? p3 * dt : p3 * dt * w;
  const double cA = lf ? p1 * dt : p1 * w * dt;
  const double cG = lf ? p1 * a.dx * dt * a.gS : w * p1 * a.dx * dt * a.gS;
  const double dtw = lf ? dt : dt * w;
  const size_t n3 = a.n3;
  for (size_t s = (size_t)blockIdx.x * blockDim.x + threadIdx.x; s < n3; s += (size_t)gridDim.x * blockDim.x) {
    f[s] = f[s] + p3 * (dtw * p[s]);
    for (int c = 1; c < 7; ++c) f[c * n3 + s] = f[c * n3 + s] + cC * p[c * n3 + s];
    for (int i = 0; i < 3; ++i) f[(7 + i) * n3 + s] = f[(7 + i) * n3 + s] + cA * p[(7 + i) * n3 + s] * 1.0;
    for (int i = 0; i < 3; ++i) {
      const size_t pb = (size_t)(10 + 3 * i) * n3 + s, fb = (size_t)(10 + 4 * i) * n3 + s;
      const Q4 E = qexp(cG * p[pb], cG * p[pb + n3], cG * p[pb + 2 * n3]);
      const Q4 U = qmul(E, Q4{f[fb], f[fb + n3], f[fb + 2 * n3], f[fb + 3 * n3]});
      f[fb] = U.w;
      f[fb + n3] = U.x;
      f[fb + 2 * n3] = U.y;
      f[fb + 3 * n3] = U.z;
    }
  }
}

// ---- tail: volume sums and the scale-factor update --------------------------------------------
struct En {
  double ks, gs, kc, gc, kd, gd, ea, ba, eg, bg;
};
__device__ __host__ inline En energies_of(const State &s, const Params &p)
{
  const double a6 = ipw_h(s.aI, -6), a2 = ipw_h(s.aI, -2), e4 = 0.5 * p.rof2 * ipw_h(s.aI, -4);
  return En{0.5 * s.pi2[0] * a6, 0.5 * s.g2S * a2, s.pi2[1] * a6, s.g2C * a2, s.pi2[2] * a6, s.g2D * a2,
            e4 * s.pi2[3] * 1.0, e4 * s.b2A / 1.0, e4 * s.pi2[4], e4 * s.b2G};
}
__device__ __forceinline__ double sf_kernel(const State &s, const Params &p)
{
  const double al = p.alpha;
  const En E = energies_of(s, p);
  return pow(s.aI, 2 * al + 1) / 3.0 * p.fm2 *
         ((((al - 2) * ((E.ks + E.kc) + E.kd) + al * ((E.gs + E.gc) + E.gd)) +
           (al - 1) * ((1.0 * (E.ea + E.ba) + E.eg) + E.bg)) +
          (al + 1) * s.potI);
}
__device__ __host__ inline double rho_of(const State &s, const Params &p)
{
  const En E = energies_of(s, p);
  return ((((((((((E.ks + E.kc) + E.kd) + E.gs) + E.gc) + E.gd) + E.ea) + E.ba) + E.eg) + E.bg) + 0.0) + s.potI;
}

static __global__ void __launch_bounds__(256)
    k_tail(const double *__restrict__ partials, TailOp op, State *__restrict__ stp, Params p)
{
  __shared__ double smem[(256 / 32) * kRed];
  double v[kRed];
  for (int k = 0; k < kRed; ++k) v[k] = 0;
  if (op.nblocks > 0) {
    for (int b = threadIdx.x; b < op.nblocks; b += blockDim.x)
      for (int k = 0; k < kRed; ++k) v[k] += partials[(size_t)b * kRed + k];
    block_reduce<kRed, 256>(v, smem);
  }
  if (threadIdx.x != 0) return;
  State s = *stp;
  for (int k = 0; k < kRed; ++k) v[k] *= p.inv_n3;
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
    double *r = op.hist + op.hist_row * kHistCols;
    r[0] = s.aI;
    r[1] = s.aDotI;
    r[2] = s.pi2[2];
    r[3] = s.g2D;
    r[4] = s.potI;
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
  s.kA = pow(s.aI, 1 + p.alpha);
  s.kB = pow(s.aI, 3 + p.alpha);
  s.kB2 = pow(s.aI, 3 + p.alpha) / 2;
  s.kG = pow(s.aI, -1 + p.alpha);
  s.p3 = pow(s.aSI, p.alpha - 3);
  s.p1 = pow(s.aSI, p.alpha - 1);
  bool ok = isfinite(s.aI) && isfinite(s.aDotI) && isfinite(s.aDotSI) && isfinite(s.potI);
  for (int g = 0; g < 5; ++g) ok = ok && isfinite(s.pi2[g]);
  if (!ok) s.status = 1;
  *stp = s;
}

// ---- measurement sums (one sweep) ----------------------------------------------------------------
// [0..4] momentum sums of the five sectors, [5..10] field sums as in the kick sweep, [11..13] the
// three potential terms, means [14..41] (seven rows of f, f^2, m, m^2 with raw values), Gauss
// U(1) [42..45] (|LHS-RHS|, |sum|, |RHS|, |LHS|), Gauss SU(2) [46..57] (same per algebra index).
static __global__ void __launch_bounds__(128)
    k_measure(const double *__restrict__ f, const double *__restrict__ p, Params a, double am, double ag,
              double *__restrict__ partials)
{
  __shared__ double smem[(128 / 32) * kMeas];
  double acc[kMeas];
  for (int k = 0; k < kMeas; ++k) acc[k] = 0;
  const size_t n3 = a.n3;
  const double dx = a.dx;
  for (size_t s = (size_t)blockIdx.x * blockDim.x + threadIdx.x; s < n3; s += (size_t)gridDim.x * blockDim.x) {
    const Site v = make_site(f, a, s);
    double q[NP];
    for (int c = 0; c < NP; ++c) q[c] = p[(size_t)c * n3 + s];
    double t[5];
    pi2s(q, t);
    for (int g = 0; g < 5; ++g) acc[g] += t[g];
    acc[5] += sGrad2(v);
    acc[6] += cGrad2(v);
    acc[7] += dGrad2(v);
    acc[8] += aB2(v);
    acc[9] += gB2(v);
    acc[10] += v.pot();
    for (int k = 0; k < 3; ++k) acc[11 + k] += v.potTerm(k);
    auto row = [&](int r, double fv, double mv) {
      acc[14 + 4 * r] += fv;
      acc[15 + 4 * r] += fv * fv;
      acc[16 + 4 * r] += mv;
      acc[17 + 4 * r] += mv * mv;
    };
    const double r2 = sqrt(2.0);
    row(0, v.F(0, s), q[0] * am);
    row(1, r2 * v.F(1, s), r2 * q[1] * am);
    row(2, r2 * v.F(2, s), r2 * q[2] * am);
    {
      const double pa = q[1] * am, pb = q[2] * am;
      row(3, v.normC(s), sqrt(pa * pa + pb * pb));
    }
    {
      double pd = 0;
      for (int c = 0; c < 4; ++c) pd += q[3 + c] * q[3 + c];
      row(4, v.normD(s), sqrt(pd) * am);
    }
    {
      const double e1 = q[7] * ag, e2 = q[8] * ag, e3 = q[9] * ag;
      const double b1 = Fij(v, 2, 1), b2 = Fij(v, 0, 2), b3 = Fij(v, 1, 0);
      row(5, sqrt(e1 * e1 + e2 * e2 + e3 * e3), sqrt(b1 * b1 + b2 * b2 + b3 * b3));
    }
    {
      double e = 0;
      for (int c = 0; c < 9; ++c) e += 4 * q[10 + c] * q[10 + c];
      row(6, ag * sqrt(e), sqrt(gB2(v)));
    }
    // Gauss U(1)
    {
      double l[3];
      for (int i = 0; i < 3; ++i) l[i] = q[7 + i] - p[(size_t)(7 + i) * n3 + v.mi(i)];
      const double LHS = ((l[0] + l[1]) + l[2]) / dx;
      const double nrm = 2 / dx * a.rfo2;
      const double imc = cmul(conj_(C2{q[1], q[2]}), v.cs(s)).im;
      const double imd = sprod(D2{C2{q[3], q[4]}, C2{q[5], q[6]}}, v.dbl(s)).im;
      const double rho = nrm * a.gC * imc + nrm * a.gD * imd;
      const double RHS = -dx * rho;
      const double L1 = l[0] / dx, L2 = l[1] / dx, L3 = l[2] / dx;
      const double diff = LHS - (RHS + 0.0), sum = L1 * L1 + L2 * L2 + L3 * L3 + (RHS + 0.0) * (RHS + 0.0);
      acc[42] += sqrt(diff * diff);
      acc[43] += sqrt(sum * sum);
      acc[44] += sqrt(RHS * RHS);
      acc[45] += sqrt(LHS * LHS);
    }
    // Gauss SU(2)
    {
      double L[3];
      for (int i = 0; i < 3; ++i) {
        const size_t sm = v.mi(i);
        const Q4 Ui = v.link(i, sm);
        const size_t pb = (size_t)(10 + 3 * i) * n3 + sm;
        const Q4 r = qmul(qmul(qdag(Ui), Q4{0, p[pb], p[pb + n3], p[pb + 2 * n3]}), Ui);
        const double rv[3] = {r.x, r.y, r.z};
        for (int b = 0; b < 3; ++b) {
          const double tt = (1 / dx) * (q[10 + 3 * i + b] - rv[b]);
          L[b] = i == 0 ? tt : L[b] + tt;
        }
      }
      const D2 D0 = v.dbl(s);
      const D2 pd{C2{q[3], q[4]}, C2{q[5], q[6]}};
      for (int b = 0; b < 3; ++b) {
        const double R = (-1.0) * (a.rfo2 / 2 * (a.gS * sprod(isig(b, D0), pd).re));
        const double df = L[b] - R, sm = L[b] + R;
        acc[46 + 4 * b] += sqrt(df * df);
        acc[47 + 4 * b] += sqrt(sm * sm);
        acc[48 + 4 * b] += sqrt(R * R);
        acc[49 + 4 * b] += sqrt(L[b] * L[b]);
      }
    }
  }
  block_reduce<kMeas, 128>(acc, smem);
  if (threadIdx.x == 0)
    for (int k = 0; k < kMeas; ++k) partials[(size_t)blockIdx.x * kMeas + k] = acc[k];
}

} // namespace su2d
} // namespace clb
