// clb_su2_body.cuh - lphi4SU2U1 site arithmetic, kick, drift and measurement kernels, templated on
// the storage type S (double or float) and the arithmetic type T of the site kernels.  The FP64
// form uses S = T = double and rounds in the reference's order (the unit is compiled without FMA
// contraction); the FP32 form stores and stencils in float (S = T = float) with every kick and
// drift increment added in FP64 and rounded once, and measures in FP64 (T = double over float
// storage).  Included by clb_su2.cuh.
#pragma once

#include "clb_su2.cuh"

#include <type_traits>

namespace clb {
namespace su2d {

template <class T> struct C2 {
  T re, im;
};
template <class T> __device__ __forceinline__ C2<T> cmul(C2<T> a, C2<T> b)
{
  return C2<T>{a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
template <class T> __device__ __forceinline__ C2<T> cadd(C2<T> a, C2<T> b) { return C2<T>{a.re + b.re, a.im + b.im}; }
template <class T> __device__ __forceinline__ C2<T> csub(C2<T> a, C2<T> b) { return C2<T>{a.re - b.re, a.im - b.im}; }
template <class T> __device__ __forceinline__ C2<T> conj_(C2<T> a) { return C2<T>{a.re, -a.im}; }
template <class T> struct Q4 {
  T w, x, y, z;
};
template <class T> __device__ __forceinline__ Q4<T> qmul(const Q4<T> &a, const Q4<T> &b)
{
  return Q4<T>{a.w * b.w - (a.x * b.x + a.y * b.y + a.z * b.z), a.w * b.x + b.w * a.x - (a.y * b.z - a.z * b.y),
               a.w * b.y + b.w * a.y - (a.z * b.x - a.x * b.z), a.w * b.z + b.w * a.z - (a.x * b.y - a.y * b.x)};
}
template <class T> __device__ __forceinline__ Q4<T> qdag(const Q4<T> &a) { return Q4<T>{a.w, -a.x, -a.y, -a.z}; }
template <class T> struct D2 {
  C2<T> u, v;
};
// U (u, v) with U = [[q0 + i q3, q2 + i q1], [-q2 + i q1, q0 - i q3]]
template <class T> __device__ __forceinline__ D2<T> qapply(const Q4<T> &q, const D2<T> &d)
{
  return D2<T>{cadd(cmul(C2<T>{q.w, q.z}, d.u), cmul(C2<T>{q.y, q.x}, d.v)),
               cadd(cmul(C2<T>{-q.y, q.x}, d.u), cmul(C2<T>{q.w, -q.z}, d.v))};
}
template <class T> __device__ __forceinline__ D2<T> dscale(C2<T> c, const D2<T> &d) { return D2<T>{cmul(c, d.u), cmul(c, d.v)}; }
template <class T> __device__ __forceinline__ C2<T> sprod(const D2<T> &a, const D2<T> &b)
{
  return cadd(cmul(conj_(a.u), b.u), cmul(conj_(a.v), b.v));
}
// i sigma_b applied to a doublet
template <class T> __device__ __forceinline__ D2<T> isig(int b, const D2<T> &d)
{
  const C2<T> I{0, 1};
  if (b == 0) return D2<T>{cmul(I, d.v), cmul(I, d.u)};
  if (b == 1) return D2<T>{d.v, C2<T>{-d.u.re, -d.u.im}};
  return D2<T>{cmul(I, d.u), cmul(C2<T>{0, -1}, d.v)};
}
// Divisions of the kernels: the FP64 form keeps the reference's rounding (a / b); the FP32 form,
// bound to no rounding order, multiplies by the reciprocal (formed once per site for dx, dx^2 and
// the field norms); the tangent-linear types divide as Tan does.
template <class T> __device__ __forceinline__ T kdiv(T a, T b) { return a / b; }
template <> __device__ __forceinline__ float kdiv<float>(float a, float b) { return a * (1.0f / b); }
// the FP32 tangent-linear form: the value part as kdiv<float> forms it (bitwise the plain form)
template <> __device__ __forceinline__ Tan<float> kdiv<Tan<float>>(Tan<float> a, Tan<float> b)
{
  const float r = 1.0f / b.v, q = a.v * r;
  return Tan<float>(q, (a.d - q * b.d) * r);
}

template <class T> __device__ __forceinline__ T ipw(T x, int n)
{
  if (n < 0) return T(1) / ipw(x, -n);
  T r = x;
  for (int i = 1; i < n; ++i) r = r * x;
  return n == 0 ? T(1) : r;
}

// Read-only view of one state at one site (storage S, arithmetic T), with the oracle's names.
// With T = Tan<S> a value reads as (f, df): the state and its tangent.
template <class S, class T> struct Site {
  const S *f;
  const S *df;
  // U(1) link phases exp(-i dx g A_i) for g = gQ of phi (C) and of Phi (D), kept by the drift:
  // [4 i + 2 (0 C, 1 D) + (0 cos, 1 sin)] x n3; null: formed from A here
  const S *ph;
  const Params *a;
  size_t s;
  long long op[3], om[3];
  T dx, gC, gD, gS, qG, qH, c4;
  __device__ __forceinline__ T F(int c, size_t t) const
  {
    const size_t i = (size_t)c * a->n3 + t;
    if constexpr (TanTraits<T>::is)
      return T((typename TanTraits<T>::base)f[i], (typename TanTraits<T>::base)df[i]);
    else
      return (T)f[i];
  }
  __device__ __forceinline__ Q4<T> link(int i, size_t t) const
  {
    const int b = 10 + 4 * i;
    return Q4<T>{F(b, t), F(b + 1, t), F(b + 2, t), F(b + 3, t)};
  }
  __device__ __forceinline__ D2<T> dbl(size_t t) const { return D2<T>{C2<T>{F(3, t), F(4, t)}, C2<T>{F(5, t), F(6, t)}}; }
  __device__ __forceinline__ C2<T> cs(size_t t) const { return C2<T>{F(1, t), F(2, t)}; }
  // the stored phases when the arithmetic type is the storage type (the same cos and sin of the
  // same argument, formed by the drift), else formed here
  __device__ __forceinline__ C2<T> phaseCD(int which, int i, size_t t) const
  {
    if constexpr (std::is_same<S, T>::value) {
      if (ph) {
        const size_t b = (size_t)(4 * i + 2 * which) * a->n3 + t;
        return C2<T>{ph[b], ph[b + a->n3]};
      }
    }
    return phase(which == 0 ? gC : gD, i, t);
  }
  __device__ __forceinline__ C2<T> phaseC(int i, size_t t) const { return phaseCD(0, i, t); }
  __device__ __forceinline__ C2<T> phaseD(int i, size_t t) const { return phaseCD(1, i, t); }
  __device__ __forceinline__ C2<T> phase(T g, int i, size_t t) const
  {
    const T th = (-dx * g) * F(7 + i, t);
    return C2<T>{cos(th), sin(th)};
  }
  __device__ __forceinline__ T normD(size_t t) const
  {
    T q = 0;
    for (int c = 0; c < 4; ++c) q = c == 0 ? F(3, t) * F(3, t) : q + F(3 + c, t) * F(3 + c, t);
    return sqrt(q);
  }
  __device__ __forceinline__ T normC(size_t t) const { return sqrt(F(1, t) * F(1, t) + F(2, t) * F(2, t)); }
  __device__ __forceinline__ T potTerm(int k) const
  {
    const T nD = normD(s);
    if (k == 0) return c4 * ipw(nD, 4);
    if (k == 1) return qG * ipw(nD * F(0, s), 2);
    return 2 * qH * ipw(nD * normC(s), 2);
  }
  __device__ __forceinline__ T pot() const { return (potTerm(0) + potTerm(1)) + potTerm(2); }
  // pot() from |Phi|, |phi| and S at this site, formed as potTerm forms them
  __device__ __forceinline__ T pot_at(T nD, T nC, T Sv) const
  {
    return (c4 * ipw(nD, 4) + qG * ipw(nD * Sv, 2)) + 2 * qH * ipw(nD * nC, 2);
  }
  __device__ __forceinline__ size_t pl(int i) const { return s + op[i]; }
  __device__ __forceinline__ size_t mi(int i) const { return s + om[i]; }
  __device__ __forceinline__ size_t plmi(int i, int j) const { return i == j ? s : s + op[i] + om[j]; }
  __device__ __forceinline__ D2<T> wD(int i) const { return dscale(phaseD(i, s), qapply(link(i, s), dbl(pl(i)))); }
  __device__ __forceinline__ C2<T> wC(int i) const { return cmul(phaseC(i, s), cs(pl(i))); }
  __device__ __forceinline__ T lapl(int comp) const
  {
    const T c = F(comp, s);
    T t[3];
    for (int d = 0; d < 3; ++d) t[d] = (F(comp, pl(d)) + F(comp, mi(d))) - 2 * c;
    return kdiv(T(1), dx * dx) * ((t[0] + t[1]) + t[2]);
  }
  __device__ __forceinline__ T fd(int comp, size_t t0, size_t t1) const { return kdiv(F(comp, t1) - F(comp, t0), dx); }
  __device__ __forceinline__ Q4<T> plaq(int i, int j) const
  {
    return qmul(qmul(qmul(link(i, s), link(j, pl(i))), qdag(link(i, pl(j)))), qdag(link(j, s)));
  }
  __device__ __forceinline__ Q4<T> plaqBack(int i, int j) const
  {
    const size_t sm = mi(j);
    return qdag(qmul(qmul(qmul(link(i, s), qdag(link(j, plmi(i, j)))), qdag(link(i, sm))), link(j, sm)));
  }
};

template <class S, class T> __device__ __forceinline__ Site<S, T> make_site(const S *f, const Params &a, size_t s)
{
  Site<S, T> v;
  v.f = f;
  v.df = nullptr;
  v.ph = nullptr;
  v.a = &a;
  v.s = s;
  v.dx = (T)a.dx;
  v.gC = (T)a.gC;
  v.gD = (T)a.gD;
  v.gS = (T)a.gS;
  v.qG = (T)a.qG;
  v.qH = (T)a.qH;
  v.c4 = (T)a.c4;
  u1_offsets(a.N, s, v.op, v.om);
  return v;
}

// Derivatives of the couplings along the tangent direction, in the model's order: qG, qH, gQ of
// phi, gQ of Phi under U(1), gQ of Phi under SU(2), c4.
struct CoupDot {
  double v[6];
};

// Tangent-linear view: the state f with its tangent df, and the couplings with their tangents.
template <class S>
__device__ __forceinline__ Site<S, Tan<S>> make_site_tan(const S *f, const S *df, const Params &a, size_t s,
                                                        const CoupDot &cd)
{
  using T = Tan<S>;
  Site<S, T> v;
  v.f = f;
  v.df = df;
  v.ph = nullptr;
  v.a = &a;
  v.s = s;
  v.dx = T(a.dx);
  auto cp = [&](double x, int k) { return T((S)x, (S)cd.v[k]); };
  v.qG = cp(a.qG, 0);
  v.qH = cp(a.qH, 1);
  v.gC = cp(a.gC, 2);
  v.gD = cp(a.gD, 3);
  v.gS = cp(a.gS, 4);
  v.c4 = cp(a.c4, 5);
  u1_offsets(a.N, s, v.op, v.om);
  return v;
}

// ---- momentum kernels at one site (momentum-component order) ----------------------------------
// Direction d's term of the gradient energies cGrad2 and dGrad2 below, from the forward product w
// (the phi or Phi value at x + d parallel transported to x) and the value c at x.
template <class S, class T> __device__ __forceinline__ T cgrad_term(const Site<S, T> &v, const C2<T> &w, const C2<T> &c)
{
  const C2<T> d0 = csub(w, c);
  const C2<T> d{kdiv(d0.re, v.dx), kdiv(d0.im, v.dx)};
  return d.re * d.re + d.im * d.im;
}
template <class S, class T> __device__ __forceinline__ T dgrad_term(const Site<S, T> &v, const D2<T> &w, const D2<T> &c)
{
  const C2<T> du0 = csub(w.u, c.u), dv0 = csub(w.v, c.v);
  const C2<T> du{kdiv(du0.re, v.dx), kdiv(du0.im, v.dx)}, dv{kdiv(dv0.re, v.dx), kdiv(dv0.im, v.dx)};
  return (du.re * du.re + du.im * du.im) + (dv.re * dv.re + dv.im * dv.im);
}

// g2: also form cGrad2 (covLapC) or dGrad2 (covLapD) from the same forward products.
template <class S, class T> __device__ __forceinline__ C2<T> covLapC(const Site<S, T> &v, T *g2 = nullptr)
{
  C2<T> plus{0, 0}, minus{0, 0};
  for (int d = 0; d < 3; ++d) {
    const C2<T> w = cmul(v.phaseC(d, v.s), v.cs(v.pl(d)));
    if (g2) {
      const T n2 = cgrad_term(v, w, v.cs(v.s));
      *g2 = d == 0 ? n2 : *g2 + n2;
    }
    const C2<T> m = cmul(conj_(v.phaseC(d, v.mi(d))), v.cs(v.mi(d)));
    plus = d == 0 ? w : cadd(plus, w);
    minus = d == 0 ? m : cadd(minus, m);
  }
  const T dx2 = v.dx * v.dx;
  const C2<T> c = v.cs(v.s);
  return C2<T>{kdiv((plus.re + minus.re) - 6 * c.re, dx2), kdiv((plus.im + minus.im) - 6 * c.im, dx2)};
}

template <class S, class T> __device__ __forceinline__ void covLapD(const Site<S, T> &v, T out[4], T *g2 = nullptr)
{
  D2<T> plus{}, minus{};
  for (int d = 0; d < 3; ++d) {
    const D2<T> w = qapply(v.link(d, v.s), dscale(v.phaseD(d, v.s), v.dbl(v.pl(d))));
    if (g2) {
      const T n2 = dgrad_term(v, w, v.dbl(v.s));
      *g2 = d == 0 ? n2 : *g2 + n2;
    }
    const size_t sm = v.mi(d);
    const D2<T> m = qapply(qdag(v.link(d, sm)), dscale(conj_(v.phaseD(d, sm)), v.dbl(sm)));
    if (d == 0) {
      plus = w;
      minus = m;
    } else {
      plus = D2<T>{cadd(plus.u, w.u), cadd(plus.v, w.v)};
      minus = D2<T>{cadd(minus.u, m.u), cadd(minus.v, m.v)};
    }
  }
  const T dx2 = v.dx * v.dx;
  const D2<T> c = v.dbl(v.s);
  out[0] = kdiv((plus.u.re + minus.u.re) - 6 * c.u.re, dx2);
  out[1] = kdiv((plus.u.im + minus.u.im) - 6 * c.u.im, dx2);
  out[2] = kdiv((plus.v.re + minus.v.re) - 6 * c.v.re, dx2);
  out[3] = kdiv((plus.v.im + minus.v.im) - 6 * c.v.im, dx2);
}

// Kick coefficients pow(aI, 1+alpha), pow(aI, 3+alpha), its half and pow(aI, -1+alpha).
template <class T> struct Coef {
  T A, B, B2, G;
};

// SECT: 0 all components; 1 S, phi, Phi and A (K[0..9]); 2 the SU(2) field (K[10..18]);
// 3 S, phi and Phi (K[0..6]); 4 A (K[7..9]); 5 S and phi (K[0..2]); 6 Phi (K[3..6]).  Each
// component's kernel is the same expression in every SECT that holds it.
__host__ __device__ constexpr bool sect_sphi(int sect) { return sect == 0 || sect == 1 || sect == 3 || sect == 5; }
__host__ __device__ constexpr bool sect_dbl(int sect) { return sect == 0 || sect == 1 || sect == 3 || sect == 6; }
__host__ __device__ constexpr bool sect_scalars(int sect) { return sect_sphi(sect) || sect_dbl(sect); }
__host__ __device__ constexpr bool sect_u1(int sect) { return sect == 0 || sect == 1 || sect == 4; }
__host__ __device__ constexpr bool sect_su2(int sect) { return sect == 0 || sect == 2; }
// momentum sectors [sect_g0, sect_g1) of SECT (0 S, 1 phi, 2 Phi, 3 A, 4 SU(2))
__host__ __device__ constexpr int sect_g0(int sect) { return sect == 2 ? 4 : sect == 4 ? 3 : sect == 6 ? 2 : 0; }
__host__ __device__ constexpr int sect_g1(int sect)
{
  return sect == 1 || sect == 4 ? 4 : sect == 3 || sect == 6 ? 3 : sect == 5 ? 2 : 5;
}
// whether SECT writes partial slot k of a kick sweep: the momentum sums of its sectors (k < 5 and
// k >= 11), the gradient sums of S, phi (5, 6) and Phi (7), B^2 of A (8) and SU(2) (9), V (10,
// with S and phi)
__host__ __device__ constexpr bool sect_owns(int sect, int k)
{
  return k < 5 || k >= 11 ? ((k < 5 ? k : k - 11) >= sect_g0(sect) && (k < 5 ? k : k - 11) < sect_g1(sect))
         : k == 7 ? sect_dbl(sect) : k == 8 ? sect_u1(sect) : k == 9 ? sect_su2(sect) : sect_sphi(sect);
}

// Per-site terms of the volume averages a kick sweep reduces with RF (fieldfunctionals.h):
// gradient energies of S, phi and Phi, B^2 of A and of SU(2), and V.  They equal, to the last
// bit, what sGrad2, cGrad2, dGrad2, aB2, gB2 and Site::pot give at the site.
template <class T> struct SiteAvg {
  T g2S, g2C, g2D, b2A, b2G, pot;
};
template <class S, class T> __device__ __forceinline__ T sGrad2(const Site<S, T> &v);
template <class S, class T> __device__ __forceinline__ T aB2(const Site<S, T> &v, const T (*g)[3] = nullptr);
template <class S, class T> __device__ __forceinline__ T gB2(const Site<S, T> &v, const T *pw = nullptr);

// AVG: also form the SiteAvg terms of the sectors in SECT into *av, from the covariant products,
// differences and plaquettes the kernels form anyway.
template <int SECT = 0, bool AVG = false, class S, class T>
__device__ __forceinline__ void kernels(const Site<S, T> &v, const Coef<T> &C, T K[NP], SiteAvg<T> *av = nullptr)
{
  const Params &a = *v.a;
  const size_t s = v.s;
  const T A = C.A, B = C.B, B2 = C.B2, G = C.G;
  const T qG = v.qG, qH = v.qH, c4 = v.c4, rfo2 = (T)a.rfo2;
  if constexpr (sect_scalars(SECT)) {
    const T nD = v.normD(s), nC = v.normC(s), Sv = v.F(0, s);
    if constexpr (sect_sphi(SECT)) {
      K[0] = A * v.lapl(0) - B * (2 * qG * ipw(nD, 2) * Sv);
      const C2<T> cl = covLapC(v, AVG ? &av->g2C : nullptr);
      const T ndC = 4 * qH * ipw(nD, 2) * nC;
      K[1] = A * cl.re - B2 * (kdiv(ndC, nC) * v.F(1, s));
      K[2] = A * cl.im - B2 * (kdiv(ndC, nC) * v.F(2, s));
    }
    if constexpr (sect_dbl(SECT)) {
      T dl[4];
      covLapD(v, dl, AVG ? &av->g2D : nullptr);
      const T ndD = c4 * (4 * ipw(nD, 3)) + nD * (2 * qG * ipw(Sv, 2) + 4 * qH * ipw(nC, 2));
      for (int c = 0; c < 4; ++c) K[3 + c] = A * dl[c] - B2 * (kdiv(ndD, nD) * v.F(3 + c, s));
    }
    if constexpr (AVG && sect_sphi(SECT)) {
      av->g2S = sGrad2(v);
      av->pot = v.pot_at(nD, nC, Sv);
    }
  }
  if constexpr (sect_u1(SECT)) {
    const D2<T> D0 = v.dbl(s);
    const C2<T> C0 = v.cs(s);
    T g0s[3][3]; // g0s[i][j]: forward difference of A_j along i
    for (int i = 0; i < 3; ++i) {
      const T lap = v.lapl(7 + i);
      T grad = 0;
      for (int j = 0; j < 3; ++j) {
        const T g0 = v.fd(7 + j, s, v.pl(i));
        g0s[i][j] = g0;
        const T g1 = v.fd(7 + j, v.mi(j), v.plmi(i, j));
        const T t = kdiv(g0 - g1, v.dx);
        grad = j == 0 ? t : grad + t;
      }
      const T Jc = v.gC * cmul(conj_(v.wC(i)), C0).im;
      const T Jd = v.gD * sprod(v.wD(i), D0).im;
      const T J = kdiv(T(2.0), v.dx) * rfo2 * (Jc + Jd);
      K[7 + i] = G * (lap - grad) - A * J;
    }
    if constexpr (AVG) av->b2A = aB2(v, g0s);
  }
  if constexpr (sect_su2(SECT)) {
    const D2<T> Dg = v.dbl(s);
    const T normGrad = kdiv(ipw(kdiv(T(1), v.dx), 3), v.gS) * G;
    const T normSrc = kdiv(T(1), v.dx) * A;
    T pw[3]; // plaq(1, 0).w, plaq(2, 0).w, plaq(2, 1).w
    for (int i = 0; i < 3; ++i) {
      T gr[3] = {0, 0, 0}, gb[3] = {0, 0, 0};
      bool first = true;
      for (int j = 0; j < 3; ++j) {
        if (j == i) continue;
        const Q4<T> P = v.plaq(i, j), Pb = v.plaqBack(i, j);
        if (j < i) pw[i + j - 1] = P.w;
        const T pv[3] = {P.x, P.y, P.z}, bv[3] = {Pb.x, Pb.y, Pb.z};
        for (int c = 0; c < 3; ++c) {
          gr[c] = first ? pv[c] : gr[c] + pv[c];
          gb[c] = first ? bv[c] : gb[c] + bv[c];
        }
        first = false;
      }
      const D2<T> W = v.wD(i);
      for (int c = 0; c < 3; ++c) {
        const T J = rfo2 / 2 * (v.gS * sprod(W, isig(c, Dg)).re);
        K[10 + 3 * i + c] = -normGrad * (gr[c] - gb[c]) - normSrc * J;
      }
    }
    if constexpr (AVG) av->b2G = gB2(v, pw);
  }
}

// ---- per-site averages (fieldfunctionals.h) -------------------------------------------------------
template <class S, class T> __device__ __forceinline__ T sGrad2(const Site<S, T> &v)
{
  T acc = 0;
  for (int j = 0; j < 3; ++j) {
    const T g = v.fd(0, v.s, v.pl(j));
    acc = j == 0 ? g * g : acc + g * g;
  }
  return acc;
}
template <class S, class T> __device__ __forceinline__ T cGrad2(const Site<S, T> &v)
{
  const C2<T> c = v.cs(v.s);
  T acc = 0;
  for (int j = 0; j < 3; ++j) {
    const T n2 = cgrad_term(v, v.wC(j), c);
    acc = j == 0 ? n2 : acc + n2;
  }
  return acc;
}
template <class S, class T> __device__ __forceinline__ T dGrad2(const Site<S, T> &v)
{
  const D2<T> c = v.dbl(v.s);
  T acc = 0;
  for (int j = 0; j < 3; ++j) {
    const T n2 = dgrad_term(v, qapply(v.link(j, v.s), dscale(v.phaseD(j, v.s), v.dbl(v.pl(j)))), c);
    acc = j == 0 ? n2 : acc + n2;
  }
  return acc;
}
// aB2's g and gB2's pw: the differences and plaquettes as kernels() formed them
template <class S, class T> __device__ __forceinline__ T Fij(const Site<S, T> &v, int i, int j)
{
  return v.fd(7 + j, v.s, v.pl(i)) - v.fd(7 + i, v.s, v.pl(j));
}
template <class S, class T> __device__ __forceinline__ T aB2(const Site<S, T> &v, const T (*g)[3])
{
  auto F = [&](int i, int j) { return g ? g[i][j] - g[j][i] : Fij(v, i, j); };
  const T f21 = F(1, 0), f31 = F(2, 0), f32 = F(2, 1);
  return f21 * f21 + (f31 * f31 + f32 * f32);
}
template <class S, class T> __device__ __forceinline__ T gB2(const Site<S, T> &v, const T *pw)
{
  const T c = kdiv(T(4.0), ipw(v.dx, 4) * ipw(v.gS, 2));
  const T t10 = 2 - 2 * (pw ? pw[0] : v.plaq(1, 0).w), t20 = 2 - 2 * (pw ? pw[1] : v.plaq(2, 0).w),
          t21 = 2 - 2 * (pw ? pw[2] : v.plaq(2, 1).w);
  return c * (t10 + (t20 + t21));
}
// The SiteAvg terms of the sectors in SECT, formed on their own (a sweep that does not kick).
template <int SECT, class S, class T> __device__ __forceinline__ SiteAvg<T> site_avg(const Site<S, T> &v)
{
  SiteAvg<T> av{};
  if constexpr (sect_sphi(SECT)) {
    av.g2S = sGrad2(v);
    av.g2C = cGrad2(v);
    av.pot = v.pot();
  }
  if constexpr (sect_dbl(SECT)) av.g2D = dGrad2(v);
  if constexpr (sect_u1(SECT)) av.b2A = aB2(v);
  if constexpr (sect_su2(SECT)) av.b2G = gB2(v);
  return av;
}

// First momentum component of sector g (0 S, 1 phi, 2 Phi, 3 A, 4 SU(2)); g = 5: one past the last.
__host__ __device__ constexpr int sector_c0(int g) { return g == 0 ? 0 : g == 1 ? 1 : g == 2 ? 3 : g == 3 ? 7 : g == 4 ? 10 : NP; }

// momentum sums of sectors [G0, G1) (FP64) from momentum values q[19], reading only their
// components q[sector_c0(G0) .. sector_c0(G1))
template <int G0 = 0, int G1 = 5, class R> __device__ __forceinline__ void pi2s(const R *qs, double out[5])
{
  double q[NP];
  for (int c = sector_c0(G0); c < sector_c0(G1); ++c) q[c] = (double)qs[c];
  if (G0 <= 0 && G1 > 0) out[0] = q[0] * q[0];
  if (G0 <= 1 && G1 > 1) out[1] = q[1] * q[1] + q[2] * q[2];
  if (G0 <= 2 && G1 > 2) out[2] = ((q[3] * q[3] + q[4] * q[4]) + q[5] * q[5]) + q[6] * q[6];
  if (G0 <= 3 && G1 > 3) out[3] = (q[7] * q[7] + q[8] * q[8]) + q[9] * q[9];
  if (G1 == 5) {
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
}

__device__ __forceinline__ int sector(int c) { return c == 0 ? 0 : c < 3 ? 1 : c < 7 ? 2 : c < 10 ? 3 : 4; }

// Kick sweep: NK (0..2) in-place kicks with the kernel at the current fields, each increment added
// in FP64 and rounded to the storage type once.  Partials: [0..4] momentum sums after the first kick
// (or as they are, NK = 0), [5..10] <grad^2> S, phi, Phi, <B^2> U(1), SU(2), <V>; [11..15] the
// momentum sums after the second kick.
// Resident 128-thread blocks per SM: FP32 gains from four (128 registers, 1.28x), FP64 keeps three
// (170 registers); more spills than occupancy pays for beyond that.
#ifndef CLB_SU2_KICK_MINB_F32
#define CLB_SU2_KICK_MINB_F32 4
#endif
#ifndef CLB_SU2_KICK_MINB_F64
#define CLB_SU2_KICK_MINB_F64 3
#endif
// SECT (as kernels()): 0 every sector in one sweep; 1 and 2 the two halves of a split sweep, or
// 3, 4 and 2 the three parts of a three-way split, run one after the other over the same grid.
// Each part updates, reduces and writes only its own components and partial slots (1: sectors S,
// phi, Phi, A, the field sums but <B^2> of SU(2); 2: the SU(2) sector and its <B^2>; 3: sectors
// S, phi, Phi, their gradient sums and <V>; 4: sector A and its <B^2>), so the parts hold fewer
// registers than the whole.  The kicks read the fields only, so the parts' order is free.
// The halves of a split sweep (192^3, ms per step, same call): FP64 8.17 whole, 6.23 halves at
// three blocks, 5.73 at four; FP32 4.66 whole, 3.31 halves at four blocks, 3.64 at five.
#ifndef CLB_SU2_HALF_MINB_F32
#define CLB_SU2_HALF_MINB_F32 4
#endif
#ifndef CLB_SU2_HALF_MINB_F64
#define CLB_SU2_HALF_MINB_F64 4
#endif
// the FP64 three-part sweep's S, phi, Phi part (SECT 3) and A part (SECT 4); four blocks timed
// best at 192^3 (ms per step): 4.99, against 5.37 with three for SECT 3 and 5.04 with five for SECT 4
#ifndef CLB_SU2_P3_MINB_F64
#define CLB_SU2_P3_MINB_F64 CLB_SU2_HALF_MINB_F64
#endif
#ifndef CLB_SU2_P4_MINB_F64
#define CLB_SU2_P4_MINB_F64 CLB_SU2_HALF_MINB_F64
#endif
// the FP64 four-part sweep's S and phi part (SECT 5) and Phi part (SECT 6)
#ifndef CLB_SU2_P5_MINB_F64
#define CLB_SU2_P5_MINB_F64 CLB_SU2_HALF_MINB_F64
#endif
#ifndef CLB_SU2_P6_MINB_F64
#define CLB_SU2_P6_MINB_F64 CLB_SU2_HALF_MINB_F64
#endif
template <class S, int NK, bool RF, bool RP, int SECT = 0>
__global__ void __launch_bounds__(128, SECT == 0   ? (sizeof(S) == 4 ? CLB_SU2_KICK_MINB_F32 : CLB_SU2_KICK_MINB_F64)
                                       : sizeof(S) == 4 ? CLB_SU2_HALF_MINB_F32
                                       : SECT == 3      ? CLB_SU2_P3_MINB_F64
                                       : SECT == 4      ? CLB_SU2_P4_MINB_F64
                                       : SECT == 5      ? CLB_SU2_P5_MINB_F64
                                       : SECT == 6      ? CLB_SU2_P6_MINB_F64
                                                        : CLB_SU2_HALF_MINB_F64)
    k_kick(const S *__restrict__ f, S *__restrict__ p, Params a, Kick kc, const State *__restrict__ stp,
           double *__restrict__ partials, const S *__restrict__ ph)
{
  constexpr int G0 = sect_g0(SECT), G1 = sect_g1(SECT);                   // sectors [G0, G1)
  constexpr int C0 = sector_c0(G0), C1 = sector_c0(G1);                    // momentum components [C0, C1)
  __shared__ double smem[(128 / 32) * kRed];
  const State st = *stp;
  double acc[kRed];
  for (int k = 0; k < kRed; ++k) acc[k] = 0;
  for_sites(a.N, a.n3, a.order, [&](size_t s) {
    Site<S, S> v = make_site<S, S>(f, a, s);
    v.ph = ph;
    S q[NP];
    for (int c = C0; c < C1; ++c) q[c] = p[(size_t)c * a.n3 + s];
    SiteAvg<S> av; // with RF: formed by kernels() when the sweep kicks, else by site_avg()
    if (NK > 0) {
      S K[NP];
      kernels<SECT, RF>(v, Coef<S>{(S)st.kA, (S)st.kB, (S)st.kB2, (S)st.kG}, K, &av);
      for (int k = 0; k < NK; ++k) {
        for (int c = C0; c < C1; ++c) q[c] = (S)((double)q[c] + kc.h[k][sector(c)] * (double)K[c]);
        if (RP) {
          double t[5];
          pi2s<G0, G1>(q, t);
          for (int g = G0; g < G1; ++g) acc[(k == 0 ? 0 : 11) + g] += t[g];
        }
      }
      for (int c = C0; c < C1; ++c) p[(size_t)c * a.n3 + s] = q[c];
    } else if (RP) {
      double t[5];
      pi2s<G0, G1>(q, t);
      for (int g = G0; g < G1; ++g) acc[g] += t[g];
    }
    if (RF && NK == 0) av = site_avg<SECT>(v);
    if (RF) {
      if (sect_sphi(SECT)) {
        acc[5] += (double)av.g2S;
        acc[6] += (double)av.g2C;
      }
      if (sect_dbl(SECT)) acc[7] += (double)av.g2D;
      if (sect_u1(SECT)) acc[8] += (double)av.b2A;
      if (sect_su2(SECT)) acc[9] += (double)av.b2G;
      if (sect_sphi(SECT)) acc[10] += (double)av.pot;
    }
  });
  if (RF || RP) {
    block_reduce<kRed, 128>(acc, smem);
    if (threadIdx.x == 0)
      for (int k = 0; k < kRed; ++k)
        if (sect_owns(SECT, k)) partials[(size_t)blockIdx.x * kRed + k] = acc[k];
  }
}

// Drifts (velocityverlet.h:181-222; the leapfrog's forms leapfrog.h:203-236 have lf = 1), in FP64
// and rounded to the storage type once.
__device__ __forceinline__ Q4<double> qexp(double p1, double p2, double p3)
{
  const double n = sqrt(p1 * p1 + p2 * p2 + p3 * p3);
  if (n == 0) return Q4<double>{1, 0, 0, 0};
  const double sn = sin(n) / n;
  return Q4<double>{cos(n), sn * p1, sn * p2, sn * p3};
}
// The U(1) link phases of A_i(x) for both couplings, exactly as Site::phase forms them, into the
// phase arrays the kick reads.
template <class S> __device__ __forceinline__ void put_phases(S *__restrict__ ph, const Params &a, int i, size_t s, S A)
{
  const size_t n3 = a.n3;
#pragma unroll
  for (int which = 0; which < 2; ++which) {
    const S th = (-(S)a.dx * (S)(which == 0 ? a.gC : a.gD)) * A;
    const size_t b = (size_t)(4 * i + 2 * which) * n3 + s;
    ph[b] = cos(th);
    ph[b + n3] = sin(th);
  }
}
template <class S> __global__ void __launch_bounds__(256) k_phases(const S *__restrict__ f, S *__restrict__ ph, Params a)
{
  for (size_t s = (size_t)blockIdx.x * blockDim.x + threadIdx.x; s < a.n3; s += (size_t)gridDim.x * blockDim.x)
    for (int i = 0; i < 3; ++i) put_phases(ph, a, i, s, f[(size_t)(7 + i) * a.n3 + s]);
}

template <class S>
__global__ void __launch_bounds__(256)
    k_drift(S *__restrict__ f, const S *__restrict__ p, Params a, double w, int lf, const State *__restrict__ stp,
            S *__restrict__ ph, double dtd)
{
  // dtd: the time step of this drift (the position Verlet's half drifts pass dt/2)
  const double dt = dtd, p3 = stp->p3, p1 = stp->p1;
  const double cC = lf ? p3 * dt : p3 * dt * w;
  const double cA = lf ? p1 * dt : p1 * w * dt;
  const double cG = lf ? p1 * a.dx * dt * a.gS : w * p1 * a.dx * dt * a.gS;
  const double dtw = lf ? dt : dt * w;
  const size_t n3 = a.n3;
  for (size_t s = (size_t)blockIdx.x * blockDim.x + threadIdx.x; s < n3; s += (size_t)gridDim.x * blockDim.x) {
    f[s] = (S)((double)f[s] + p3 * (dtw * (double)p[s]));
    for (int c = 1; c < 7; ++c) f[c * n3 + s] = (S)((double)f[c * n3 + s] + cC * (double)p[c * n3 + s]);
    for (int i = 0; i < 3; ++i) {
      const S A = (S)((double)f[(7 + i) * n3 + s] + cA * (double)p[(7 + i) * n3 + s] * 1.0);
      f[(7 + i) * n3 + s] = A;
      put_phases(ph, a, i, s, A);
    }
    for (int i = 0; i < 3; ++i) {
      const size_t pb = (size_t)(10 + 3 * i) * n3 + s, fb = (size_t)(10 + 4 * i) * n3 + s;
      const Q4<double> E = qexp(cG * (double)p[pb], cG * (double)p[pb + n3], cG * (double)p[pb + 2 * n3]);
      const Q4<double> U = qmul(E, Q4<double>{(double)f[fb], (double)f[fb + n3], (double)f[fb + 2 * n3], (double)f[fb + 3 * n3]});
      f[fb] = (S)U.w;
      f[fb + n3] = (S)U.x;
      f[fb + 2 * n3] = (S)U.y;
      f[fb + 3 * n3] = (S)U.z;
    }
  }
}

// Re-unitarisation of the stored links (FP32 form): U <- U / |U| in FP64.
template <class S> __global__ void __launch_bounds__(256) k_unitarize(S *__restrict__ f, size_t n3)
{
  for (size_t s = (size_t)blockIdx.x * blockDim.x + threadIdx.x; s < 3 * n3; s += (size_t)gridDim.x * blockDim.x) {
    const size_t i = s / n3, t = s - i * n3, fb = (size_t)(10 + 4 * i) * n3 + t;
    const double w = f[fb], x = f[fb + n3], y = f[fb + 2 * n3], z = f[fb + 3 * n3];
    const double r = 1.0 / sqrt(((w * w + x * x) + y * y) + z * z);
    f[fb] = (S)(w * r);
    f[fb + n3] = (S)(x * r);
    f[fb + 2 * n3] = (S)(y * r);
    f[fb + 3 * n3] = (S)(z * r);
  }
}

// ---- measurement sums (one sweep) ----------------------------------------------------------------
// [0..4] momentum sums of the five sectors, [5..10] field sums as in the kick sweep, [11..13] the
// three potential terms, means [14..41] (seven rows of f, f^2, m, m^2 with raw values), Gauss
// U(1) [42..45] (|LHS-RHS|, |sum|, |RHS|, |LHS|), Gauss SU(2) [46..57] (same per algebra index).
template <class S>
__global__ void __launch_bounds__(128)
    k_measure(const S *__restrict__ f, const S *__restrict__ p, Params a, double am, double ag,
              double *__restrict__ partials)
{
  __shared__ double smem[(128 / 32) * kMeas];
  double acc[kMeas];
  for (int k = 0; k < kMeas; ++k) acc[k] = 0;
  const size_t n3 = a.n3;
  const double dx = a.dx;
  for (size_t s = (size_t)blockIdx.x * blockDim.x + threadIdx.x; s < n3; s += (size_t)gridDim.x * blockDim.x) {
    const Site<S, double> v = make_site<S, double>(f, a, s);
    double q[NP];
    for (int c = 0; c < NP; ++c) q[c] = (double)p[(size_t)c * n3 + s];
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
      for (int i = 0; i < 3; ++i) l[i] = q[7 + i] - (double)p[(size_t)(7 + i) * n3 + v.mi(i)];
      const double LHS = ((l[0] + l[1]) + l[2]) / dx;
      const double nrm = 2 / dx * a.rfo2;
      const double imc = cmul(conj_(C2<double>{q[1], q[2]}), v.cs(s)).im;
      const double imd = sprod(D2<double>{C2<double>{q[3], q[4]}, C2<double>{q[5], q[6]}}, v.dbl(s)).im;
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
        const Q4<double> Ui = v.link(i, sm);
        const size_t pb = (size_t)(10 + 3 * i) * n3 + sm;
        const Q4<double> r =
            qmul(qmul(qdag(Ui), Q4<double>{0, (double)p[pb], (double)p[pb + n3], (double)p[pb + 2 * n3]}), Ui);
        const double rv[3] = {r.x, r.y, r.z};
        for (int b = 0; b < 3; ++b) {
          const double tt = (1 / dx) * (q[10 + 3 * i + b] - rv[b]);
          L[b] = i == 0 ? tt : L[b] + tt;
        }
      }
      const D2<double> D0 = v.dbl(s);
      const D2<double> pd{C2<double>{q[3], q[4]}, C2<double>{q[5], q[6]}};
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

// ---- tangent-linear form ---------------------------------------------------------------------------
// The kernels below evolve (state, tangent) pairs: every expression is the plain kernel's, in
// Tan arithmetic, so the state follows the plain evolution bitwise and the tangent is its exact
// derivative along the coupling direction (and the tangent of the start state).

// derivative of pi2s along the momentum tangent dq (sectors [G0, G1) as pi2s)
template <int G0 = 0, int G1 = 5, class R> __device__ __forceinline__ void pi2s_tan(const R *qs, const R *dqs, double out[5])
{
  double q[NP], d[NP];
  for (int c = sector_c0(G0); c < sector_c0(G1); ++c) {
    q[c] = (double)qs[c];
    d[c] = (double)dqs[c];
  }
  if (G0 <= 0 && G1 > 0) out[0] = 2 * (q[0] * d[0]);
  if (G0 <= 1 && G1 > 1) out[1] = 2 * (q[1] * d[1] + q[2] * d[2]);
  if (G0 <= 2 && G1 > 2) out[2] = 2 * (((q[3] * d[3] + q[4] * d[4]) + q[5] * d[5]) + q[6] * d[6]);
  if (G0 <= 3 && G1 > 3) out[3] = 2 * ((q[7] * d[7] + q[8] * d[8]) + q[9] * d[9]);
  if (G1 == 5) {
    double acc = 0;
    for (int c = 10; c < NP; ++c) acc += 8 * (q[c] * d[c]);
    out[4] = acc;
  }
}

// Tangent kick sweep: k_kick on (p, dp) with kernels and field sums in Tan<S>; partials
// [block][2 kRed]: the kRed sums of k_kick, then their tangents.
// SECT as k_kick: 0 whole; 1 and 2 the halves, or 3, 4 and 2 the three parts, of a split sweep.
// Resident blocks per SM of the tangent kick parts: three in FP64, four in FP32, timed at 256^3 VV2
// (ms per tangent step, 1 / 2 / 3 / 4 blocks): FP64 39.2, 39.3, 37.9, 39.3; FP32 23.2, 23.3, 21.9,
// 21.4.  The value part stays the plain evolution's bitwise either way.
#ifndef CLB_SU2_TAN_MINB_F64
#define CLB_SU2_TAN_MINB_F64 3
#endif
#ifndef CLB_SU2_TAN_MINB_F32
#define CLB_SU2_TAN_MINB_F32 4
#endif
template <class S, int NK, bool RF, bool RP, int SECT = 0>
__global__ void __launch_bounds__(128, sizeof(S) == 4 ? CLB_SU2_TAN_MINB_F32 : CLB_SU2_TAN_MINB_F64)
    k_kick_tan(const S *__restrict__ f, const S *__restrict__ df, S *__restrict__ p, S *__restrict__ dp, Params a,
               Kick kc, const TState *__restrict__ stp, CoupDot cd, double *__restrict__ partials)
{
  using T = Tan<S>;
  constexpr int G0 = sect_g0(SECT), G1 = sect_g1(SECT);                   // sectors [G0, G1)
  constexpr int C0 = sector_c0(G0), C1 = sector_c0(G1);                    // momentum components [C0, C1)
  __shared__ double smem[(128 / 32) * 2 * kRed];
  const Coef<T> C{T(stp->kA), T(stp->kB), T(stp->kB2), T(stp->kG)};
  double acc[2 * kRed];
  for (int k = 0; k < 2 * kRed; ++k) acc[k] = 0;
  for_sites(a.N, a.n3, a.order, [&](size_t s) {
    const Site<S, T> v = make_site_tan<S>(f, df, a, s, cd);
    S q[NP], dq[NP];
    for (int c = C0; c < C1; ++c) {
      q[c] = p[(size_t)c * a.n3 + s];
      dq[c] = dp[(size_t)c * a.n3 + s];
    }
    auto add_pi = [&](int base) {
      double t[5], td[5];
      pi2s<G0, G1>(q, t);
      pi2s_tan<G0, G1>(q, dq, td);
      for (int g = G0; g < G1; ++g) {
        acc[base + g] += t[g];
        acc[kRed + base + g] += td[g];
      }
    };
    SiteAvg<T> av;
    if (NK > 0) {
      T K[NP];
      kernels<SECT, RF>(v, C, K, &av);
      for (int k = 0; k < NK; ++k) {
        for (int c = C0; c < C1; ++c) {
          const double h = kc.h[k][sector(c)];
          q[c] = (S)((double)q[c] + h * (double)K[c].v);
          dq[c] = (S)((double)dq[c] + h * (double)K[c].d);
        }
        if (RP) add_pi(k == 0 ? 0 : 11);
      }
      for (int c = C0; c < C1; ++c) {
        p[(size_t)c * a.n3 + s] = q[c];
        dp[(size_t)c * a.n3 + s] = dq[c];
      }
    } else if (RP) {
      add_pi(0);
    }
    if (RF && NK == 0) av = site_avg<SECT>(v);
    if (RF) {
      auto addf = [&](int k, T r) {
        acc[5 + k] += (double)r.v;
        acc[kRed + 5 + k] += (double)r.d;
      };
      if (sect_sphi(SECT)) {
        addf(0, av.g2S);
        addf(1, av.g2C);
      }
      if (sect_dbl(SECT)) addf(2, av.g2D);
      if (sect_u1(SECT)) addf(3, av.b2A);
      if (sect_su2(SECT)) addf(4, av.b2G);
      if (sect_sphi(SECT)) addf(5, av.pot);
    }
  });
  if (RF || RP) {
    block_reduce<2 * kRed, 128>(acc, smem);
    if (threadIdx.x == 0)
      for (int k = 0; k < 2 * kRed; ++k) // value and tangent slots alike
        if (sect_owns(SECT, k % kRed)) partials[(size_t)blockIdx.x * 2 * kRed + k] = acc[k];
  }
}

// exp of an algebra element with its tangent; the value is qexp's.  d(sin n / n)/dn =
// (n cos n - sin n) / n^2 is taken from its Taylor series below n = 0.1, where the closed form
// cancels.
__device__ __forceinline__ Q4<Tan<double>> qexp_tan(Tan<double> p1, Tan<double> p2, Tan<double> p3)
{
  using T = Tan<double>;
  const double n = sqrt(p1.v * p1.v + p2.v * p2.v + p3.v * p3.v);
  if (n == 0) return Q4<T>{T(1.0), T(0.0, p1.d), T(0.0, p2.d), T(0.0, p3.d)};
  const double sn = sin(n) / n, cn = cos(n);
  const double dn = ((p1.v * p1.d + p2.v * p2.d) + p3.v * p3.d) / n;
  double ds;
  if (n < 0.1) {
    const double x = n * n;
    ds = -n * (1.0 / 3 - x * (1.0 / 30 - x * (1.0 / 840 - x / 45360)));
  } else {
    ds = (n * cn - sin(n)) / (n * n);
  }
  const double sd = ds * dn;
  return Q4<T>{T(cn, -sin(n) * dn), T(sn * p1.v, sd * p1.v + sn * p1.d), T(sn * p2.v, sd * p2.v + sn * p2.d),
               T(sn * p3.v, sd * p3.v + sn * p3.d)};
}

// Tangent drift: k_drift on (f, df) with the drift coefficients' tangents (through aS, and g_SU2 in
// the link step).
template <class S>
__global__ void __launch_bounds__(256)
    k_drift_tan(S *__restrict__ f, S *__restrict__ df, const S *__restrict__ p, const S *__restrict__ dp, Params a,
                double w, int lf, const TState *__restrict__ stp, CoupDot cd)
{
  using T = Tan<double>;
  const double dt = a.dt;
  const T p3 = stp->p3, p1 = stp->p1;
  const T gS(a.gS, cd.v[4]);
  const T cC = lf ? p3 * dt : p3 * dt * w;
  const T cA = lf ? p1 * dt : p1 * w * dt;
  const T cG = lf ? p1 * a.dx * dt * gS : w * p1 * a.dx * dt * gS;
  const double dtw = lf ? dt : dt * w;
  const size_t n3 = a.n3;
  auto ld = [](const S *x, const S *dx, size_t i) { return T((double)x[i], (double)dx[i]); };
  auto put = [](S *x, S *dx, size_t i, T r) {
    x[i] = (S)r.v;
    dx[i] = (S)r.d;
  };
  for (size_t s = (size_t)blockIdx.x * blockDim.x + threadIdx.x; s < n3; s += (size_t)gridDim.x * blockDim.x) {
    put(f, df, s, ld(f, df, s) + p3 * (dtw * ld(p, dp, s)));
    for (int c = 1; c < 7; ++c) put(f, df, c * n3 + s, ld(f, df, c * n3 + s) + cC * ld(p, dp, c * n3 + s));
    for (int i = 0; i < 3; ++i)
      put(f, df, (7 + i) * n3 + s, ld(f, df, (7 + i) * n3 + s) + cA * ld(p, dp, (7 + i) * n3 + s) * 1.0);
    for (int i = 0; i < 3; ++i) {
      const size_t pb = (size_t)(10 + 3 * i) * n3 + s, fb = (size_t)(10 + 4 * i) * n3 + s;
      const Q4<T> E = qexp_tan(cG * ld(p, dp, pb), cG * ld(p, dp, pb + n3), cG * ld(p, dp, pb + 2 * n3));
      const Q4<T> U = qmul(E, Q4<T>{ld(f, df, fb), ld(f, df, fb + n3), ld(f, df, fb + 2 * n3), ld(f, df, fb + 3 * n3)});
      put(f, df, fb, U.w);
      put(f, df, fb + n3, U.x);
      put(f, df, fb + 2 * n3, U.y);
      put(f, df, fb + 3 * n3, U.z);
    }
  }
}

// Tangent re-unitarisation (FP32 form): U <- U / |U| on (f, df).
template <class S> __global__ void __launch_bounds__(256) k_unitarize_tan(S *__restrict__ f, S *__restrict__ df, size_t n3)
{
  using T = Tan<double>;
  for (size_t s = (size_t)blockIdx.x * blockDim.x + threadIdx.x; s < 3 * n3; s += (size_t)gridDim.x * blockDim.x) {
    const size_t i = s / n3, t = s - i * n3, fb = (size_t)(10 + 4 * i) * n3 + t;
    T q[4];
    for (int c = 0; c < 4; ++c) q[c] = T((double)f[fb + c * n3], (double)df[fb + c * n3]);
    const T r = 1.0 / sqrt(((q[0] * q[0] + q[1] * q[1]) + q[2] * q[2]) + q[3] * q[3]);
    for (int c = 0; c < 4; ++c) {
      const T u = q[c] * r;
      f[fb + c * n3] = (S)u.v;
      df[fb + c * n3] = (S)u.d;
    }
  }
}

} // namespace su2d
} // namespace clb
