// lphi4.h - the lphi4 model header (CosmoLattice models/lphi4.h:154-226) for libclb200: two real
// scalars phi, chi with V = c0/4 phi^4 + q/2 phi^2 chi^2 in program variables (lambda absorbed into
// omegaStar = sqrt(lambda) phi0, lphi4.h:125-127; c0 = lambda_prog, 1 in the reference header).
// With one field the daughter chi is absent.  The terms are written in the rounding order the
// FP64 sweeps and the oracle share: (c0/4) ((phi phi) phi) phi, (q/2) (phi chi)^2, c0 (phi phi) phi
// + (q phi) chi^2, (q chi) phi^2.
#pragma once

#include "model_api.h"

namespace clb_models {

struct lphi4 {
  static constexpr const char *name = "lphi4";
  static constexpr int NScalarsMax = 2;
  template <int NS> static constexpr int NPotTerms = NS; // the q term needs the daughter field

  // c0, q and the factors c0/4, q/2 the terms multiply by (clb_model_desc couplings {c0, q}); a
  // term of storage type R reads them rounded to R
  struct Couplings {
    double c0, q, c0_4, q_2;
  };
  static CLB_MD Couplings couplings(const double *c) { return {c[0], c[1], 0.25 * c[0], 0.5 * c[1]}; }

  // potentialTerms(Tag<0>): lphi4.h:161-166; potentialTerms(Tag<1>): lphi4.h:173-178
  template <class A, class R, int NS, class C = Couplings> static CLB_MD R potentialTerms(Tag<0>, const R (&f)[NS], const C &c)
  {
    return A::mul(R(c.c0_4), pow4<A>(f[0]));
  }
  template <class A, class R, int NS, class C = Couplings> static CLB_MD R potentialTerms(Tag<1>, const R (&f)[NS], const C &c)
  {
    if constexpr (NS > 1) return A::mul(R(c.q_2), pow2<A>(A::mul(f[0], f[1])));
    return R(0);
  }
  // potDeriv(Tag<0>), (Tag<1>): lphi4.h:195-206
  template <class A, class R, int NS, class C = Couplings> static CLB_MD R potDeriv(Tag<0>, const R (&f)[NS], const C &c)
  {
    if constexpr (NS > 1) return A::add(A::mul(R(c.c0), pow3<A>(f[0])), A::mul(A::mul(R(c.q), f[0]), pow2<A>(f[1])));
    return A::mul(R(c.c0), pow3<A>(f[0]));
  }
  template <class A, class R, int NS, class C = Couplings> static CLB_MD R potDeriv(Tag<1>, const R (&f)[NS], const C &c)
  {
    if constexpr (NS > 1) return A::mul(A::mul(R(c.q), f[1]), pow2<A>(f[0]));
    return R(0);
  }
  // potDeriv2(Tag<0>), (Tag<1>): lphi4.h:213-226
  template <class A, class R, int NS, class C = Couplings> static CLB_MD R potDeriv2(Tag<0>, const R (&f)[NS], const C &c)
  {
    const R t = A::mul(A::mul(R(3), R(c.c0)), pow2<A>(f[0]));
    if constexpr (NS > 1) return A::add(t, A::mul(R(c.q), pow2<A>(f[1])));
    return t;
  }
  template <class A, class R, int NS, class C = Couplings> static CLB_MD R potDeriv2(Tag<1>, const R (&f)[NS], const C &c)
  {
    if constexpr (NS > 1) return A::mul(R(c.q), pow2<A>(f[0]));
    return R(0);
  }

  // FP32 fluctuation form (one field): with s the fluctuation about phi_r, the exact polynomial
  // differences
  //   potDeriv(phi_r + s) - potDeriv(phi_r) = s (a1 + s (a2 + c0 s)),  a1 = 3 c0 phi_r^2, a2 = 3 c0 phi_r
  //   V(phi_r + s) - V(phi_r) = s (b1 + s (b2 + s (b3 + c0/4 s))),     b1 = c0 phi_r^3,
  //                                                                  b2 = 3/2 c0 phi_r^2, b3 = c0 phi_r
  // evaluated in FP32 (relative precision of the fluctuation's own force and energy).
  struct Fluct {
    float a1, a2, c0, b1, b2, b3, c0q;
    template <class C> static CLB_MD Fluct make(double phi_r, const C &c)
    {
      const double k = c.c0;
      Fluct r;
      r.a1 = (float)(3.0 * k * phi_r * phi_r);
      r.a2 = (float)(3.0 * k * phi_r);
      r.c0 = (float)k;
      r.b1 = (float)(k * phi_r * phi_r * phi_r);
      r.b2 = (float)(1.5 * k * phi_r * phi_r);
      r.b3 = (float)(k * phi_r);
      r.c0q = (float)(0.25 * k);
      return r;
    }
#if defined(__CUDACC__)
    __device__ __forceinline__ float dV(float s) const { return s * fmaf(s, fmaf(c0, s, a2), a1); }
    __device__ __forceinline__ float V(float s) const { return s * fmaf(s, fmaf(s, fmaf(c0q, s, b3), b2), b1); }
#endif
  };
};

} // namespace clb_models
