// tanh2.h - the tanh2 model header (CosmoLattice models/tanh2.h) for libclb200: an inflaton phi
// with a T-model potential and a daughter field chi,
//   V = (M/phi_i)^2 tanh^2(phi phi_i / M) / 2 + q/2 phi^2 chi^2
// in program variables (alpha = 0, fStar = phi_i, omegaStar = sqrt(Lambda4) / M; tanh2.h constructor),
// with the derivatives as that header writes them (potDeriv(Tag<0>) = 2 (M/phi_i) tanh^2(x) /
// sinh(2x) + q phi chi^2, x = phi phi_i / M; potDeriv2(Tag<0>) = 4 (2 - cosh 2x) tanh^2 x /
// sinh^2 2x + q chi^2).  The couplings (clb_model_desc) are {M/phi_i, q}.  It has no FP32
// fluctuation form, so FP32 storage takes the potential differences in FP64.
#pragma once

#include "model_api.h"

#include <cmath>

namespace clb_models {

struct tanh2 {
  static constexpr const char *name = "tanh2";
  static constexpr int NScalarsMax = 2;
  template <int NS> static constexpr int NPotTerms = NS;

  struct Couplings {
    double mu, inv_mu, q, q_2; // M/phi_i, phi_i/M, q, q/2
  };
  static CLB_MD Couplings couplings(const double *c) { return {c[0], 1.0 / c[0], c[1], 0.5 * c[1]}; }

  template <class A, class R, int NS, class C = Couplings> static CLB_MD R potentialTerms(Tag<0>, const R (&f)[NS], const C &c)
  {
    using std::tanh;
    const R t = tanh(A::mul(f[0], R(c.inv_mu)));
    return A::mul(A::mul(pow2<A>(R(c.mu)), pow2<A>(t)), R(0.5));
  }
  template <class A, class R, int NS, class C = Couplings> static CLB_MD R potentialTerms(Tag<1>, const R (&f)[NS], const C &c)
  {
    if constexpr (NS > 1) return A::mul(R(c.q_2), pow2<A>(A::mul(f[0], f[1])));
    return R(0);
  }
  template <class A, class R, int NS, class C = Couplings> static CLB_MD R potDeriv(Tag<0>, const R (&f)[NS], const C &c)
  {
    using std::sinh;
    using std::tanh;
    const R x = A::mul(f[0], R(c.inv_mu));
    const R t = tanh(x);
    const R d = A::mul(A::mul(R(2), R(c.mu)), pow2<A>(t)) / sinh(A::mul(R(2), x));
    if constexpr (NS > 1) return A::add(d, A::mul(A::mul(R(c.q), f[0]), pow2<A>(f[1])));
    return d;
  }
  template <class A, class R, int NS, class C = Couplings> static CLB_MD R potDeriv(Tag<1>, const R (&f)[NS], const C &c)
  {
    if constexpr (NS > 1) return A::mul(A::mul(R(c.q), f[1]), pow2<A>(f[0]));
    return R(0);
  }
  template <class A, class R, int NS, class C = Couplings> static CLB_MD R potDeriv2(Tag<0>, const R (&f)[NS], const C &c)
  {
    using std::cosh;
    using std::sinh;
    using std::tanh;
    const R x = A::mul(f[0], R(c.inv_mu));
    const R x2 = A::mul(R(2), x);
    const R d = A::mul(A::mul(R(4), A::sub(R(2), cosh(x2))), pow2<A>(tanh(x))) / pow2<A>(sinh(x2));
    if constexpr (NS > 1) return A::add(d, A::mul(R(c.q), pow2<A>(f[1])));
    return d;
  }
  template <class A, class R, int NS, class C = Couplings> static CLB_MD R potDeriv2(Tag<1>, const R (&f)[NS], const C &c)
  {
    if constexpr (NS > 1) return A::mul(R(c.q), pow2<A>(f[0]));
    return R(0);
  }
};

} // namespace clb_models
