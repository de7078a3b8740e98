// model_api.h - what a scalar-singlet model header provides to libclb200, in the shape of
// CosmoInterface's model headers (abstractmodel.h:35-98; models/lphi4.h, models/tanh2.h).
//
// A model header defines one struct M with
//   static constexpr const char *name;
//   static constexpr int NScalarsMax;           the singlet count of the header (1 or 2 used)
//   struct Couplings;                           the program-unit couplings the terms read (FP64,
//                                               at most 8 doubles; a term of storage type R rounds
//                                               them to R)
//   static Couplings couplings(const double *c);   from clb_model_desc::couplings
//   template <class A, class R, int NS> static R potentialTerms(Tag<k>, const R (&phi)[NS], const Couplings<R> &);
//   template <class A, class R, int NS> static R potDeriv(Tag<f>, const R (&phi)[NS], const Couplings<R> &);
//   template <class A, class R, int NS> static R potDeriv2(Tag<f>, const R (&phi)[NS], const Couplings<R> &);
// for k < NPotTerms<NS> and f < NS, each evaluated at one site in program variables, with the
// arithmetic policy A (A::add, A::sub, A::mul; the FP64 sweeps pass one that pins every rounding).
// Optionally, for FP32 storage of fluctuations s about an FP64 homogeneous value (one field):
//   struct Fluct { static Fluct make(double phi_r, const Couplings &);
//                  float dV(float s) const;  (potDeriv(phi_r + s) - potDeriv(phi_r))
//                  float V(float s) const; } (potential(phi_r + s) - potential(phi_r))
// Without it the FP32 form takes both differences in FP64 at every site.
//
// The header that the scalar-singlet kernels use is chosen when the library is built
// (CLB_SCALAR_MODEL_HEADER, CLB_SCALAR_MODEL; python -m cosmolattice_b200.build --scalar-model
// NAME), as the reference chooses its model when it compiles (CMakeLists.txt:133-146).
#pragma once

#if defined(__CUDACC__)
#define CLB_MD __host__ __device__ __forceinline__
#else
#define CLB_MD inline
#endif

namespace clb_models {

template <int K> struct Tag {};

// plain arithmetic (host, and the FP32 device forms)
struct PlainOps {
  template <class R> static CLB_MD R add(R a, R b) { return a + b; }
  template <class R> static CLB_MD R sub(R a, R b) { return a - b; }
  template <class R> static CLB_MD R mul(R a, R b) { return a * b; }
};

template <class A, class R> CLB_MD R pow2(R x) { return A::mul(x, x); }
template <class A, class R> CLB_MD R pow3(R x) { return A::mul(A::mul(x, x), x); }
template <class A, class R> CLB_MD R pow4(R x) { return A::mul(A::mul(A::mul(x, x), x), x); }

// run-time term / field index over the header's Tag overloads
template <class M, class A, class R, int NS, class C> CLB_MD R potential_term(int k, const R (&v)[NS], const C &c)
{
  if (k == 0) return M::template potentialTerms<A>(Tag<0>{}, v, c);
  if constexpr (M::template NPotTerms<NS> > 1)
    if (k == 1) return M::template potentialTerms<A>(Tag<1>{}, v, c);
  return R(0);
}
template <class M, class A, class R, int NS, class C> CLB_MD R potential(const R (&v)[NS], const C &c)
{
  R r = M::template potentialTerms<A>(Tag<0>{}, v, c);
  if constexpr (M::template NPotTerms<NS> > 1) r = A::add(r, M::template potentialTerms<A>(Tag<1>{}, v, c));
  return r;
}
template <class M, class A, class R, int NS, class C> CLB_MD R pot_deriv(int f, const R (&v)[NS], const C &c)
{
  if constexpr (NS > 1)
    if (f == 1) return M::template potDeriv<A>(Tag<1>{}, v, c);
  return M::template potDeriv<A>(Tag<0>{}, v, c);
}
template <class M, class A, class R, int NS, class C> CLB_MD R pot_deriv2(int f, const R (&v)[NS], const C &c)
{
  if constexpr (NS > 1)
    if (f == 1) return M::template potDeriv2<A>(Tag<1>{}, v, c);
  return M::template potDeriv2<A>(Tag<0>{}, v, c);
}

// whether M provides the FP32 fluctuation form
template <class M, class = void> struct HasFluct {
  static constexpr bool value = false;
};
template <class M> struct HasFluct<M, decltype((void)sizeof(typename M::Fluct), void())> {
  static constexpr bool value = true;
};

} // namespace clb_models
