// clb_tangent.cuh - first-order dual numbers for the forward-mode (tangent-linear) evolution.
//
// Tan<T> carries a value and its derivative along one direction (a coupling, through the state).
// Every operation forms the value part with exactly the operation of plain T arithmetic, in the
// same order, so a kernel instantiated on Tan<T> reproduces the plain kernel's values bitwise
// (the units that use it are compiled without FMA contraction) while the derivative part follows
// the chain rule.
#pragma once

#include <cmath>

namespace clb {

// The Tan overloads below share their names with the math library's; these declarations keep the
// plain overloads visible to unqualified calls inside namespace clb.
using ::cos;
using ::pow;
using ::sin;
using ::sqrt;

template <class T> struct Tan {
  T v, d;
  __host__ __device__ Tan() : v(0), d(0) {}
  __host__ __device__ Tan(double x) : v((T)x), d(0) {}
  __host__ __device__ Tan(T x, T dx) : v(x), d(dx) {}
  template <class U> __host__ __device__ explicit Tan(const Tan<U> &o) : v((T)o.v), d((T)o.d) {}
};

template <class T> struct TanTraits {
  static constexpr bool is = false;
  using base = T;
};
template <class U> struct TanTraits<Tan<U>> {
  static constexpr bool is = true;
  using base = U;
};
template <class T> struct Id {
  using type = T;
};

template <class T> __host__ __device__ __forceinline__ Tan<T> operator-(Tan<T> a) { return Tan<T>(-a.v, -a.d); }
template <class T> __host__ __device__ __forceinline__ Tan<T> operator+(Tan<T> a, Tan<T> b)
{
  return Tan<T>(a.v + b.v, a.d + b.d);
}
template <class T> __host__ __device__ __forceinline__ Tan<T> operator-(Tan<T> a, Tan<T> b)
{
  return Tan<T>(a.v - b.v, a.d - b.d);
}
template <class T> __host__ __device__ __forceinline__ Tan<T> operator*(Tan<T> a, Tan<T> b)
{
  return Tan<T>(a.v * b.v, a.d * b.v + a.v * b.d);
}
template <class T> __host__ __device__ __forceinline__ Tan<T> operator/(Tan<T> a, Tan<T> b)
{
  const T q = a.v / b.v;
  return Tan<T>(q, (a.d - q * b.d) / b.v);
}
// mixed forms with a plain constant (int, float and double literals convert to T)
template <class T> __host__ __device__ __forceinline__ Tan<T> operator+(Tan<T> a, typename Id<T>::type s)
{
  return Tan<T>(a.v + s, a.d);
}
template <class T> __host__ __device__ __forceinline__ Tan<T> operator+(typename Id<T>::type s, Tan<T> a)
{
  return Tan<T>(s + a.v, a.d);
}
template <class T> __host__ __device__ __forceinline__ Tan<T> operator-(Tan<T> a, typename Id<T>::type s)
{
  return Tan<T>(a.v - s, a.d);
}
template <class T> __host__ __device__ __forceinline__ Tan<T> operator-(typename Id<T>::type s, Tan<T> a)
{
  return Tan<T>(s - a.v, -a.d);
}
template <class T> __host__ __device__ __forceinline__ Tan<T> operator*(Tan<T> a, typename Id<T>::type s)
{
  return Tan<T>(a.v * s, a.d * s);
}
template <class T> __host__ __device__ __forceinline__ Tan<T> operator*(typename Id<T>::type s, Tan<T> a)
{
  return Tan<T>(s * a.v, s * a.d);
}
template <class T> __host__ __device__ __forceinline__ Tan<T> operator/(Tan<T> a, typename Id<T>::type s)
{
  return Tan<T>(a.v / s, a.d / s);
}
template <class T> __host__ __device__ __forceinline__ Tan<T> operator/(typename Id<T>::type s, Tan<T> a)
{
  const T q = s / a.v;
  return Tan<T>(q, -q * a.d / a.v);
}
template <class T> __host__ __device__ __forceinline__ Tan<T> &operator+=(Tan<T> &a, Tan<T> b)
{
  a = a + b;
  return a;
}

template <class T> __host__ __device__ __forceinline__ Tan<T> sqrt(Tan<T> a)
{
  const T r = ::sqrt(a.v);
  return Tan<T>(r, a.d / (2 * r));
}
template <class T> __host__ __device__ __forceinline__ Tan<T> sin(Tan<T> a)
{
  return Tan<T>(::sin(a.v), ::cos(a.v) * a.d);
}
template <class T> __host__ __device__ __forceinline__ Tan<T> cos(Tan<T> a)
{
  return Tan<T>(::cos(a.v), -::sin(a.v) * a.d);
}
template <class T> __host__ __device__ __forceinline__ Tan<T> pow(Tan<T> a, typename Id<T>::type e)
{
  return Tan<T>(::pow(a.v, e), e * ::pow(a.v, e - 1) * a.d);
}

__host__ __device__ __forceinline__ double val(double x) { return x; }
__host__ __device__ __forceinline__ float val(float x) { return x; }
template <class T> __host__ __device__ __forceinline__ T val(Tan<T> x) { return x.v; }
__host__ __device__ __forceinline__ double der(double) { return 0; }
template <class T> __host__ __device__ __forceinline__ T der(Tan<T> x) { return x.d; }
__host__ __device__ __forceinline__ bool finite_(double x)
{
#ifdef __CUDA_ARCH__
  return isfinite(x);
#else
  return std::isfinite(x);
#endif
}
template <class T> __host__ __device__ __forceinline__ bool finite_(Tan<T> x) { return finite_(x.v) && finite_(x.d); }

} // namespace clb
