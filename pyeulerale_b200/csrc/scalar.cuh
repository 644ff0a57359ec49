// Forward-mode scalar algebra for the FP64 stencil kernels.
//
// The reference (PyEulerALE `src/spatial_discretization.f90`) differentiates its residual by
// complex step: every Jacobian column is `aimag(make_ode(x + i*h*e))/h` with h = 1e-12
// (f90:52-53). Here derivatives come from dual numbers instead: `Dual<T, K>` carries a value
// and K tangent components, all of type T. Nesting (`Dual<Dual<double, 2>, 4>`) gives exact
// mixed second derivatives, which replace the reference's finite differences of complex-step
// Jacobians (`core.py:718-1275`).
//
// Arithmetic between different scalar types is allowed when one embeds into the other
// (double -> Dual<double,K>, Dual<double,2> -> Dual<Dual<double,2>,4>, ...): the lower operand
// is treated as a constant. The two branch primitives of the reference keep its semantics:
//   abs_c(x): derivative sign taken from the sign of Re x (f90:97-102), zeros as positive;
//   max_c(x, y): x only if Re x > Re y + 1e-8 (f90:111-120), tangents follow the selection.
#pragma once

#include <cuda_runtime.h>
#include <type_traits>

#define EB_HD __host__ __device__ __forceinline__

namespace eb {

template <class T, int K>
struct Dual {
  T v;
  T d[K];
};

template <class T>
struct is_dual : std::false_type {};
template <class T, int K>
struct is_dual<Dual<T, K>> : std::true_type {};

// embeds<S, D>: S is D itself or a scalar nested inside D.
template <class S, class D>
struct embeds : std::is_same<S, D> {};
template <class S, class T, int K>
struct embeds<S, Dual<T, K>>
    : std::integral_constant<bool, std::is_same<S, Dual<T, K>>::value || embeds<S, T>::value> {};

// promote<A, B>: the larger of two comparable scalar types.
template <class A, class B, class = void>
struct promote;
template <class A, class B>
struct promote<A, B, std::enable_if_t<embeds<A, B>::value>> {
  using type = B;
};
template <class A, class B>
struct promote<A, B, std::enable_if_t<!embeds<A, B>::value && embeds<B, A>::value>> {
  using type = A;
};
template <class A, class B>
using promote_t = typename promote<A, B>::type;

// lift<D>(s): the embedding of a lower scalar s into D with zero tangents.
template <class D, class S>
EB_HD std::enable_if_t<std::is_same<D, S>::value, D> lift(const S& s) {
  return s;
}
template <class D, class S>
EB_HD std::enable_if_t<!std::is_same<D, S>::value && is_dual<D>::value, D> lift(const S& s) {
  D r;
  r.v = lift<decltype(r.v)>(s);
#pragma unroll
  for (int i = 0; i < (int)(sizeof(r.d) / sizeof(r.d[0])); ++i) r.d[i] = lift<decltype(r.v)>(0.0);
  return r;
}

// value(x): the plain double value.
EB_HD double value(double x) { return x; }
template <class T, int K>
EB_HD double value(const Dual<T, K>& x) {
  return value(x.v);
}

// ---- Dual (op) Dual ------------------------------------------------------------------------
template <class T, int K>
EB_HD Dual<T, K> operator+(const Dual<T, K>& a, const Dual<T, K>& b) {
  Dual<T, K> r;
  r.v = a.v + b.v;
#pragma unroll
  for (int i = 0; i < K; ++i) r.d[i] = a.d[i] + b.d[i];
  return r;
}
template <class T, int K>
EB_HD Dual<T, K> operator-(const Dual<T, K>& a, const Dual<T, K>& b) {
  Dual<T, K> r;
  r.v = a.v - b.v;
#pragma unroll
  for (int i = 0; i < K; ++i) r.d[i] = a.d[i] - b.d[i];
  return r;
}
template <class T, int K>
EB_HD Dual<T, K> operator-(const Dual<T, K>& a) {
  Dual<T, K> r;
  r.v = -a.v;
#pragma unroll
  for (int i = 0; i < K; ++i) r.d[i] = -a.d[i];
  return r;
}
template <class T, int K>
EB_HD Dual<T, K> operator*(const Dual<T, K>& a, const Dual<T, K>& b) {
  Dual<T, K> r;
  r.v = a.v * b.v;
#pragma unroll
  for (int i = 0; i < K; ++i) r.d[i] = a.d[i] * b.v + a.v * b.d[i];
  return r;
}
template <class T, int K>
EB_HD Dual<T, K> operator/(const Dual<T, K>& a, const Dual<T, K>& b) {
  Dual<T, K> r;
  r.v = a.v / b.v;
#pragma unroll
  for (int i = 0; i < K; ++i) r.d[i] = (a.d[i] - r.v * b.d[i]) / b.v;
  return r;
}

// ---- Dual (op) lower scalar and lower scalar (op) Dual ------------------------------------
#define EB_LOWER(S, T) std::enable_if_t<embeds<S, T>::value, int> = 0

template <class T, int K, class S, EB_LOWER(S, T)>
EB_HD Dual<T, K> operator+(const Dual<T, K>& a, const S& b) {
  Dual<T, K> r = a;
  r.v = a.v + b;
  return r;
}
template <class T, int K, class S, EB_LOWER(S, T)>
EB_HD Dual<T, K> operator+(const S& a, const Dual<T, K>& b) {
  Dual<T, K> r = b;
  r.v = a + b.v;
  return r;
}
template <class T, int K, class S, EB_LOWER(S, T)>
EB_HD Dual<T, K> operator-(const Dual<T, K>& a, const S& b) {
  Dual<T, K> r = a;
  r.v = a.v - b;
  return r;
}
template <class T, int K, class S, EB_LOWER(S, T)>
EB_HD Dual<T, K> operator-(const S& a, const Dual<T, K>& b) {
  Dual<T, K> r;
  r.v = a - b.v;
#pragma unroll
  for (int i = 0; i < K; ++i) r.d[i] = -b.d[i];
  return r;
}
template <class T, int K, class S, EB_LOWER(S, T)>
EB_HD Dual<T, K> operator*(const Dual<T, K>& a, const S& b) {
  Dual<T, K> r;
  r.v = a.v * b;
#pragma unroll
  for (int i = 0; i < K; ++i) r.d[i] = a.d[i] * b;
  return r;
}
template <class T, int K, class S, EB_LOWER(S, T)>
EB_HD Dual<T, K> operator*(const S& a, const Dual<T, K>& b) {
  Dual<T, K> r;
  r.v = a * b.v;
#pragma unroll
  for (int i = 0; i < K; ++i) r.d[i] = a * b.d[i];
  return r;
}
template <class T, int K, class S, EB_LOWER(S, T)>
EB_HD Dual<T, K> operator/(const Dual<T, K>& a, const S& b) {
  Dual<T, K> r;
  r.v = a.v / b;
#pragma unroll
  for (int i = 0; i < K; ++i) r.d[i] = a.d[i] / b;
  return r;
}
template <class T, int K, class S, EB_LOWER(S, T)>
EB_HD Dual<T, K> operator/(const S& a, const Dual<T, K>& b) {
  Dual<T, K> r;
  r.v = a / b.v;
#pragma unroll
  for (int i = 0; i < K; ++i) r.d[i] = -(r.v * b.d[i]) / b.v;
  return r;
}
#undef EB_LOWER

// ---- elementary functions ------------------------------------------------------------------
EB_HD double sqrt_(double x) { return ::sqrt(x); }
template <class T, int K>
EB_HD Dual<T, K> sqrt_(const Dual<T, K>& a) {
  Dual<T, K> r;
  r.v = sqrt_(a.v);
  T two_r = 2.0 * r.v;
#pragma unroll
  for (int i = 0; i < K; ++i) r.d[i] = a.d[i] / two_r;
  return r;
}

// abs_c, f90:97-102: value |x|, derivative times sign(1, Re x). The reference evaluates the
// argument in complex arithmetic, where an exact cancellation (p - 2p + p at a uniform state)
// and a quotient with a zero numerator (Smith's division adds a +0 term) come out as +0; in
// real arithmetic the same values can come out as -0 depending on how the compiler contracts
// the expression. Both zeros therefore count as positive here, which is what the reference
// sees at such degenerate points (e.g. an exact free stream).
EB_HD double abs_c(double x) { return ::fabs(x); }
template <class T, int K>
EB_HD Dual<T, K> abs_c(const Dual<T, K>& a) {
  Dual<T, K> r;
  const double s = value(a) < 0.0 ? -1.0 : 1.0;
  r.v = abs_c(a.v);
#pragma unroll
  for (int i = 0; i < K; ++i) r.d[i] = a.d[i] * s;
  return r;
}

// max_c, f90:111-120: returns x only if Re x > Re y + 1e-8, else y (asymmetric on purpose).
template <class A, class B>
EB_HD promote_t<A, B> max_c(const A& x, const B& y) {
  using R = promote_t<A, B>;
  return (value(x) > value(y) + 1e-8) ? lift<R>(x) : lift<R>(y);
}

}  // namespace eb
