// Per-opcode semantics on the device for the three value kinds the interpreter
// carries per slot:
//   * T            — plain float/double (forward, gradient),
//   * Dual<T>      — value + tangent (JVP forward, HVP forward-over-reverse),
//   * Jet<T,K>     — K Taylor coefficients c_k = f^(k)/k! (Taylor / STDE).
//
// The formulas restate the reference's CPU semantics so GPU results agree with
// the f64 tape to the stated tolerances:
//   scalar forward / partials      src/opcode.rs:228-535, src/kernels/mod.rs:85-285
//   Dual arithmetic + elementals   src/dual.rs:40-464, src/traits/std_ops.rs:14-82
//   Taylor coefficient recurrences src/taylor_ops.rs:18-916, src/taylor.rs:180-370
// Arithmetic order is kept (the library is built with -fmad=false), so +,-,*,/
// and sqrt round exactly like the CPU; libm-backed functions use CUDA's math
// library and differ from glibc by its documented ulp bounds.
#pragma once
#include <stdint.h>
#include <math.h>
#include "ech_types.h"

namespace ech {
namespace dm {

// ───────────────────────────── scalar math by precision ────────────────────
template <class T> struct fm;
template <> struct fm<double> {
  static __device__ __forceinline__ double exp(double x) { return ::exp(x); }
  static __device__ __forceinline__ double exp2(double x) { return ::exp2(x); }
  static __device__ __forceinline__ double expm1(double x) { return ::expm1(x); }
  static __device__ __forceinline__ double log(double x) { return ::log(x); }
  static __device__ __forceinline__ double log2(double x) { return ::log2(x); }
  static __device__ __forceinline__ double log10(double x) { return ::log10(x); }
  static __device__ __forceinline__ double log1p(double x) { return ::log1p(x); }
  static __device__ __forceinline__ double sin(double x) { return ::sin(x); }
  static __device__ __forceinline__ double cos(double x) { return ::cos(x); }
  static __device__ __forceinline__ double tan(double x) { return ::tan(x); }
  static __device__ __forceinline__ double asin(double x) { return ::asin(x); }
  static __device__ __forceinline__ double acos(double x) { return ::acos(x); }
  static __device__ __forceinline__ double atan(double x) { return ::atan(x); }
  static __device__ __forceinline__ double sinh(double x) { return ::sinh(x); }
  static __device__ __forceinline__ double cosh(double x) { return ::cosh(x); }
  static __device__ __forceinline__ double tanh(double x) { return ::tanh(x); }
  static __device__ __forceinline__ double asinh(double x) { return ::asinh(x); }
  static __device__ __forceinline__ double acosh(double x) { return ::acosh(x); }
  static __device__ __forceinline__ double atanh(double x) { return ::atanh(x); }
  static __device__ __forceinline__ double sqrt(double x) { return ::sqrt(x); }
  static __device__ __forceinline__ double cbrt(double x) { return ::cbrt(x); }
  static __device__ __forceinline__ double pow(double x, double y) { return ::pow(x, y); }
  static __device__ __forceinline__ double atan2(double x, double y) { return ::atan2(x, y); }
  static __device__ __forceinline__ double hypot(double x, double y) { return ::hypot(x, y); }
  static __device__ __forceinline__ double fmod(double x, double y) { return ::fmod(x, y); }
  static __device__ __forceinline__ double fabs(double x) { return ::fabs(x); }
  static __device__ __forceinline__ double floor(double x) { return ::floor(x); }
  static __device__ __forceinline__ double ceil(double x) { return ::ceil(x); }
  static __device__ __forceinline__ double round(double x) { return ::round(x); }
  static __device__ __forceinline__ double trunc(double x) { return ::trunc(x); }
  static __device__ __forceinline__ double copysign(double x, double y) { return ::copysign(x, y); }
  static __device__ __forceinline__ double fmax(double x, double y) { return ::fmax(x, y); }
  static __device__ __forceinline__ double nan() { return __longlong_as_double(0x7ff8000000000000ll); }
  static __device__ __forceinline__ double inf() { return __longlong_as_double(0x7ff0000000000000ll); }
  static constexpr double LN2 = 0.693147180559945309417232121458176568;
  static constexpr double LN10 = 2.302585092994045684017991454684364208;
};
template <> struct fm<float> {
  static __device__ __forceinline__ float exp(float x) { return ::expf(x); }
  static __device__ __forceinline__ float exp2(float x) { return ::exp2f(x); }
  static __device__ __forceinline__ float expm1(float x) { return ::expm1f(x); }
  static __device__ __forceinline__ float log(float x) { return ::logf(x); }
  static __device__ __forceinline__ float log2(float x) { return ::log2f(x); }
  static __device__ __forceinline__ float log10(float x) { return ::log10f(x); }
  static __device__ __forceinline__ float log1p(float x) { return ::log1pf(x); }
  static __device__ __forceinline__ float sin(float x) { return ::sinf(x); }
  static __device__ __forceinline__ float cos(float x) { return ::cosf(x); }
  static __device__ __forceinline__ float tan(float x) { return ::tanf(x); }
  static __device__ __forceinline__ float asin(float x) { return ::asinf(x); }
  static __device__ __forceinline__ float acos(float x) { return ::acosf(x); }
  static __device__ __forceinline__ float atan(float x) { return ::atanf(x); }
  static __device__ __forceinline__ float sinh(float x) { return ::sinhf(x); }
  static __device__ __forceinline__ float cosh(float x) { return ::coshf(x); }
  static __device__ __forceinline__ float tanh(float x) { return ::tanhf(x); }
  static __device__ __forceinline__ float asinh(float x) { return ::asinhf(x); }
  static __device__ __forceinline__ float acosh(float x) { return ::acoshf(x); }
  static __device__ __forceinline__ float atanh(float x) { return ::atanhf(x); }
  static __device__ __forceinline__ float sqrt(float x) { return ::sqrtf(x); }
  static __device__ __forceinline__ float cbrt(float x) { return ::cbrtf(x); }
  static __device__ __forceinline__ float pow(float x, float y) { return ::powf(x, y); }
  static __device__ __forceinline__ float atan2(float x, float y) { return ::atan2f(x, y); }
  static __device__ __forceinline__ float hypot(float x, float y) { return ::hypotf(x, y); }
  static __device__ __forceinline__ float fmod(float x, float y) { return ::fmodf(x, y); }
  static __device__ __forceinline__ float fabs(float x) { return ::fabsf(x); }
  static __device__ __forceinline__ float floor(float x) { return ::floorf(x); }
  static __device__ __forceinline__ float ceil(float x) { return ::ceilf(x); }
  static __device__ __forceinline__ float round(float x) { return ::roundf(x); }
  static __device__ __forceinline__ float trunc(float x) { return ::truncf(x); }
  static __device__ __forceinline__ float copysign(float x, float y) { return ::copysignf(x, y); }
  static __device__ __forceinline__ float fmax(float x, float y) { return ::fmaxf(x, y); }
  static __device__ __forceinline__ float nan() { return __int_as_float(0x7fc00000); }
  static __device__ __forceinline__ float inf() { return __int_as_float(0x7f800000); }
  static constexpr double LN2 = 0.693147180559945309417232121458176568;
  static constexpr double LN10 = 2.302585092994045684017991454684364208;
};

template <class T> __device__ __forceinline__ bool isnan_(T x) { return x != x; }
template <class T> __device__ __forceinline__ bool isfinite_(T x) { return fm<T>::fabs(x) <= fm<T>::fmax(x, -x) && !(fm<T>::fabs(x) == fm<T>::inf()) && x == x; }
template <> __device__ __forceinline__ bool isfinite_<double>(double x) { return ::isfinite(x); }
template <> __device__ __forceinline__ bool isfinite_<float>(float x) { return ::isfinite(x); }

// Rust powi lowers to square-and-multiply (binary exponentiation).
template <class T> __device__ __forceinline__ T powi_s(T a, int32_t n) {
  const bool recip = n < 0;
  uint32_t m = n < 0 ? (uint32_t)(-(int64_t)n) : (uint32_t)n;
  T r = T(1);
  for (;;) {
    if (m & 1u) r = r * a;
    m >>= 1;
    if (m == 0) break;
    a = a * a;
  }
  return recip ? T(1) / r : r;
}
template <class T> __device__ __forceinline__ T signum_s(T x) { return isnan_(x) ? x : fm<T>::copysign(T(1), x); }
template <class T> __device__ __forceinline__ T fract_s(T x) { return x - fm<T>::trunc(x); }
// num_traits to_i32 plus the integrality test (src/dual.rs:364-369).
template <class T> __device__ __forceinline__ bool as_i32(T x, int32_t* out) {
  if (!(x > T(-2147483649.0) && x < T(2147483648.0))) return false;
  int32_t ni = (int32_t)x;
  if ((T)ni != x) return false;
  *out = ni;
  return true;
}

// ───────────────────────────── value kinds ──────────────────────────────────
template <class T> struct Dual {
  T re, eps;
};
template <class T, int K> struct Jet {
  T c[K];
};

template <class V> struct VT;  // value traits: scalar type, primal, constants
template <> struct VT<double> {
  using S = double;
  static __device__ __forceinline__ double prim(double x) { return x; }
  static __device__ __forceinline__ double cst(double v) { return v; }
  static __device__ __forceinline__ double cst_s(double v) { return v; }
};
template <> struct VT<float> {
  using S = float;
  static __device__ __forceinline__ float prim(float x) { return x; }
  static __device__ __forceinline__ float cst(double v) { return (float)v; }
  static __device__ __forceinline__ float cst_s(float v) { return v; }
};
template <class T> struct VT<Dual<T>> {
  using S = T;
  static __device__ __forceinline__ T prim(const Dual<T>& x) { return x.re; }
  static __device__ __forceinline__ Dual<T> cst(double v) { return {(T)v, T(0)}; }
  static __device__ __forceinline__ Dual<T> cst_s(T v) { return {v, T(0)}; }
};
template <class T, int K> struct VT<Jet<T, K>> {
  using S = T;
  static __device__ __forceinline__ T prim(const Jet<T, K>& x) { return x.c[0]; }
  static __device__ __forceinline__ Jet<T, K> cst_s(T v) {
    Jet<T, K> j;
    j.c[0] = v;
#pragma unroll
    for (int k = 1; k < K; ++k) j.c[k] = T(0);
    return j;
  }
  static __device__ __forceinline__ Jet<T, K> cst(double v) {
    Jet<T, K> j;
    j.c[0] = (T)v;
#pragma unroll
    for (int k = 1; k < K; ++k) j.c[k] = T(0);
    return j;
  }
};

// ───────────────────────────── scalar kind ──────────────────────────────────
template <class T> struct SK {
  using V = T;
  static __device__ __forceinline__ V c(double v) { return (T)v; }
  static __device__ __forceinline__ V add(V a, V b) { return a + b; }
  static __device__ __forceinline__ V sub(V a, V b) { return a - b; }
  static __device__ __forceinline__ V mul(V a, V b) { return a * b; }
  static __device__ __forceinline__ V div(V a, V b) { return a / b; }
  static __device__ __forceinline__ V neg(V a) { return -a; }
  static __device__ __forceinline__ V rem(V a, V b) { return fm<T>::fmod(a, b); }
  static __device__ __forceinline__ V powf(V a, V b) { return fm<T>::pow(a, b); }
  static __device__ __forceinline__ V atan2(V a, V b) { return fm<T>::atan2(a, b); }
  static __device__ __forceinline__ V hypot(V a, V b) { return fm<T>::hypot(a, b); }
  static __device__ __forceinline__ V recip(V a) { return T(1) / a; }
  static __device__ __forceinline__ V sqrt(V a) { return fm<T>::sqrt(a); }
  static __device__ __forceinline__ V cbrt(V a) { return fm<T>::cbrt(a); }
  static __device__ __forceinline__ V powi(V a, int32_t n) { return powi_s(a, n); }
  static __device__ __forceinline__ V exp(V a) { return fm<T>::exp(a); }
  static __device__ __forceinline__ V exp2(V a) { return fm<T>::exp2(a); }
  static __device__ __forceinline__ V exp_m1(V a) { return fm<T>::expm1(a); }
  static __device__ __forceinline__ V ln(V a) { return fm<T>::log(a); }
  static __device__ __forceinline__ V log2(V a) { return fm<T>::log2(a); }
  static __device__ __forceinline__ V log10(V a) { return fm<T>::log10(a); }
  static __device__ __forceinline__ V ln_1p(V a) { return fm<T>::log1p(a); }
  static __device__ __forceinline__ V sin(V a) { return fm<T>::sin(a); }
  static __device__ __forceinline__ V cos(V a) { return fm<T>::cos(a); }
  static __device__ __forceinline__ V tan(V a) { return fm<T>::tan(a); }
  static __device__ __forceinline__ V asin(V a) { return fm<T>::asin(a); }
  static __device__ __forceinline__ V acos(V a) { return fm<T>::acos(a); }
  static __device__ __forceinline__ V atan(V a) { return fm<T>::atan(a); }
  static __device__ __forceinline__ V sinh(V a) { return fm<T>::sinh(a); }
  static __device__ __forceinline__ V cosh(V a) { return fm<T>::cosh(a); }
  static __device__ __forceinline__ V tanh(V a) { return fm<T>::tanh(a); }
  static __device__ __forceinline__ V asinh(V a) { return fm<T>::asinh(a); }
  static __device__ __forceinline__ V acosh(V a) { return fm<T>::acosh(a); }
  static __device__ __forceinline__ V atanh(V a) { return fm<T>::atanh(a); }
  static __device__ __forceinline__ V abs(V a) { return fm<T>::fabs(a); }
  static __device__ __forceinline__ V signum(V a) { return signum_s(a); }
  static __device__ __forceinline__ V floor(V a) { return fm<T>::floor(a); }
  static __device__ __forceinline__ V ceil(V a) { return fm<T>::ceil(a); }
  static __device__ __forceinline__ V round(V a) { return fm<T>::round(a); }
  static __device__ __forceinline__ V trunc(V a) { return fm<T>::trunc(a); }
  static __device__ __forceinline__ V fract(V a) { return fract_s(a); }
  static __device__ __forceinline__ bool all_zero(V a) { return a == T(0); }
  static __device__ __forceinline__ V nan() { return fm<T>::nan(); }
};

// Kind selector.
template <class V> struct KindOf;
template <> struct KindOf<double> { using K = SK<double>; };
template <> struct KindOf<float> { using K = SK<float>; };

// Derivative kernels shared by every kind (src/kernels/mod.rs:85-285).
template <class Kd, class V> __device__ __forceinline__ void hypot_partials(V a, V b, V r, V& da, V& db) {
  using VTV = VT<V>;
  if (VTV::prim(r) == 0) { da = Kd::c(0); db = Kd::c(0); return; }
  da = Kd::div(a, r);
  db = Kd::div(b, r);
}
template <class Kd, class V> __device__ __forceinline__ void atan2_partials(V a, V b, V& da, V& db) {
  using VTV = VT<V>;
  V h = Kd::hypot(a, b);
  if (VTV::prim(h) == 0) { da = Kd::c(0); db = Kd::c(0); return; }
  da = Kd::div(Kd::div(b, h), h);
  db = Kd::div(Kd::div(Kd::neg(a), h), h);
}
template <class Kd, class V> __device__ __forceinline__ V atan_deriv(V a) {
  V one = Kd::c(1);
  if (VT<V>::prim(Kd::abs(a)) > 1e8) {
    V inv = Kd::div(one, a);
    return Kd::div(Kd::mul(inv, inv), Kd::add(one, Kd::mul(inv, inv)));
  }
  return Kd::div(one, Kd::add(one, Kd::mul(a, a)));
}
template <class Kd, class V> __device__ __forceinline__ V asinh_deriv(V a) {
  V one = Kd::c(1);
  if (VT<V>::prim(Kd::abs(a)) > 1e8) {
    V inv = Kd::div(one, a);
    return Kd::div(Kd::abs(inv), Kd::sqrt(Kd::add(one, Kd::mul(inv, inv))));
  }
  return Kd::div(one, Kd::sqrt(Kd::add(Kd::mul(a, a), one)));
}
template <class Kd, class V> __device__ __forceinline__ V acosh_deriv(V a) {
  V one = Kd::c(1);
  if (VT<V>::prim(a) < 1) return Kd::nan();
  if (VT<V>::prim(a) > 1e8) {
    V inv = Kd::div(one, a);
    return Kd::div(Kd::abs(inv), Kd::sqrt(Kd::sub(one, Kd::mul(inv, inv))));
  }
  return Kd::div(one, Kd::sqrt(Kd::mul(Kd::sub(a, one), Kd::add(a, one))));
}
template <class Kd, class V> __device__ __forceinline__ V ln_deriv(V a) {
  if (VT<V>::prim(a) >= 0) return Kd::div(Kd::c(1), a);
  return Kd::nan();
}
template <class Kd, class V> __device__ __forceinline__ V log2_deriv(V a) {
  if (VT<V>::prim(a) >= 0) return Kd::div(Kd::c(1), Kd::mul(a, Kd::c(fm<typename VT<V>::S>::LN2)));
  return Kd::nan();
}
template <class Kd, class V> __device__ __forceinline__ V log10_deriv(V a) {
  if (VT<V>::prim(a) >= 0) return Kd::div(Kd::c(1), Kd::mul(a, Kd::c(fm<typename VT<V>::S>::LN10)));
  return Kd::nan();
}
template <class Kd, class V> __device__ __forceinline__ V ln_1p_deriv(V a) {
  if (VT<V>::prim(a) >= VT<V>::prim(Kd::neg(Kd::c(1)))) return Kd::div(Kd::c(1), Kd::add(Kd::c(1), a));
  return Kd::nan();
}
template <class Kd, class V> __device__ __forceinline__ V atanh_deriv(V a) {
  V one = Kd::c(1);
  auto p = VT<V>::prim(a);
  if (p >= VT<V>::prim(Kd::neg(one)) && p <= VT<V>::prim(one))
    return Kd::div(one, Kd::mul(Kd::sub(one, a), Kd::add(one, a)));
  return Kd::nan();
}
template <class Kd, class V> __device__ __forceinline__ V abs_deriv(V a) {
  if (VT<V>::prim(a) == 0) return Kd::c(0);
  return Kd::signum(a);
}

// ───────────────────────────── Dual kind (src/dual.rs) ──────────────────────
template <class T> struct DK {
  using V = Dual<T>;
  using S = SK<T>;
  static __device__ __forceinline__ V c(double v) { return {(T)v, T(0)}; }
  static __device__ __forceinline__ V c0(T v) { return {v, T(0)}; }
  static __device__ __forceinline__ V add(V a, V b) { return {a.re + b.re, a.eps + b.eps}; }
  static __device__ __forceinline__ V sub(V a, V b) { return {a.re - b.re, a.eps - b.eps}; }
  static __device__ __forceinline__ V mul(V a, V b) { return {a.re * b.re, a.re * b.eps + a.eps * b.re}; }
  static __device__ __forceinline__ V div(V a, V b) {
    T inv = T(1) / b.re;
    T re = a.re / b.re;
    return {re, (a.eps - re * b.eps) * inv};
  }
  static __device__ __forceinline__ V neg(V a) { return {-a.re, -a.eps}; }
  static __device__ __forceinline__ V rem(V a, V b) {
    return {fm<T>::fmod(a.re, b.re), a.eps - b.eps * fm<T>::trunc(a.re / b.re)};
  }
  static __device__ __forceinline__ V chain(V x, T fv, T fd) { return {fv, (x.eps == T(0)) ? T(0) : x.eps * fd}; }
  static __device__ __forceinline__ V recip(V a) { T inv = T(1) / a.re; return chain(a, inv, -inv * inv); }
  static __device__ __forceinline__ V sqrt(V a) {
    T s = fm<T>::sqrt(a.re);
    T two = T(1) + T(1);
    return chain(a, s, T(1) / (two * s));
  }
  static __device__ __forceinline__ V cbrt(V a) {
    T cr = fm<T>::cbrt(a.re);
    return chain(a, cr, T(1) / (T(3) * cr * cr));
  }
  static __device__ __forceinline__ V powi(V a, int32_t n) {
    if (n == 0) return c(1);
    T val = powi_s(a.re, n);
    T deriv = (n == (int32_t)0x80000000) ? T(n) * val / a.re : T(n) * powi_s(a.re, n - 1);
    return chain(a, val, deriv);
  }
  static __device__ __forceinline__ V exp(V a) { T e = fm<T>::exp(a.re); return chain(a, e, e); }
  static __device__ __forceinline__ V exp2(V a) { T e = fm<T>::exp2(a.re); return chain(a, e, e * (T)fm<T>::LN2); }
  static __device__ __forceinline__ V exp_m1(V a) { return chain(a, fm<T>::expm1(a.re), fm<T>::exp(a.re)); }
  static __device__ __forceinline__ V ln(V a) { return chain(a, fm<T>::log(a.re), ln_deriv<S>(a.re)); }
  static __device__ __forceinline__ V log2(V a) { return chain(a, fm<T>::log2(a.re), log2_deriv<S>(a.re)); }
  static __device__ __forceinline__ V log10(V a) { return chain(a, fm<T>::log10(a.re), log10_deriv<S>(a.re)); }
  static __device__ __forceinline__ V ln_1p(V a) { return chain(a, fm<T>::log1p(a.re), ln_1p_deriv<S>(a.re)); }
  static __device__ __forceinline__ V sin(V a) { return chain(a, fm<T>::sin(a.re), fm<T>::cos(a.re)); }
  static __device__ __forceinline__ V cos(V a) { return chain(a, fm<T>::cos(a.re), -fm<T>::sin(a.re)); }
  static __device__ __forceinline__ V tan(V a) { T cc = fm<T>::cos(a.re); return chain(a, fm<T>::tan(a.re), T(1) / (cc * cc)); }
  static __device__ __forceinline__ V asin(V a) {
    return chain(a, fm<T>::asin(a.re), T(1) / fm<T>::sqrt((T(1) - a.re) * (T(1) + a.re)));
  }
  static __device__ __forceinline__ V acos(V a) {
    return chain(a, fm<T>::acos(a.re), -T(1) / fm<T>::sqrt((T(1) - a.re) * (T(1) + a.re)));
  }
  static __device__ __forceinline__ V atan(V a) { return chain(a, fm<T>::atan(a.re), atan_deriv<S>(a.re)); }
  static __device__ __forceinline__ V sinh(V a) { return chain(a, fm<T>::sinh(a.re), fm<T>::cosh(a.re)); }
  static __device__ __forceinline__ V cosh(V a) { return chain(a, fm<T>::cosh(a.re), fm<T>::sinh(a.re)); }
  static __device__ __forceinline__ V tanh(V a) { T cc = fm<T>::cosh(a.re); return chain(a, fm<T>::tanh(a.re), T(1) / (cc * cc)); }
  static __device__ __forceinline__ V asinh(V a) { return chain(a, fm<T>::asinh(a.re), asinh_deriv<S>(a.re)); }
  static __device__ __forceinline__ V acosh(V a) { return chain(a, fm<T>::acosh(a.re), acosh_deriv<S>(a.re)); }
  static __device__ __forceinline__ V atanh(V a) { return chain(a, fm<T>::atanh(a.re), atanh_deriv<S>(a.re)); }
  static __device__ __forceinline__ V abs(V a) { return chain(a, fm<T>::fabs(a.re), abs_deriv<S>(a.re)); }
  static __device__ __forceinline__ V signum(V a) { return c0(signum_s(a.re)); }
  static __device__ __forceinline__ V floor(V a) { return c0(fm<T>::floor(a.re)); }
  static __device__ __forceinline__ V ceil(V a) { return c0(fm<T>::ceil(a.re)); }
  static __device__ __forceinline__ V round(V a) { return c0(fm<T>::round(a.re)); }
  static __device__ __forceinline__ V trunc(V a) { return c0(fm<T>::trunc(a.re)); }
  static __device__ __forceinline__ V fract(V a) { return {fract_s(a.re), a.eps}; }
  static __device__ __forceinline__ bool all_zero(V a) { return a.re == T(0) && a.eps == T(0); }
  static __device__ __forceinline__ V nan() { return c0(fm<T>::nan()); }
  static __device__ V powf(V self, V n) {
    int32_t ni;
    if (n.eps == T(0) && as_i32(n.re, &ni)) return powi(self, ni);
    if (n.re == T(0)) {
      T dy = (self.re > T(0)) ? fm<T>::log(self.re) : T(0);
      return {T(1), dy * n.eps};
    }
    T val = fm<T>::pow(self.re, n.re);
    T dx;
    if (self.eps == T(0)) dx = T(0);
    else if (self.re == T(0) || val == T(0) || !isfinite_(self.re) || !isfinite_(val))
      dx = n.re * fm<T>::pow(self.re, n.re - T(1)) * self.eps;
    else
      dx = n.re * val / self.re * self.eps;
    T dy;
    if (n.eps == T(0) || val == T(0) || self.re <= T(0)) dy = T(0);
    else dy = val * fm<T>::log(self.re) * n.eps;
    return {val, dx + dy};
  }
  static __device__ V atan2(V self, V other) {
    T da, db;
    atan2_partials<S>(self.re, other.re, da, db);
    return {fm<T>::atan2(self.re, other.re), da * self.eps + db * other.eps};
  }
  static __device__ V hypot(V self, V other) {
    T h = fm<T>::hypot(self.re, other.re);
    if (h == T(0)) return c0(h);
    T da, db;
    hypot_partials<S>(self.re, other.re, h, da, db);
    return {h, da * self.eps + db * other.eps};
  }
};
template <class T> struct KindOf<Dual<T>> { using K = DK<T>; };

// ───────────────────────────── Taylor kind (src/taylor_ops.rs) ──────────────
namespace jt {
template <class T, int K> __device__ __forceinline__ void mul(const T* a, const T* b, T* c) {
#pragma unroll
  for (int k = 0; k < K; ++k) {
    T sum = T(0);
#pragma unroll
    for (int j = 0; j <= k; ++j) sum = sum + a[j] * b[k - j];
    c[k] = sum;
  }
}
template <class T, int K> __device__ __forceinline__ void div(const T* a, const T* b, T* c) {
  c[0] = a[0] / b[0];
  T inv_b0 = T(1) / b[0];
#pragma unroll
  for (int k = 1; k < K; ++k) {
    T sum = a[k];
#pragma unroll
    for (int j = 1; j <= k; ++j) sum = sum - b[j] * c[k - j];
    c[k] = sum * inv_b0;
  }
}
template <class T, int K> __device__ __forceinline__ void recip(const T* a, T* c) {
  T inv_a0 = T(1) / a[0];
  c[0] = inv_a0;
#pragma unroll
  for (int k = 1; k < K; ++k) {
    T sum = T(0);
#pragma unroll
    for (int j = 1; j <= k; ++j) sum = sum + a[j] * c[k - j];
    c[k] = -sum * inv_a0;
  }
}
template <class T, int K> __device__ __forceinline__ void expv(const T* a, T* c) {
  c[0] = fm<T>::exp(a[0]);
#pragma unroll
  for (int k = 1; k < K; ++k) {
    T sum = T(0);
#pragma unroll
    for (int j = 1; j <= k; ++j) sum = sum + T(j) * a[j] * c[k - j];
    c[k] = sum / T(k);
  }
}
template <class T, int K> __device__ __forceinline__ void nan_jet(T* c) {
#pragma unroll
  for (int k = 0; k < K; ++k) c[k] = fm<T>::nan();
}
template <class T, int K> __device__ __forceinline__ void vertical(T* c) {
  c[0] = T(0);
#pragma unroll
  for (int k = 1; k < K; ++k) c[k] = fm<T>::inf();
}
template <class T, int K> __device__ __forceinline__ void ln(const T* a, T* c) {
  if (a[0] < T(0)) { nan_jet<T, K>(c); return; }
  T inv_a0 = T(1) / a[0];
  c[0] = fm<T>::log(a[0]);
#pragma unroll
  for (int k = 1; k < K; ++k) {
    T sum = T(0);
#pragma unroll
    for (int j = 1; j < k; ++j) sum = sum + T(j) * c[j] * a[k - j];
    c[k] = (a[k] - sum / T(k)) * inv_a0;
  }
}
template <class T, int K> __device__ __forceinline__ void sqrt(const T* a, T* c) {
  if (a[0] == T(0)) { vertical<T, K>(c); return; }
  if (a[0] < T(0)) { nan_jet<T, K>(c); return; }
  c[0] = fm<T>::sqrt(a[0]);
  T two_c0 = T(2) * c[0];
#pragma unroll
  for (int k = 1; k < K; ++k) {
    T sum = T(0);
#pragma unroll
    for (int j = 1; j < k; ++j) sum = sum + c[j] * c[k - j];
    c[k] = (a[k] - sum) / two_c0;
  }
}
template <class T, int K> __device__ __forceinline__ void sin_cos(const T* a, T* s, T* co) {
  s[0] = fm<T>::sin(a[0]);
  co[0] = fm<T>::cos(a[0]);
#pragma unroll
  for (int k = 1; k < K; ++k) {
    T inv_k = T(1) / T(k);
    T ss = T(0), sc = T(0);
#pragma unroll
    for (int j = 1; j <= k; ++j) {
      T jf = T(j);
      ss = ss + jf * a[j] * co[k - j];
      sc = sc + jf * a[j] * s[k - j];
    }
    s[k] = ss * inv_k;
    co[k] = -sc * inv_k;
  }
}
template <class T, int K> __device__ __forceinline__ void sinh_cosh(const T* a, T* sh, T* ch) {
  sh[0] = fm<T>::sinh(a[0]);
  ch[0] = fm<T>::cosh(a[0]);
#pragma unroll
  for (int k = 1; k < K; ++k) {
    T inv_k = T(1) / T(k);
    T ss = T(0), sc = T(0);
#pragma unroll
    for (int j = 1; j <= k; ++j) {
      T jf = T(j);
      ss = ss + jf * a[j] * ch[k - j];
      sc = sc + jf * a[j] * sh[k - j];
    }
    sh[k] = ss * inv_k;
    ch[k] = sc * inv_k;
  }
}
template <class T, int K> __device__ __forceinline__ void integrate(const T* a, const T* g, T* c) {
#pragma unroll
  for (int k = 1; k < K; ++k) {
    T sum = T(0);
#pragma unroll
    for (int j = 1; j <= k; ++j) sum = sum + T(j) * a[j] * g[k - j];
    c[k] = sum / T(k);
  }
}
template <class T, int K> __device__ void atan(const T* a, T* c) {
  T s1[K], s2[K];
  mul<T, K>(a, a, s1);
#pragma unroll
  for (int k = 0; k < K; ++k) s2[k] = s1[k];
  s2[0] = T(1) + s1[0];
  c[0] = fm<T>::atan(a[0]);
  recip<T, K>(s2, s1);
  integrate<T, K>(a, s1, c);
}
template <class T, int K> __device__ void asin(const T* a, T* c) {
  T s1[K], s2[K];
  c[0] = fm<T>::asin(a[0]);
  mul<T, K>(a, a, s1);
  s2[0] = (T(1) - a[0]) * (T(1) + a[0]);
#pragma unroll
  for (int k = 1; k < K; ++k) s2[k] = -s1[k];
  sqrt<T, K>(s2, s1);
  recip<T, K>(s1, s2);
  integrate<T, K>(a, s2, c);
}
template <class T, int K> __device__ void acos(const T* a, T* c) {
  asin<T, K>(a, c);
  c[0] = fm<T>::acos(a[0]);
#pragma unroll
  for (int k = 1; k < K; ++k) c[k] = -c[k];
}
template <class T, int K> __device__ __forceinline__ void tan(const T* a, T* c) {
  T sc[K];
  c[0] = fm<T>::tan(a[0]);
  sc[0] = T(1) + c[0] * c[0];
#pragma unroll
  for (int k = 1; k < K; ++k) {
    T sum = T(0);
#pragma unroll
    for (int j = 1; j <= k; ++j) sum = sum + T(j) * a[j] * sc[k - j];
    c[k] = sum / T(k);
    T s_k = T(0);
#pragma unroll
    for (int j = 0; j <= k; ++j) s_k = s_k + c[j] * c[k - j];
    sc[k] = s_k;
  }
}
template <class T, int K> __device__ __forceinline__ void tanh(const T* a, T* c) {
  T sc[K];
  c[0] = fm<T>::tanh(a[0]);
  sc[0] = T(1) - c[0] * c[0];
#pragma unroll
  for (int k = 1; k < K; ++k) {
    T sum = T(0);
#pragma unroll
    for (int j = 1; j <= k; ++j) sum = sum + T(j) * a[j] * sc[k - j];
    c[k] = sum / T(k);
    T s_k = T(0);
#pragma unroll
    for (int j = 0; j <= k; ++j) s_k = s_k + c[j] * c[k - j];
    sc[k] = -s_k;
  }
}
template <class T, int K> __device__ void asinh(const T* a, T* c) {
  T s1[K], s2[K];
  c[0] = fm<T>::asinh(a[0]);
  mul<T, K>(a, a, s1);
#pragma unroll
  for (int k = 0; k < K; ++k) s2[k] = s1[k];
  s2[0] = T(1) + s1[0];
  sqrt<T, K>(s2, s1);
  recip<T, K>(s1, s2);
  integrate<T, K>(a, s2, c);
}
template <class T, int K> __device__ void acosh(const T* a, T* c) {
  if (a[0] < T(1)) { nan_jet<T, K>(c); return; }
  T s1[K], s2[K];
  c[0] = fm<T>::acosh(a[0]);
  mul<T, K>(a, a, s1);
#pragma unroll
  for (int k = 0; k < K; ++k) s2[k] = s1[k];
  s2[0] = (a[0] - T(1)) * (a[0] + T(1));
  sqrt<T, K>(s2, s1);
  recip<T, K>(s1, s2);
  integrate<T, K>(a, s2, c);
}
template <class T, int K> __device__ void atanh(const T* a, T* c) {
  if (a[0] < -T(1) || a[0] > T(1)) { nan_jet<T, K>(c); return; }
  T s1[K], s2[K];
  c[0] = fm<T>::atanh(a[0]);
  mul<T, K>(a, a, s1);
  s2[0] = (T(1) - a[0]) * (T(1) + a[0]);
#pragma unroll
  for (int k = 1; k < K; ++k) s2[k] = -s1[k];
  recip<T, K>(s2, s1);
  integrate<T, K>(a, s1, c);
}
template <class T, int K> __device__ void powi_squaring(const T* a, int32_t n, T* c) {
  T s1[K], s2[K];
  uint32_t power = n < 0 ? (uint32_t)(-(int64_t)n) : (uint32_t)n;
  c[0] = T(1);
#pragma unroll
  for (int k = 1; k < K; ++k) c[k] = T(0);
#pragma unroll
  for (int k = 0; k < K; ++k) s1[k] = a[k];
  while (power > 0) {
    if (power & 1u) {
      mul<T, K>(c, s1, s2);
#pragma unroll
      for (int k = 0; k < K; ++k) c[k] = s2[k];
    }
    power >>= 1;
    if (power > 0) {
      mul<T, K>(s1, s1, s2);
#pragma unroll
      for (int k = 0; k < K; ++k) s1[k] = s2[k];
    }
  }
  if (n < 0) {
#pragma unroll
    for (int k = 0; k < K; ++k) s1[k] = c[k];
    recip<T, K>(s1, c);
  }
}
template <class T, int K> __device__ void powi(const T* a, int32_t n, T* c) {
  if (n == 0) {
    c[0] = T(1);
#pragma unroll
    for (int k = 1; k < K; ++k) c[k] = T(0);
    return;
  }
  if (n == 1) {
#pragma unroll
    for (int k = 0; k < K; ++k) c[k] = a[k];
    return;
  }
  if (n == -1) { recip<T, K>(a, c); return; }
  uint32_t absn = n < 0 ? (uint32_t)(-(int64_t)n) : (uint32_t)n;
  if (a[0] <= T(0) || absn <= 8u) {
    powi_squaring<T, K>(a, n, c);
  } else {
    T s1[K], s2[K];
    ln<T, K>(a, s1);
#pragma unroll
    for (int k = 0; k < K; ++k) s2[k] = T(n) * s1[k];
    expv<T, K>(s2, c);
    c[0] = powi_s(a[0], n);
  }
}
template <class T, int K> __device__ void powf(const T* a, const T* b, T* c) {
  bool hi_zero = true;
#pragma unroll
  for (int k = 1; k < K; ++k) hi_zero = hi_zero && (b[k] == T(0));
  int32_t ni;
  if (hi_zero && as_i32(b[0], &ni)) { powi<T, K>(a, ni, c); return; }
  if (a[0] == T(0)) {
    T b0 = b[0];
    int32_t bi;
    if (as_i32(b0, &bi)) { nan_jet<T, K>(c); return; }
    c[0] = fm<T>::pow(a[0], b0);
#pragma unroll
    for (int k = 1; k < K; ++k) c[k] = (T(k) < b0) ? T(0) : fm<T>::inf();
    return;
  }
  T s1[K], s2[K];
  ln<T, K>(a, s1);
  mul<T, K>(b, s1, s2);
  expv<T, K>(s2, c);
  if (a[0] < T(0)) c[0] = fm<T>::nan();
  else c[0] = fm<T>::pow(a[0], b[0]);
}
template <class T, int K> __device__ void cbrt(const T* a, T* c) {
  if (a[0] == T(0)) { vertical<T, K>(c); return; }
  T third = T(1) / T(3);
  T s1[K], s2[K], na[K];
  const bool neg = a[0] < T(0);
#pragma unroll
  for (int i = 0; i < K; ++i) na[i] = neg ? -a[i] : a[i];
  ln<T, K>(na, s1);
#pragma unroll
  for (int k = 0; k < K; ++k) s2[k] = third * s1[k];
  expv<T, K>(s2, c);
  c[0] = fm<T>::cbrt(a[0]);
  if (neg) {
#pragma unroll
    for (int i = 1; i < K; ++i) c[i] = -c[i];
  }
}
template <class T, int K> __device__ void hypot(const T* a, const T* b, T* c) {
  int m = 0;
  if (fm<T>::fmax(fm<T>::fabs(a[0]), fm<T>::fabs(b[0])) == T(0)) {
    if (isnan_(a[0]) || isnan_(b[0])) { nan_jet<T, K>(c); return; }
    int found = -1;
#pragma unroll
    for (int k = K - 1; k >= 1; --k)
      if (a[k] != T(0) || b[k] != T(0)) found = k;
    if (found < 0) {
#pragma unroll
      for (int k = 0; k < K; ++k) c[k] = T(0);
      return;
    }
    m = found;
    T am = a[0], bm = b[0];
#pragma unroll
    for (int k = 1; k < K; ++k) if (k == m) { am = a[k]; bm = b[k]; }
    if (isnan_(am) || isnan_(bm)) {
#pragma unroll
      for (int k = 0; k < K; ++k) c[k] = (k < m) ? T(0) : (k == m ? fm<T>::hypot(am, bm) : fm<T>::nan());
      return;
    }
  }
  T s1[K], s2[K], sh[K], tt[K];
  T am = a[0], bm = b[0];
#pragma unroll
  for (int k = 1; k < K; ++k) if (k == m) { am = a[k]; bm = b[k]; }
  T scl = fm<T>::fmax(fm<T>::fabs(am), fm<T>::fabs(bm));
  T inv_scale = T(1) / scl;
#pragma unroll
  for (int k = 0; k < K; ++k) {
    T av = T(0), bv = T(0);
#pragma unroll
    for (int q = 0; q < K; ++q) if (q == k + m) { av = a[q]; bv = b[q]; }
    s1[k] = (k + m < K) ? av * inv_scale : T(0);
    s2[k] = (k + m < K) ? bv * inv_scale : T(0);
  }
  mul<T, K>(s1, s1, tt);
  mul<T, K>(s2, s2, s1);
#pragma unroll
  for (int k = 0; k < K; ++k) tt[k] = tt[k] + s1[k];
  sqrt<T, K>(tt, s1);
#pragma unroll
  for (int k = 0; k < K; ++k) sh[k] = s1[k] * scl;
  sh[0] = fm<T>::hypot(am, bm);
#pragma unroll
  for (int k = 0; k < K; ++k) {
    T v = T(0);
#pragma unroll
    for (int q = 0; q < K; ++q) if (q + m == k) v = sh[q];
    c[k] = (k < m) ? T(0) : v;
  }
}
template <class T, int K> __device__ void atan2(const T* a, const T* b, T* c) {
  T s1[K];
  if (b[0] != T(0)) {
    div<T, K>(a, b, s1);
    atan<T, K>(s1, c);
    c[0] = fm<T>::atan2(a[0], b[0]);
  } else if (a[0] != T(0)) {
    div<T, K>(b, a, s1);
    atan<T, K>(s1, c);
#pragma unroll
    for (int k = 0; k < K; ++k) c[k] = -c[k];
    c[0] = fm<T>::atan2(a[0], b[0]);
  } else {
    c[0] = T(0);
#pragma unroll
    for (int k = 1; k < K; ++k) c[k] = T(0);
  }
}
}  // namespace jt

template <class T, int K> struct JK {
  using V = Jet<T, K>;
  static __device__ __forceinline__ V c(double v) { return VT<V>::cst(v); }
  static __device__ __forceinline__ V c0(T v) {
    V r;
    r.c[0] = v;
#pragma unroll
    for (int k = 1; k < K; ++k) r.c[k] = T(0);
    return r;
  }
  static __device__ __forceinline__ V add(const V& a, const V& b) { V r; for (int k = 0; k < K; ++k) r.c[k] = a.c[k] + b.c[k]; return r; }
  static __device__ __forceinline__ V sub(const V& a, const V& b) { V r; for (int k = 0; k < K; ++k) r.c[k] = a.c[k] - b.c[k]; return r; }
  static __device__ __forceinline__ V mul(const V& a, const V& b) { V r; jt::mul<T, K>(a.c, b.c, r.c); return r; }
  static __device__ __forceinline__ V div(const V& a, const V& b) { V r; jt::div<T, K>(a.c, b.c, r.c); return r; }
  static __device__ __forceinline__ V neg(const V& a) { V r; for (int k = 0; k < K; ++k) r.c[k] = -a.c[k]; return r; }
  static __device__ __forceinline__ V rem(const V& a, const V& b) {
    V r;
    if (b.c[0] == T(0)) { jt::nan_jet<T, K>(r.c); return r; }
    T q = fm<T>::trunc(a.c[0] / b.c[0]);
    r.c[0] = fm<T>::fmod(a.c[0], b.c[0]);
#pragma unroll
    for (int k = 1; k < K; ++k) r.c[k] = a.c[k] - b.c[k] * q;
    return r;
  }
  static __device__ V powf(const V& a, const V& b) { V r; jt::powf<T, K>(a.c, b.c, r.c); return r; }
  static __device__ V atan2(const V& a, const V& b) { V r; jt::atan2<T, K>(a.c, b.c, r.c); return r; }
  static __device__ V hypot(const V& a, const V& b) { V r; jt::hypot<T, K>(a.c, b.c, r.c); return r; }
  static __device__ __forceinline__ V recip(const V& a) { V r; jt::recip<T, K>(a.c, r.c); return r; }
  static __device__ __forceinline__ V sqrt(const V& a) { V r; jt::sqrt<T, K>(a.c, r.c); return r; }
  static __device__ V cbrt(const V& a) { V r; jt::cbrt<T, K>(a.c, r.c); return r; }
  static __device__ V powi(const V& a, int32_t n) { V r; jt::powi<T, K>(a.c, n, r.c); return r; }
  static __device__ __forceinline__ V exp(const V& a) { V r; jt::expv<T, K>(a.c, r.c); return r; }
  static __device__ V exp2(const V& a) {
    V s, r;
    T ln2 = fm<T>::log(T(2));
    for (int k = 0; k < K; ++k) s.c[k] = ln2 * a.c[k];
    jt::expv<T, K>(s.c, r.c);
    r.c[0] = fm<T>::exp2(a.c[0]);
    return r;
  }
  static __device__ __forceinline__ V exp_m1(const V& a) { V r; jt::expv<T, K>(a.c, r.c); r.c[0] = fm<T>::expm1(a.c[0]); return r; }
  static __device__ __forceinline__ V ln(const V& a) { V r; jt::ln<T, K>(a.c, r.c); return r; }
  static __device__ V log2(const V& a) {
    V r;
    jt::ln<T, K>(a.c, r.c);
    T inv = T(1) / fm<T>::log(T(2));
    r.c[0] = fm<T>::log2(a.c[0]);
    for (int k = 1; k < K; ++k) r.c[k] = r.c[k] * inv;
    return r;
  }
  static __device__ V log10(const V& a) {
    V r;
    jt::ln<T, K>(a.c, r.c);
    T inv = T(1) / fm<T>::log(T(10));
    r.c[0] = fm<T>::log10(a.c[0]);
    for (int k = 1; k < K; ++k) r.c[k] = r.c[k] * inv;
    return r;
  }
  static __device__ V ln_1p(const V& a) {
    V s, r;
    for (int k = 1; k < K; ++k) s.c[k] = a.c[k];
    s.c[0] = T(1) + a.c[0];
    jt::ln<T, K>(s.c, r.c);
    r.c[0] = fm<T>::log1p(a.c[0]);
    return r;
  }
  static __device__ __forceinline__ V sin(const V& a) { V s, co; jt::sin_cos<T, K>(a.c, s.c, co.c); return s; }
  static __device__ __forceinline__ V cos(const V& a) { V s, co; jt::sin_cos<T, K>(a.c, s.c, co.c); return co; }
  static __device__ __forceinline__ V tan(const V& a) { V r; jt::tan<T, K>(a.c, r.c); return r; }
  static __device__ V asin(const V& a) { V r; jt::asin<T, K>(a.c, r.c); return r; }
  static __device__ V acos(const V& a) { V r; jt::acos<T, K>(a.c, r.c); return r; }
  static __device__ V atan(const V& a) { V r; jt::atan<T, K>(a.c, r.c); return r; }
  static __device__ __forceinline__ V sinh(const V& a) { V s, co; jt::sinh_cosh<T, K>(a.c, s.c, co.c); return s; }
  static __device__ __forceinline__ V cosh(const V& a) { V s, co; jt::sinh_cosh<T, K>(a.c, s.c, co.c); return co; }
  static __device__ __forceinline__ V tanh(const V& a) { V r; jt::tanh<T, K>(a.c, r.c); return r; }
  static __device__ V asinh(const V& a) { V r; jt::asinh<T, K>(a.c, r.c); return r; }
  static __device__ V acosh(const V& a) { V r; jt::acosh<T, K>(a.c, r.c); return r; }
  static __device__ V atanh(const V& a) { V r; jt::atanh<T, K>(a.c, r.c); return r; }
  static __device__ V abs(const V& a) {
    // Taylor::abs: sign of the first non-zero coefficient (src/taylor.rs:278-294).
    T sign;
    if (a.c[0] != T(0)) sign = signum_s(a.c[0]);
    else {
      sign = T(1);
#pragma unroll
      for (int k = K - 1; k >= 1; --k) if (a.c[k] != T(0)) sign = signum_s(a.c[k]);
    }
    V r;
    for (int k = 0; k < K; ++k) r.c[k] = a.c[k] * sign;
    return r;
  }
  static __device__ __forceinline__ V signum(const V& a) { return c0(signum_s(a.c[0])); }
  static __device__ __forceinline__ V floor(const V& a) { return c0(fm<T>::floor(a.c[0])); }
  static __device__ __forceinline__ V ceil(const V& a) { return c0(fm<T>::ceil(a.c[0])); }
  static __device__ __forceinline__ V round(const V& a) { return c0(fm<T>::round(a.c[0])); }
  static __device__ __forceinline__ V trunc(const V& a) { return c0(fm<T>::trunc(a.c[0])); }
  static __device__ __forceinline__ V fract(const V& a) { V r = a; r.c[0] = fract_s(a.c[0]); return r; }
  static __device__ __forceinline__ bool all_zero(const V& a) {
    bool z = true;
    for (int k = 0; k < K; ++k) z = z && (a.c[k] == T(0));
    return z;
  }
  static __device__ __forceinline__ V nan() { return c0(fm<T>::nan()); }
};
template <class T, int N> struct KindOf<Jet<T, N>> { using K = JK<T, N>; };

// ───────────────────────────── opcode dispatch ──────────────────────────────
// Forward evaluation of one opcode (src/opcode.rs:228-318).  `Powi` takes its
// exponent from the instruction.
template <class V> __device__ __forceinline__ V eval_forward(uint32_t op, const V& a, const V& b, int32_t aux) {
  using Kd = typename KindOf<V>::K;
  switch (op) {
    case OP_ADD: return Kd::add(a, b);
    case OP_SUB: return Kd::sub(a, b);
    case OP_MUL: return Kd::mul(a, b);
    case OP_DIV: return Kd::div(a, b);
    case OP_REM: return Kd::rem(a, b);
    case OP_POWF: return Kd::powf(a, b);
    case OP_ATAN2: return Kd::atan2(a, b);
    case OP_HYPOT: return Kd::hypot(a, b);
    case OP_MAX: return (VT<V>::prim(a) >= VT<V>::prim(b) || isnan_(VT<V>::prim(b))) ? a : b;
    case OP_MIN: return (VT<V>::prim(a) <= VT<V>::prim(b) || isnan_(VT<V>::prim(b))) ? a : b;
    case OP_NEG: return Kd::neg(a);
    case OP_RECIP: return Kd::recip(a);
    case OP_SQRT: return Kd::sqrt(a);
    case OP_CBRT: return Kd::cbrt(a);
    case OP_POWI: return Kd::powi(a, aux);
    case OP_EXP: return Kd::exp(a);
    case OP_EXP2: return Kd::exp2(a);
    case OP_EXPM1: return Kd::exp_m1(a);
    case OP_LN: return Kd::ln(a);
    case OP_LOG2: return Kd::log2(a);
    case OP_LOG10: return Kd::log10(a);
    case OP_LN1P: return Kd::ln_1p(a);
    case OP_SIN: return Kd::sin(a);
    case OP_COS: return Kd::cos(a);
    case OP_TAN: return Kd::tan(a);
    case OP_ASIN: return Kd::asin(a);
    case OP_ACOS: return Kd::acos(a);
    case OP_ATAN: return Kd::atan(a);
    case OP_SINH: return Kd::sinh(a);
    case OP_COSH: return Kd::cosh(a);
    case OP_TANH: return Kd::tanh(a);
    case OP_ASINH: return Kd::asinh(a);
    case OP_ACOSH: return Kd::acosh(a);
    case OP_ATANH: return Kd::atanh(a);
    case OP_ABS: return Kd::abs(a);
    case OP_SIGNUM: return Kd::signum(a);
    case OP_FLOOR: return Kd::floor(a);
    case OP_CEIL: return Kd::ceil(a);
    case OP_ROUND: return Kd::round(a);
    case OP_TRUNC: return Kd::trunc(a);
    case OP_FRACT: return Kd::fract(a);
    default: return Kd::nan();
  }
}

// Reverse partials (src/opcode.rs:331-483, powi via src/opcode.rs:503-513).
template <class V> __device__ __forceinline__ void reverse_partials(uint32_t op, const V& a, const V& b, const V& r,
                                                                    int32_t aux, V& da, V& db) {
  using Kd = typename KindOf<V>::K;
  using P = VT<V>;
  const V zero = Kd::c(0), one = Kd::c(1);
  db = zero;
  switch (op) {
    case OP_ADD: da = one; db = one; return;
    case OP_SUB: da = one; db = Kd::neg(one); return;
    case OP_MUL: da = b; db = a; return;
    case OP_DIV: { V inv = Kd::div(one, b); da = inv; db = Kd::mul(Kd::neg(r), inv); return; }
    case OP_REM: da = one; db = Kd::neg(Kd::trunc(Kd::div(a, b))); return;
    case OP_POWF: {
      if (P::prim(b) == 0) {
        da = zero;
        db = (P::prim(a) > 0) ? Kd::ln(a) : zero;
        return;
      }
      if (P::prim(a) == 0 || P::prim(r) == 0 || !isfinite_(P::prim(a)) || !isfinite_(P::prim(r)))
        da = Kd::mul(b, Kd::powf(a, Kd::sub(b, one)));
      else
        da = Kd::div(Kd::mul(b, r), a);
      db = (P::prim(r) == 0 || P::prim(a) <= 0) ? zero : Kd::mul(r, Kd::ln(a));
      return;
    }
    case OP_ATAN2: atan2_partials<Kd>(a, b, da, db); return;
    case OP_HYPOT: hypot_partials<Kd>(a, b, r, da, db); return;
    case OP_MAX:
      if (P::prim(a) >= P::prim(b) || isnan_(P::prim(b))) { da = one; db = zero; } else { da = zero; db = one; }
      return;
    case OP_MIN:
      if (P::prim(a) <= P::prim(b) || isnan_(P::prim(b))) { da = one; db = zero; } else { da = zero; db = one; }
      return;
    case OP_NEG: da = Kd::neg(one); return;
    case OP_RECIP: { V inv = Kd::div(one, a); da = Kd::mul(Kd::neg(inv), inv); return; }
    case OP_SQRT: { V two = Kd::add(one, one); da = Kd::div(one, Kd::mul(two, r)); return; }
    case OP_CBRT: { V three = Kd::c(3.0); da = Kd::div(one, Kd::mul(Kd::mul(three, r), r)); return; }
    case OP_POWI: {
      if (aux == 0) da = zero;
      else if (aux == (int32_t)0x80000000) da = Kd::div(Kd::mul(Kd::c((double)aux), r), a);
      else da = Kd::mul(Kd::c((double)aux), Kd::powi(a, aux - 1));
      return;
    }
    case OP_EXP: da = r; return;
    case OP_EXP2: da = Kd::mul(r, Kd::c(fm<typename P::S>::LN2)); return;
    case OP_EXPM1: da = Kd::add(r, one); return;
    case OP_LN: da = ln_deriv<Kd>(a); return;
    case OP_LOG2: da = log2_deriv<Kd>(a); return;
    case OP_LOG10: da = log10_deriv<Kd>(a); return;
    case OP_LN1P: da = ln_1p_deriv<Kd>(a); return;
    case OP_SIN: da = Kd::cos(a); return;
    case OP_COS: da = Kd::neg(Kd::sin(a)); return;
    case OP_TAN: { V cc = Kd::cos(a); da = Kd::div(one, Kd::mul(cc, cc)); return; }
    case OP_ASIN: da = Kd::div(one, Kd::sqrt(Kd::mul(Kd::sub(one, a), Kd::add(one, a)))); return;
    case OP_ACOS: da = Kd::div(Kd::neg(one), Kd::sqrt(Kd::mul(Kd::sub(one, a), Kd::add(one, a)))); return;
    case OP_ATAN: da = atan_deriv<Kd>(a); return;
    case OP_SINH: da = Kd::cosh(a); return;
    case OP_COSH: da = Kd::sinh(a); return;
    case OP_TANH: { V cc = Kd::cosh(a); da = Kd::div(one, Kd::mul(cc, cc)); return; }
    case OP_ASINH: da = asinh_deriv<Kd>(a); return;
    case OP_ACOSH: da = acosh_deriv<Kd>(a); return;
    case OP_ATANH: da = atanh_deriv<Kd>(a); return;
    case OP_ABS: da = abs_deriv<Kd>(a); return;
    case OP_SIGNUM: case OP_FLOOR: case OP_CEIL: case OP_ROUND: case OP_TRUNC: da = zero; return;
    case OP_FRACT: da = one; return;
    default: da = zero; return;
  }
}

}  // namespace dm
}  // namespace ech
