// Oracle — TEST INFRASTRUCTURE ONLY.
//
// A CPU restatement of echidna's BytecodeTape sweeps, used by the tests, by
// __graft_entry__.smoke() and by bench.py's CPU-baseline leg as the checker.
// Nothing in the product (echidna_b200/) links or calls this file.
//
// It follows the reference's CPU f64/f32 path operation by operation, with the
// same evaluation order (compile with -ffp-contract=off, no fast-math):
//   * scalar forward / partials:  src/opcode.rs:228-535, src/kernels/mod.rs:85-285
//   * forward sweep:              src/bytecode_tape/forward.rs:11-43, 194-229
//   * reverse sweep:              src/bytecode_tape/reverse.rs:32-105
//   * tangent sweeps / HVP:       src/bytecode_tape/tangent.rs:97-310
//   * Dual arithmetic:            src/dual.rs:40-464, src/traits/std_ops.rs:14-82,
//                                 src/traits/num_traits_impls.rs:17-380
//   * Taylor jets:                src/taylor_ops.rs:18-916, src/taylor.rs:180-370,
//                                 src/traits/taylor_std_ops.rs:74-101
//   * STDE estimators:            src/stde/{types,jet,laplacian,pipeline,higher_order}.rs
//
// Third-party arithmetic: Rust std forwards most transcendentals to the platform
// libm; this oracle calls glibc libm for them, so agreement with a Rust build is
// pinned only to the tolerances the reference's own tests use.  powi is the
// square-and-multiply loop that Rust's powi lowers to (binary exponentiation,
// Knuth TAOCP 4.6.3).
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <thread>
#include <utility>
#include <vector>
#include <algorithm>

namespace orc {

constexpr uint32_t UNUSED = 0xFFFFFFFFu;
// std::f64::consts::LN_2 / LN_10 at full precision.
constexpr double kLN2 = 0.693147180559945309417232121458176568;
constexpr double kLN10 = 2.302585092994045684017991454684364208;

enum Op : uint32_t {
  INPUT = 0, CONST, ADD, SUB, MUL, DIV, REM, POWF, ATAN2, HYPOT, MAX, MIN,
  NEG, RECIP, SQRT, CBRT, POWI, EXP, EXP2, EXPM1, LN, LOG2, LOG10, LN1P,
  SIN, COS, TAN, ASIN, ACOS, ATAN, SINH, COSH, TANH, ASINH, ACOSH, ATANH,
  ABS, SIGNUM, FLOOR, CEIL, ROUND, TRUNC, FRACT, CUSTOM
};

// ───────────────────────── scalar helpers (F = double | float) ─────────────
template <class F> F s_powi(F a, int32_t n) {
  // src/opcode.rs:233-251 via Rust powi -> binary exponentiation.
  bool recip = n < 0;
  uint32_t m = n < 0 ? (uint32_t)(-(int64_t)n) : (uint32_t)n;
  F r = F(1);
  for (;;) {
    if (m & 1u) r = r * a;
    m >>= 1;
    if (m == 0) break;
    a = a * a;
  }
  return recip ? F(1) / r : r;
}
template <class F> F s_signum(F x) { return std::isnan(x) ? x : std::copysign(F(1), x); }
template <class F> F s_fract(F x) { return x - std::trunc(x); }
template <class F> F s_nan() { return std::numeric_limits<F>::quiet_NaN(); }
template <class F> F s_inf() { return std::numeric_limits<F>::infinity(); }

// num_traits Float::to_i32 followed by the integrality check used by
// Dual::powf and taylor_powf (src/dual.rs:364-369, src/taylor_ops.rs:471-476).
template <class F> bool s_as_i32(F x, int32_t* out) {
  if (!(x > F(-2147483649.0) && x < F(2147483648.0))) return false;
  int32_t ni = (int32_t)x;  // truncation
  if ((F)ni != x) return false;
  *out = ni;
  return true;
}

// ───────────────────────── Dual<F> (src/dual.rs) ───────────────────────────
template <class F> struct Dual {
  F re, eps;
};
template <class F> inline Dual<F> dconst(F v) { return {v, F(0)}; }
template <class F> inline Dual<F> operator+(Dual<F> a, Dual<F> b) { return {a.re + b.re, a.eps + b.eps}; }
template <class F> inline Dual<F> operator-(Dual<F> a, Dual<F> b) { return {a.re - b.re, a.eps - b.eps}; }
template <class F> inline Dual<F> operator*(Dual<F> a, Dual<F> b) {
  return {a.re * b.re, a.re * b.eps + a.eps * b.re};
}
template <class F> inline Dual<F> operator/(Dual<F> a, Dual<F> b) {
  F inv = F(1) / b.re;
  F re = a.re / b.re;
  return {re, (a.eps - re * b.eps) * inv};
}
template <class F> inline Dual<F> operator-(Dual<F> a) { return {-a.re, -a.eps}; }

// ───────────────────────── Taylor<F,K> (src/taylor_ops.rs) ─────────────────
template <class F, int K> struct Tay {
  F c[K];
};

namespace tops {
template <class F> void mul(const F* a, const F* b, F* c, int n) {
  for (int k = 0; k < n; ++k) {
    F sum = F(0);
    for (int j = 0; j <= k; ++j) sum = sum + a[j] * b[k - j];
    c[k] = sum;
  }
}
template <class F> void div(const F* a, const F* b, F* c, int n) {
  c[0] = a[0] / b[0];
  F inv_b0 = F(1) / b[0];
  for (int k = 1; k < n; ++k) {
    F sum = a[k];
    for (int j = 1; j <= k; ++j) sum = sum - b[j] * c[k - j];
    c[k] = sum * inv_b0;
  }
}
template <class F> void recip(const F* a, F* c, int n) {
  F inv_a0 = F(1) / a[0];
  c[0] = inv_a0;
  for (int k = 1; k < n; ++k) {
    F sum = F(0);
    for (int j = 1; j <= k; ++j) sum = sum + a[j] * c[k - j];
    c[k] = -sum * inv_a0;
  }
}
template <class F> void exp(const F* a, F* c, int n) {
  c[0] = std::exp(a[0]);
  for (int k = 1; k < n; ++k) {
    F sum = F(0);
    for (int j = 1; j <= k; ++j) sum = sum + F(j) * a[j] * c[k - j];
    c[k] = sum / F(k);
  }
}
template <class F> void nan_jet(F* c, int n) {
  for (int k = 0; k < n; ++k) c[k] = s_nan<F>();
}
template <class F> void vertical_tangent_jet(F* c, int n) {
  c[0] = F(0);
  for (int k = 1; k < n; ++k) c[k] = s_inf<F>();
}
template <class F> void ln(const F* a, F* c, int n) {
  if (a[0] < F(0)) { nan_jet(c, n); return; }
  F inv_a0 = F(1) / a[0];
  c[0] = std::log(a[0]);
  for (int k = 1; k < n; ++k) {
    F sum = F(0);
    for (int j = 1; j < k; ++j) sum = sum + F(j) * c[j] * a[k - j];
    c[k] = (a[k] - sum / F(k)) * inv_a0;
  }
}
template <class F> void sqrt(const F* a, F* c, int n) {
  if (a[0] == F(0)) { vertical_tangent_jet(c, n); return; }
  if (a[0] < F(0)) { nan_jet(c, n); return; }
  c[0] = std::sqrt(a[0]);
  F two_c0 = F(2) * c[0];
  for (int k = 1; k < n; ++k) {
    F sum = F(0);
    for (int j = 1; j < k; ++j) sum = sum + c[j] * c[k - j];
    c[k] = (a[k] - sum) / two_c0;
  }
}
template <class F> void sin_cos(const F* a, F* s, F* co, int n) {
  s[0] = std::sin(a[0]);
  co[0] = std::cos(a[0]);
  for (int k = 1; k < n; ++k) {
    F inv_k = F(1) / F(k);
    F sum_s = F(0), sum_c = F(0);
    for (int j = 1; j <= k; ++j) {
      F jf = F(j);
      sum_s = sum_s + jf * a[j] * co[k - j];
      sum_c = sum_c + jf * a[j] * s[k - j];
    }
    s[k] = sum_s * inv_k;
    co[k] = -sum_c * inv_k;
  }
}
template <class F> void sinh_cosh(const F* a, F* sh, F* ch, int n) {
  sh[0] = std::sinh(a[0]);
  ch[0] = std::cosh(a[0]);
  for (int k = 1; k < n; ++k) {
    F inv_k = F(1) / F(k);
    F sum_sh = F(0), sum_ch = F(0);
    for (int j = 1; j <= k; ++j) {
      F jf = F(j);
      sum_sh = sum_sh + jf * a[j] * ch[k - j];
      sum_ch = sum_ch + jf * a[j] * sh[k - j];
    }
    sh[k] = sum_sh * inv_k;
    ch[k] = sum_ch * inv_k;
  }
}
template <class F> void integrate_from_deriv(const F* a, const F* g, F* c, int n) {
  for (int k = 1; k < n; ++k) {
    F sum = F(0);
    for (int j = 1; j <= k; ++j) sum = sum + F(j) * a[j] * g[k - j];
    c[k] = sum / F(k);
  }
}
template <class F> void atan(const F* a, F* c, F* s1, F* s2, int n) {
  mul(a, a, s1, n);
  for (int k = 0; k < n; ++k) s2[k] = s1[k];
  s2[0] = F(1) + s1[0];
  c[0] = std::atan(a[0]);
  recip(s2, s1, n);
  integrate_from_deriv(a, s1, c, n);
}
template <class F> void asin(const F* a, F* c, F* s1, F* s2, int n) {
  c[0] = std::asin(a[0]);
  mul(a, a, s1, n);
  s2[0] = (F(1) - a[0]) * (F(1) + a[0]);
  for (int k = 1; k < n; ++k) s2[k] = -s1[k];
  sqrt(s2, s1, n);
  recip(s1, s2, n);
  integrate_from_deriv(a, s2, c, n);
}
template <class F> void acos(const F* a, F* c, F* s1, F* s2, int n) {
  asin(a, c, s1, s2, n);
  c[0] = std::acos(a[0]);
  for (int k = 1; k < n; ++k) c[k] = -c[k];
}
template <class F> void tan(const F* a, F* c, F* sc, int n) {
  c[0] = std::tan(a[0]);
  sc[0] = F(1) + c[0] * c[0];
  for (int k = 1; k < n; ++k) {
    F sum = F(0);
    for (int j = 1; j <= k; ++j) sum = sum + F(j) * a[j] * sc[k - j];
    c[k] = sum / F(k);
    F s_k = F(0);
    for (int j = 0; j <= k; ++j) s_k = s_k + c[j] * c[k - j];
    sc[k] = s_k;
  }
}
template <class F> void tanh(const F* a, F* c, F* sc, int n) {
  c[0] = std::tanh(a[0]);
  sc[0] = F(1) - c[0] * c[0];
  for (int k = 1; k < n; ++k) {
    F sum = F(0);
    for (int j = 1; j <= k; ++j) sum = sum + F(j) * a[j] * sc[k - j];
    c[k] = sum / F(k);
    F s_k = F(0);
    for (int j = 0; j <= k; ++j) s_k = s_k + c[j] * c[k - j];
    sc[k] = -s_k;
  }
}
template <class F> void asinh(const F* a, F* c, F* s1, F* s2, int n) {
  c[0] = std::asinh(a[0]);
  mul(a, a, s1, n);
  for (int k = 0; k < n; ++k) s2[k] = s1[k];
  s2[0] = F(1) + s1[0];
  sqrt(s2, s1, n);
  recip(s1, s2, n);
  integrate_from_deriv(a, s2, c, n);
}
template <class F> void acosh(const F* a, F* c, F* s1, F* s2, int n) {
  if (a[0] < F(1)) { nan_jet(c, n); return; }
  c[0] = std::acosh(a[0]);
  mul(a, a, s1, n);
  for (int k = 0; k < n; ++k) s2[k] = s1[k];
  s2[0] = (a[0] - F(1)) * (a[0] + F(1));
  sqrt(s2, s1, n);
  recip(s1, s2, n);
  integrate_from_deriv(a, s2, c, n);
}
template <class F> void atanh(const F* a, F* c, F* s1, F* s2, int n) {
  if (a[0] < -F(1) || a[0] > F(1)) { nan_jet(c, n); return; }
  c[0] = std::atanh(a[0]);
  mul(a, a, s1, n);
  s2[0] = (F(1) - a[0]) * (F(1) + a[0]);
  for (int k = 1; k < n; ++k) s2[k] = -s1[k];
  recip(s2, s1, n);
  integrate_from_deriv(a, s1, c, n);
}
template <class F> void scale(const F* a, F s, F* c, int n) {
  for (int k = 0; k < n; ++k) c[k] = s * a[k];
}
template <class F> void powi_squaring(const F* a, int32_t nexp, F* c, F* s1, F* s2, int n) {
  uint32_t abs_n = nexp < 0 ? (uint32_t)(-(int64_t)nexp) : (uint32_t)nexp;
  c[0] = F(1);
  for (int k = 1; k < n; ++k) c[k] = F(0);
  for (int k = 0; k < n; ++k) s1[k] = a[k];
  uint32_t power = abs_n;
  while (power > 0) {
    if (power & 1u) {
      mul(c, s1, s2, n);
      for (int k = 0; k < n; ++k) c[k] = s2[k];
    }
    power >>= 1;
    if (power > 0) {
      for (int k = 0; k < n; ++k) {
        F sum = F(0);
        for (int j = 0; j <= k; ++j) sum = sum + s1[j] * s1[k - j];
        s2[k] = sum;
      }
      for (int k = 0; k < n; ++k) s1[k] = s2[k];
    }
  }
  if (nexp < 0) {
    for (int k = 0; k < n; ++k) s1[k] = c[k];
    recip(s1, c, n);
  }
}
template <class F> void powi(const F* a, int32_t nexp, F* c, F* s1, F* s2, int n) {
  if (nexp == 0) {
    c[0] = F(1);
    for (int k = 1; k < n; ++k) c[k] = F(0);
    return;
  }
  if (nexp == 1) { for (int k = 0; k < n; ++k) c[k] = a[k]; return; }
  if (nexp == -1) { recip(a, c, n); return; }
  uint32_t absn = nexp < 0 ? (uint32_t)(-(int64_t)nexp) : (uint32_t)nexp;
  if (a[0] <= F(0) || absn <= 8) {
    powi_squaring(a, nexp, c, s1, s2, n);
  } else {
    ln(a, s1, n);
    scale(s1, F(nexp), s2, n);
    exp(s2, c, n);
    c[0] = s_powi(a[0], nexp);
  }
}
template <class F> void powf(const F* a, const F* b, F* c, F* s1, F* s2, int n) {
  bool hi_zero = true;
  for (int k = 1; k < n; ++k) if (!(b[k] == F(0))) hi_zero = false;
  int32_t ni;
  if (hi_zero && s_as_i32(b[0], &ni)) { powi(a, ni, c, s1, s2, n); return; }
  if (a[0] == F(0)) {
    F b0 = b[0];
    int32_t bi;
    if (s_as_i32(b0, &bi)) { nan_jet(c, n); return; }
    c[0] = std::pow(a[0], b0);
    for (int k = 1; k < n; ++k) c[k] = (F(k) < b0) ? F(0) : s_inf<F>();
    return;
  }
  ln(a, s1, n);
  mul(b, s1, s2, n);
  exp(s2, c, n);
  if (a[0] < F(0)) c[0] = s_nan<F>();
  else c[0] = std::pow(a[0], b[0]);
}
template <class F> void cbrt(const F* a, F* c, F* s1, F* s2, int n) {
  if (a[0] == F(0)) { vertical_tangent_jet(c, n); return; }
  F third = F(1) / F(3);
  if (a[0] < F(0)) {
    for (int i = 0; i < n; ++i) c[i] = -a[i];
    ln(c, s1, n);
    scale(s1, third, s2, n);
    exp(s2, c, n);
    c[0] = std::cbrt(a[0]);
    for (int i = 1; i < n; ++i) c[i] = -c[i];
  } else {
    ln(a, s1, n);
    scale(s1, third, s2, n);
    exp(s2, c, n);
    c[0] = std::cbrt(a[0]);
  }
}
template <class F> void exp2(const F* a, F* c, F* s, int n) {
  F ln2 = std::log(F(2));
  scale(a, ln2, s, n);
  exp(s, c, n);
  c[0] = std::exp2(a[0]);
}
template <class F> void exp_m1(const F* a, F* c, int n) {
  exp(a, c, n);
  c[0] = std::expm1(a[0]);
}
template <class F> void log2(const F* a, F* c, int n) {
  ln(a, c, n);
  F inv_ln2 = F(1) / std::log(F(2));
  c[0] = std::log2(a[0]);
  for (int k = 1; k < n; ++k) c[k] = c[k] * inv_ln2;
}
template <class F> void log10(const F* a, F* c, int n) {
  ln(a, c, n);
  F inv_ln10 = F(1) / std::log(F(10));
  c[0] = std::log10(a[0]);
  for (int k = 1; k < n; ++k) c[k] = c[k] * inv_ln10;
}
template <class F> void ln_1p(const F* a, F* c, F* s, int n) {
  for (int k = 1; k < n; ++k) s[k] = a[k];
  s[0] = F(1) + a[0];
  ln(s, c, n);
  c[0] = std::log1p(a[0]);
}
template <class F> void hypot(const F* a, const F* b, F* c, F* s1, F* s2, int n) {
  int m = 0;
  if (std::fmax(std::fabs(a[0]), std::fabs(b[0])) == F(0)) {
    if (std::isnan(a[0]) || std::isnan(b[0])) { nan_jet(c, n); return; }
    int found = -1;
    for (int k = 1; k < n; ++k) if (a[k] != F(0) || b[k] != F(0)) { found = k; break; }
    if (found < 0) { for (int k = 0; k < n; ++k) c[k] = F(0); return; }
    m = found;
    if (std::isnan(a[m]) || std::isnan(b[m])) {
      for (int k = 0; k < m; ++k) c[k] = F(0);
      c[m] = std::hypot(a[m], b[m]);
      for (int k = m + 1; k < n; ++k) c[k] = s_nan<F>();
      return;
    }
  }
  // Rust Float::max: maxNum semantics (NaN dropped).
  F scl = std::fmax(std::fabs(a[m]), std::fabs(b[m]));
  F inv_scale = F(1) / scl;
  for (int k = 0; k < n; ++k) s1[k] = (k + m < n) ? a[k + m] * inv_scale : F(0);
  for (int k = 0; k < n; ++k) s2[k] = (k + m < n) ? b[k + m] * inv_scale : F(0);
  mul(s1, s1, c, n);
  mul(s2, s2, s1, n);
  for (int k = 0; k < n; ++k) c[k] = c[k] + s1[k];
  sqrt(c, s1, n);
  for (int k = 0; k < n; ++k) c[k] = s1[k] * scl;
  c[0] = std::hypot(a[m], b[m]);
  if (m > 0) {
    for (int k = n - 1; k >= m; --k) c[k] = c[k - m];
    for (int k = 0; k < m; ++k) c[k] = F(0);
  }
}
template <class F> void discontinuous(F val, F* c, int n) {
  c[0] = val;
  for (int k = 1; k < n; ++k) c[k] = F(0);
}
template <class F> void atan2(const F* a, const F* b, F* c, F* s1, F* s2, F* s3, int n) {
  if (b[0] != F(0)) {
    div(a, b, s1, n);
    atan(s1, c, s2, s3, n);
    c[0] = std::atan2(a[0], b[0]);
  } else if (a[0] != F(0)) {
    div(b, a, s1, n);
    atan(s1, c, s2, s3, n);
    for (int k = 0; k < n; ++k) c[k] = -c[k];
    c[0] = std::atan2(a[0], b[0]);
  } else {
    discontinuous(F(0), c, n);
  }
}
}  // namespace tops

// ───────────────────────── uniform "Float" interface ───────────────────────
// prim(): the primal value (Dual::re, Taylor::coeffs[0]) that comparisons and
// classification predicates inspect (num_traits_impls.rs:207-227,
// taylor_num_traits.rs:199-207).
template <class F> inline F prim(F x) { return x; }
template <class F> inline F prim(Dual<F> x) { return x.re; }
template <class F, int K> inline F prim(const Tay<F, K>& x) { return x.c[0]; }

template <class T> struct M;  // math for T

template <class F> struct MScalar {
  using T = F;
  static T c(double v) { return (F)v; }
  static T fromF(F v) { return v; }
  static T add(T a, T b) { return a + b; }
  static T sub(T a, T b) { return a - b; }
  static T mul(T a, T b) { return a * b; }
  static T div(T a, T b) { return a / b; }
  static T neg(T a) { return -a; }
  static T rem(T a, T b) { return std::fmod(a, b); }
  static T powf(T a, T b) { return std::pow(a, b); }
  static T atan2(T a, T b) { return std::atan2(a, b); }
  static T hypot(T a, T b) { return std::hypot(a, b); }
  static T recip(T a) { return F(1) / a; }
  static T sqrt(T a) { return std::sqrt(a); }
  static T cbrt(T a) { return std::cbrt(a); }
  static T powi(T a, int32_t n) { return s_powi(a, n); }
  static T exp(T a) { return std::exp(a); }
  static T exp2(T a) { return std::exp2(a); }
  static T exp_m1(T a) { return std::expm1(a); }
  static T ln(T a) { return std::log(a); }
  static T log2(T a) { return std::log2(a); }
  static T log10(T a) { return std::log10(a); }
  static T ln_1p(T a) { return std::log1p(a); }
  static T sin(T a) { return std::sin(a); }
  static T cos(T a) { return std::cos(a); }
  static T tan(T a) { return std::tan(a); }
  static T asin(T a) { return std::asin(a); }
  static T acos(T a) { return std::acos(a); }
  static T atan(T a) { return std::atan(a); }
  static T sinh(T a) { return std::sinh(a); }
  static T cosh(T a) { return std::cosh(a); }
  static T tanh(T a) { return std::tanh(a); }
  static T asinh(T a) { return std::asinh(a); }
  static T acosh(T a) { return std::acosh(a); }
  static T atanh(T a) { return std::atanh(a); }
  static T abs(T a) { return std::fabs(a); }
  static T signum(T a) { return s_signum(a); }
  static T floor(T a) { return std::floor(a); }
  static T ceil(T a) { return std::ceil(a); }
  static T round(T a) { return std::round(a); }
  static T trunc(T a) { return std::trunc(a); }
  static T fract(T a) { return s_fract(a); }
  static bool all_zero(T a) { return a == F(0); }
  static T nan() { return s_nan<F>(); }
};
template <> struct M<double> : MScalar<double> {};
template <> struct M<float> : MScalar<float> {};

// kernels (src/kernels/mod.rs:85-285), generic over T.
template <class T> std::pair<T, T> hypot_partials(T a, T b, T r) {
  using Mt = M<T>;
  if (prim(r) == 0) return {Mt::c(0), Mt::c(0)};
  return {Mt::div(a, r), Mt::div(b, r)};
}
template <class T> std::pair<T, T> atan2_partials(T a, T b) {
  using Mt = M<T>;
  T h = Mt::hypot(a, b);
  if (prim(h) == 0) return {Mt::c(0), Mt::c(0)};
  return {Mt::div(Mt::div(b, h), h), Mt::div(Mt::div(Mt::neg(a), h), h)};
}
template <class T> T atan_deriv(T a) {
  using Mt = M<T>;
  T one = Mt::c(1);
  if (prim(Mt::abs(a)) > 1e8) {
    T inv = Mt::div(one, a);
    return Mt::div(Mt::mul(inv, inv), Mt::add(one, Mt::mul(inv, inv)));
  }
  return Mt::div(one, Mt::add(one, Mt::mul(a, a)));
}
template <class T> T asinh_deriv(T a) {
  using Mt = M<T>;
  T one = Mt::c(1);
  if (prim(Mt::abs(a)) > 1e8) {
    T inv = Mt::div(one, a);
    return Mt::div(Mt::abs(inv), Mt::sqrt(Mt::add(one, Mt::mul(inv, inv))));
  }
  return Mt::div(one, Mt::sqrt(Mt::add(Mt::mul(a, a), one)));
}
template <class T> T acosh_deriv(T a) {
  using Mt = M<T>;
  T one = Mt::c(1);
  if (prim(a) < prim(one)) return Mt::nan();
  if (prim(a) > 1e8) {
    T inv = Mt::div(one, a);
    return Mt::div(Mt::abs(inv), Mt::sqrt(Mt::sub(one, Mt::mul(inv, inv))));
  }
  return Mt::div(one, Mt::sqrt(Mt::mul(Mt::sub(a, one), Mt::add(a, one))));
}
template <class T> T ln_deriv(T a) {
  using Mt = M<T>;
  if (prim(a) >= 0) return Mt::div(Mt::c(1), a);
  return Mt::nan();
}
template <class T> T log2_deriv(T a) {
  using Mt = M<T>;
  if (prim(a) >= 0) return Mt::div(Mt::c(1), Mt::mul(a, Mt::c(kLN2)));
  return Mt::nan();
}
template <class T> T log10_deriv(T a) {
  using Mt = M<T>;
  if (prim(a) >= 0) return Mt::div(Mt::c(1), Mt::mul(a, Mt::c(kLN10)));
  return Mt::nan();
}
template <class T> T ln_1p_deriv(T a) {
  using Mt = M<T>;
  if (prim(a) >= prim(Mt::neg(Mt::c(1)))) return Mt::div(Mt::c(1), Mt::add(Mt::c(1), a));
  return Mt::nan();
}
template <class T> T atanh_deriv(T a) {
  using Mt = M<T>;
  T one = Mt::c(1);
  if (prim(a) >= prim(Mt::neg(one)) && prim(a) <= prim(one))
    return Mt::div(one, Mt::mul(Mt::sub(one, a), Mt::add(one, a)));
  return Mt::nan();
}
template <class T> T abs_deriv(T a) {
  using Mt = M<T>;
  if (prim(a) == 0) return Mt::c(0);
  return Mt::signum(a);
}

// Dual<F> math (src/dual.rs).
template <class F> struct M<Dual<F>> {
  using T = Dual<F>;
  using S = MScalar<F>;
  static T c(double v) { return {(F)v, F(0)}; }
  static T add(T a, T b) { return a + b; }
  static T sub(T a, T b) { return a - b; }
  static T mul(T a, T b) { return a * b; }
  static T div(T a, T b) { return a / b; }
  static T neg(T a) { return -a; }
  static T rem(T a, T b) { return {std::fmod(a.re, b.re), a.eps - b.eps * std::trunc(a.re / b.re)}; }
  static T chain(T x, F fv, F fd) { return {fv, (x.eps == F(0)) ? F(0) : x.eps * fd}; }
  static T recip(T a) { F inv = F(1) / a.re; return chain(a, inv, -inv * inv); }
  static T sqrt(T a) { F s = std::sqrt(a.re); F two = F(1) + F(1); return chain(a, s, F(1) / (two * s)); }
  static T cbrt(T a) { F c = std::cbrt(a.re); F three = F(3); return chain(a, c, F(1) / (three * c * c)); }
  static T powi(T a, int32_t n) {
    if (n == 0) return c(1);
    F val = s_powi(a.re, n);
    F deriv = (n == std::numeric_limits<int32_t>::min()) ? F(n) * val / a.re : F(n) * s_powi(a.re, n - 1);
    return chain(a, val, deriv);
  }
  static T exp(T a) { F e = std::exp(a.re); return chain(a, e, e); }
  static T exp2(T a) { F e = std::exp2(a.re); return chain(a, e, e * (F)kLN2); }
  static T exp_m1(T a) { return chain(a, std::expm1(a.re), std::exp(a.re)); }
  static T ln(T a) { return chain(a, std::log(a.re), ln_deriv<F>(a.re)); }
  static T log2(T a) { return chain(a, std::log2(a.re), log2_deriv<F>(a.re)); }
  static T log10(T a) { return chain(a, std::log10(a.re), log10_deriv<F>(a.re)); }
  static T ln_1p(T a) { return chain(a, std::log1p(a.re), ln_1p_deriv<F>(a.re)); }
  static T sin(T a) { return chain(a, std::sin(a.re), std::cos(a.re)); }
  static T cos(T a) { return chain(a, std::cos(a.re), -std::sin(a.re)); }
  static T tan(T a) { F c = std::cos(a.re); return chain(a, std::tan(a.re), F(1) / (c * c)); }
  static T asin(T a) { return chain(a, std::asin(a.re), F(1) / std::sqrt((F(1) - a.re) * (F(1) + a.re))); }
  static T acos(T a) { return chain(a, std::acos(a.re), -F(1) / std::sqrt((F(1) - a.re) * (F(1) + a.re))); }
  static T atan(T a) { return chain(a, std::atan(a.re), atan_deriv<F>(a.re)); }
  static T sinh(T a) { return chain(a, std::sinh(a.re), std::cosh(a.re)); }
  static T cosh(T a) { return chain(a, std::cosh(a.re), std::sinh(a.re)); }
  static T tanh(T a) { F c = std::cosh(a.re); return chain(a, std::tanh(a.re), F(1) / (c * c)); }
  static T asinh(T a) { return chain(a, std::asinh(a.re), asinh_deriv<F>(a.re)); }
  static T acosh(T a) { return chain(a, std::acosh(a.re), acosh_deriv<F>(a.re)); }
  static T atanh(T a) { return chain(a, std::atanh(a.re), atanh_deriv<F>(a.re)); }
  static T abs(T a) { return chain(a, std::fabs(a.re), abs_deriv<F>(a.re)); }
  static T signum(T a) { return c0(s_signum(a.re)); }
  static T floor(T a) { return c0(std::floor(a.re)); }
  static T ceil(T a) { return c0(std::ceil(a.re)); }
  static T round(T a) { return c0(std::round(a.re)); }
  static T trunc(T a) { return c0(std::trunc(a.re)); }
  static T fract(T a) { return {s_fract(a.re), a.eps}; }
  static T c0(F v) { return {v, F(0)}; }
  static T fromF(F v) { return c0(v); }
  static bool all_zero(T a) { return a.re == F(0) && a.eps == F(0); }
  static T nan() { return c0(s_nan<F>()); }
  static T powf(T self, T n) {
    int32_t ni;
    if (n.eps == F(0) && s_as_i32(n.re, &ni)) return powi(self, ni);
    if (n.re == F(0)) {
      F dy = (self.re > F(0)) ? std::log(self.re) : F(0);
      return {F(1), dy * n.eps};
    }
    F val = std::pow(self.re, n.re);
    F dx;
    if (self.eps == F(0)) {
      dx = F(0);
    } else if (self.re == F(0) || val == F(0) || !std::isfinite(self.re) || !std::isfinite(val)) {
      dx = n.re * std::pow(self.re, n.re - F(1)) * self.eps;
    } else {
      dx = n.re * val / self.re * self.eps;
    }
    F dy;
    if (n.eps == F(0) || val == F(0) || self.re <= F(0)) dy = F(0);
    else dy = val * std::log(self.re) * n.eps;
    return {val, dx + dy};
  }
  static T atan2(T self, T other) {
    auto p = atan2_partials<F>(self.re, other.re);
    return {std::atan2(self.re, other.re), p.first * self.eps + p.second * other.eps};
  }
  static T hypot(T self, T other) {
    F h = std::hypot(self.re, other.re);
    if (h == F(0)) return c0(h);
    auto p = hypot_partials<F>(self.re, other.re, h);
    return {h, p.first * self.eps + p.second * other.eps};
  }
};

// Taylor<F,K> math (src/taylor.rs, src/traits/taylor_std_ops.rs).
template <class F, int K> struct M<Tay<F, K>> {
  using T = Tay<F, K>;
  static T c(double v) { T t; t.c[0] = (F)v; for (int k = 1; k < K; ++k) t.c[k] = F(0); return t; }
  static T c0(F v) { T t; t.c[0] = v; for (int k = 1; k < K; ++k) t.c[k] = F(0); return t; }
  static T fromF(F v) { return c0(v); }
  static T add(const T& a, const T& b) { T r; for (int k = 0; k < K; ++k) r.c[k] = a.c[k] + b.c[k]; return r; }
  static T sub(const T& a, const T& b) { T r; for (int k = 0; k < K; ++k) r.c[k] = a.c[k] - b.c[k]; return r; }
  static T mul(const T& a, const T& b) { T r; tops::mul(a.c, b.c, r.c, K); return r; }
  static T div(const T& a, const T& b) { T r; tops::div(a.c, b.c, r.c, K); return r; }
  static T neg(const T& a) { T r; for (int k = 0; k < K; ++k) r.c[k] = -a.c[k]; return r; }
  static T rem(const T& a, const T& b) {
    T r;
    if (b.c[0] == F(0)) { for (int k = 0; k < K; ++k) r.c[k] = s_nan<F>(); return r; }
    F q = std::trunc(a.c[0] / b.c[0]);
    for (int k = 0; k < K; ++k) r.c[k] = (k == 0) ? std::fmod(a.c[0], b.c[0]) : a.c[k] - b.c[k] * q;
    return r;
  }
  static T powf(const T& a, const T& b) { T r, s1, s2; tops::powf(a.c, b.c, r.c, s1.c, s2.c, K); return r; }
  static T atan2(const T& a, const T& b) { T r, s1, s2, s3; tops::atan2(a.c, b.c, r.c, s1.c, s2.c, s3.c, K); return r; }
  static T hypot(const T& a, const T& b) { T r, s1, s2; tops::hypot(a.c, b.c, r.c, s1.c, s2.c, K); return r; }
  static T recip(const T& a) { T r; tops::recip(a.c, r.c, K); return r; }
  static T sqrt(const T& a) { T r; tops::sqrt(a.c, r.c, K); return r; }
  static T cbrt(const T& a) { T r, s1, s2; tops::cbrt(a.c, r.c, s1.c, s2.c, K); return r; }
  static T powi(const T& a, int32_t n) { T r, s1, s2; tops::powi(a.c, n, r.c, s1.c, s2.c, K); return r; }
  static T exp(const T& a) { T r; tops::exp(a.c, r.c, K); return r; }
  static T exp2(const T& a) { T r, s; tops::exp2(a.c, r.c, s.c, K); return r; }
  static T exp_m1(const T& a) { T r; tops::exp_m1(a.c, r.c, K); return r; }
  static T ln(const T& a) { T r; tops::ln(a.c, r.c, K); return r; }
  static T log2(const T& a) { T r; tops::log2(a.c, r.c, K); return r; }
  static T log10(const T& a) { T r; tops::log10(a.c, r.c, K); return r; }
  static T ln_1p(const T& a) { T r, s; tops::ln_1p(a.c, r.c, s.c, K); return r; }
  static T sin(const T& a) { T s, co; tops::sin_cos(a.c, s.c, co.c, K); return s; }
  static T cos(const T& a) { T s, co; tops::sin_cos(a.c, s.c, co.c, K); return co; }
  static T tan(const T& a) { T r, s; tops::tan(a.c, r.c, s.c, K); return r; }
  static T asin(const T& a) { T r, s1, s2; tops::asin(a.c, r.c, s1.c, s2.c, K); return r; }
  static T acos(const T& a) { T r, s1, s2; tops::acos(a.c, r.c, s1.c, s2.c, K); return r; }
  static T atan(const T& a) { T r, s1, s2; tops::atan(a.c, r.c, s1.c, s2.c, K); return r; }
  static T sinh(const T& a) { T sh, ch; tops::sinh_cosh(a.c, sh.c, ch.c, K); return sh; }
  static T cosh(const T& a) { T sh, ch; tops::sinh_cosh(a.c, sh.c, ch.c, K); return ch; }
  static T tanh(const T& a) { T r, s; tops::tanh(a.c, r.c, s.c, K); return r; }
  static T asinh(const T& a) { T r, s1, s2; tops::asinh(a.c, r.c, s1.c, s2.c, K); return r; }
  static T acosh(const T& a) { T r, s1, s2; tops::acosh(a.c, r.c, s1.c, s2.c, K); return r; }
  static T atanh(const T& a) { T r, s1, s2; tops::atanh(a.c, r.c, s1.c, s2.c, K); return r; }
  static T abs(const T& a) {
    F sign;
    if (a.c[0] != F(0)) sign = s_signum(a.c[0]);
    else {
      sign = F(1);
      for (int k = 1; k < K; ++k) if (a.c[k] != F(0)) { sign = s_signum(a.c[k]); break; }
    }
    T r;
    for (int k = 0; k < K; ++k) r.c[k] = a.c[k] * sign;
    return r;
  }
  static T signum(const T& a) { return c0(s_signum(a.c[0])); }
  static T floor(const T& a) { return c0(std::floor(a.c[0])); }
  static T ceil(const T& a) { return c0(std::ceil(a.c[0])); }
  static T round(const T& a) { return c0(std::round(a.c[0])); }
  static T trunc(const T& a) { return c0(std::trunc(a.c[0])); }
  static T fract(const T& a) { T r = a; r.c[0] = s_fract(a.c[0]); return r; }
  static bool all_zero(const T& a) { for (int k = 0; k < K; ++k) if (a.c[k] != F(0)) return false; return true; }
  static T nan() { return c0(s_nan<F>()); }
};

// ───────────────────────── opcode dispatch (src/opcode.rs) ──────────────────
template <class T> T eval_forward(uint32_t op, T a, T b) {
  using Mt = M<T>;
  switch (op) {
    case ADD: return Mt::add(a, b);
    case SUB: return Mt::sub(a, b);
    case MUL: return Mt::mul(a, b);
    case DIV: return Mt::div(a, b);
    case REM: return Mt::rem(a, b);
    case POWF: return Mt::powf(a, b);
    case ATAN2: return Mt::atan2(a, b);
    case HYPOT: return Mt::hypot(a, b);
    case MAX: return (prim(a) >= prim(b) || std::isnan(prim(b))) ? a : b;
    case MIN: return (prim(a) <= prim(b) || std::isnan(prim(b))) ? a : b;
    case NEG: return Mt::neg(a);
    case RECIP: return Mt::recip(a);
    case SQRT: return Mt::sqrt(a);
    case CBRT: return Mt::cbrt(a);
    case EXP: return Mt::exp(a);
    case EXP2: return Mt::exp2(a);
    case EXPM1: return Mt::exp_m1(a);
    case LN: return Mt::ln(a);
    case LOG2: return Mt::log2(a);
    case LOG10: return Mt::log10(a);
    case LN1P: return Mt::ln_1p(a);
    case SIN: return Mt::sin(a);
    case COS: return Mt::cos(a);
    case TAN: return Mt::tan(a);
    case ASIN: return Mt::asin(a);
    case ACOS: return Mt::acos(a);
    case ATAN: return Mt::atan(a);
    case SINH: return Mt::sinh(a);
    case COSH: return Mt::cosh(a);
    case TANH: return Mt::tanh(a);
    case ASINH: return Mt::asinh(a);
    case ACOSH: return Mt::acosh(a);
    case ATANH: return Mt::atanh(a);
    case ABS: return Mt::abs(a);
    case SIGNUM: return Mt::signum(a);
    case FLOOR: return Mt::floor(a);
    case CEIL: return Mt::ceil(a);
    case ROUND: return Mt::round(a);
    case TRUNC: return Mt::trunc(a);
    case FRACT: return Mt::fract(a);
    default: return Mt::nan();
  }
}

template <class T> std::pair<T, T> reverse_partials(uint32_t op, T a, T b, T r) {
  using Mt = M<T>;
  T zero = Mt::c(0), one = Mt::c(1);
  switch (op) {
    case ADD: return {one, one};
    case SUB: return {one, Mt::neg(one)};
    case MUL: return {b, a};
    case DIV: { T inv = Mt::div(one, b); return {inv, Mt::mul(Mt::neg(r), inv)}; }
    case REM: return {one, Mt::neg(Mt::trunc(Mt::div(a, b)))};
    case POWF: {
      if (prim(b) == 0) {
        T db = (prim(a) > 0) ? Mt::ln(a) : zero;
        return {zero, db};
      }
      T da;
      if (prim(a) == 0 || prim(r) == 0 || !std::isfinite(prim(a)) || !std::isfinite(prim(r)))
        da = Mt::mul(b, Mt::powf(a, Mt::sub(b, one)));
      else
        da = Mt::div(Mt::mul(b, r), a);
      T db = (prim(r) == 0 || prim(a) <= 0) ? zero : Mt::mul(r, Mt::ln(a));
      return {da, db};
    }
    case ATAN2: return atan2_partials<T>(a, b);
    case HYPOT: return hypot_partials<T>(a, b, r);
    case MAX: return (prim(a) >= prim(b) || std::isnan(prim(b))) ? std::make_pair(one, zero) : std::make_pair(zero, one);
    case MIN: return (prim(a) <= prim(b) || std::isnan(prim(b))) ? std::make_pair(one, zero) : std::make_pair(zero, one);
    case NEG: return {Mt::neg(one), zero};
    case RECIP: { T inv = Mt::div(one, a); return {Mt::mul(Mt::neg(inv), inv), zero}; }
    case SQRT: { T two = Mt::add(one, one); return {Mt::div(one, Mt::mul(two, r)), zero}; }
    case CBRT: { T three = Mt::c(3.0); return {Mt::div(one, Mt::mul(Mt::mul(three, r), r)), zero}; }
    case EXP: return {r, zero};
    case EXP2: return {Mt::mul(r, Mt::c(kLN2)), zero};
    case EXPM1: return {Mt::add(r, one), zero};
    case LN: return {ln_deriv<T>(a), zero};
    case LOG2: return {log2_deriv<T>(a), zero};
    case LOG10: return {log10_deriv<T>(a), zero};
    case LN1P: return {ln_1p_deriv<T>(a), zero};
    case SIN: return {Mt::cos(a), zero};
    case COS: return {Mt::neg(Mt::sin(a)), zero};
    case TAN: { T c = Mt::cos(a); return {Mt::div(one, Mt::mul(c, c)), zero}; }
    case ASIN: return {Mt::div(one, Mt::sqrt(Mt::mul(Mt::sub(one, a), Mt::add(one, a)))), zero};
    case ACOS: return {Mt::div(Mt::neg(one), Mt::sqrt(Mt::mul(Mt::sub(one, a), Mt::add(one, a)))), zero};
    case ATAN: return {atan_deriv<T>(a), zero};
    case SINH: return {Mt::cosh(a), zero};
    case COSH: return {Mt::sinh(a), zero};
    case TANH: { T c = Mt::cosh(a); return {Mt::div(one, Mt::mul(c, c)), zero}; }
    case ASINH: return {asinh_deriv<T>(a), zero};
    case ACOSH: return {acosh_deriv<T>(a), zero};
    case ATANH: return {atanh_deriv<T>(a), zero};
    case ABS: return {abs_deriv<T>(a), zero};
    case SIGNUM: case FLOOR: case CEIL: case ROUND: case TRUNC: return {zero, zero};
    case FRACT: return {one, zero};
    default: return {zero, zero};
  }
}

template <class T> T powi_reverse_partial(int32_t e, T a, T r) {
  using Mt = M<T>;
  if (e == 0) return Mt::c(0);
  if (e == std::numeric_limits<int32_t>::min()) return Mt::div(Mt::mul(Mt::c((double)e), r), a);
  return Mt::mul(Mt::c((double)e), Mt::powi(a, e - 1));
}

// ───────────────────────── tape + sweeps ────────────────────────────────────
template <class F> struct Tape {
  const uint32_t* op;
  const uint32_t* a0;
  const uint32_t* a1;
  const F* vals;
  uint32_t nv, ni, out_idx;
  const uint32_t* outs;
  uint32_t nout;
};

// forward_into + forward_dispatch (src/bytecode_tape/forward.rs:11-43, 194-229)
template <class F> void forward_into(const Tape<F>& t, const F* x, std::vector<F>& v) {
  v.assign(t.vals, t.vals + t.nv);
  for (uint32_t i = 0; i < t.ni; ++i) v[i] = x[i];
  for (uint32_t i = 0; i < t.nv; ++i) {
    uint32_t op = t.op[i];
    if (op == INPUT || op == CONST) continue;
    F a = v[t.a0[i]];
    if (op == POWI) { v[i] = s_powi(a, (int32_t)t.a1[i]); continue; }
    F b = (t.a1[i] != UNUSED) ? v[t.a1[i]] : F(0);
    v[i] = eval_forward<F>(op, a, b);
  }
}

// reverse_sweep_core (src/bytecode_tape/reverse.rs:32-105)
template <class F> void reverse_from(const Tape<F>& t, const std::vector<F>& v, std::vector<F>& adj, uint32_t seed) {
  adj.assign(t.nv, F(0));
  adj[seed] = F(1);
  for (int64_t ii = (int64_t)t.nv - 1; ii >= 0; --ii) {
    uint32_t i = (uint32_t)ii;
    F ad = adj[i];
    if (ad == F(0)) continue;
    uint32_t op = t.op[i];
    if (op == INPUT || op == CONST) continue;
    adj[i] = F(0);
    uint32_t ai = t.a0[i], bi = t.a1[i];
    F a = v[ai];
    if (op == POWI) {
      F da = powi_reverse_partial<F>((int32_t)bi, a, v[i]);
      if (da != F(0)) adj[ai] = adj[ai] + da * ad;
      continue;
    }
    F b = (bi != UNUSED) ? v[bi] : F(0);
    auto p = reverse_partials<F>(op, a, b, v[i]);
    if (p.first != F(0)) adj[ai] = adj[ai] + p.first * ad;
    if (bi != UNUSED && p.second != F(0)) adj[bi] = adj[bi] + p.second * ad;
  }
}

// forward_tangent_inner (src/bytecode_tape/tangent.rs:97-147)
template <class F, class T> void forward_tangent(const Tape<F>& t, const T* inputs, std::vector<T>& buf) {
  using Mt = M<T>;
  buf.assign(t.nv, Mt::c(0));
  uint32_t k = 0;
  for (uint32_t i = 0; i < t.nv; ++i) {
    uint32_t op = t.op[i];
    if (op == INPUT) { buf[i] = inputs[k++]; continue; }
    if (op == CONST) { buf[i] = Mt::fromF(t.vals[i]); continue; }
    T a = buf[t.a0[i]];
    if (op == POWI) { buf[i] = Mt::powi(a, (int32_t)t.a1[i]); continue; }
    T b = (t.a1[i] != UNUSED) ? buf[t.a1[i]] : Mt::c(0);
    buf[i] = eval_forward<T>(op, a, b);
  }
}

}  // namespace orc

namespace orc {

// reverse_tangent_inner (src/bytecode_tape/tangent.rs:191-262)
template <class F, class T> void reverse_tangent(const Tape<F>& t, const std::vector<T>& tv, std::vector<T>& buf) {
  using Mt = M<T>;
  buf.assign(t.nv, Mt::c(0));
  buf[t.out_idx] = Mt::c(1);
  for (int64_t ii = (int64_t)t.nv - 1; ii >= 0; --ii) {
    uint32_t i = (uint32_t)ii;
    uint32_t op = t.op[i];
    if (op == INPUT || op == CONST) continue;
    T adj = buf[i];
    if (Mt::all_zero(adj)) continue;
    buf[i] = Mt::c(0);
    uint32_t ai = t.a0[i], bi = t.a1[i];
    T a = tv[ai];
    if (op == POWI) {
      T da = powi_reverse_partial<T>((int32_t)bi, a, tv[i]);
      if (!Mt::all_zero(da)) buf[ai] = Mt::add(buf[ai], Mt::mul(da, adj));
      continue;
    }
    T b = (bi != UNUSED) ? tv[bi] : Mt::c(0);
    auto p = reverse_partials<T>(op, a, b, tv[i]);
    if (!Mt::all_zero(p.first)) buf[ai] = Mt::add(buf[ai], Mt::mul(p.first, adj));
    if (bi != UNUSED && !Mt::all_zero(p.second)) buf[bi] = Mt::add(buf[bi], Mt::mul(p.second, adj));
  }
}

// hvp (src/bytecode_tape/tangent.rs:268-310): forward_tangent_dual + reverse_tangent_dual.
template <class F> void hvp_point(const Tape<F>& t, const F* x, const F* v, F* grad, F* hv,
                                  std::vector<Dual<F>>& din, std::vector<Dual<F>>& dv, std::vector<Dual<F>>& adj) {
  din.resize(t.ni);
  for (uint32_t i = 0; i < t.ni; ++i) din[i] = {x[i], v[i]};
  forward_tangent<F, Dual<F>>(t, din.data(), dv);
  reverse_tangent<F, Dual<F>>(t, dv, adj);
  for (uint32_t i = 0; i < t.ni; ++i) { grad[i] = adj[i].re; hv[i] = adj[i].eps; }
}

// Taylor jet along x + t v: inputs [x_i, v_i, 0, ...] (src/stde/jet.rs:26-46,
// src/stde/higher_order.rs:239-267).  Output coefficients of every declared output.
template <class F, int K> void taylor_point(const Tape<F>& t, const F* x, const F* v, F* out /*nout*K*/,
                                            std::vector<Tay<F, K>>& in, std::vector<Tay<F, K>>& buf) {
  in.resize(t.ni);
  for (uint32_t i = 0; i < t.ni; ++i) {
    for (int k = 0; k < K; ++k) in[i].c[k] = F(0);
    in[i].c[0] = x[i];
    if (K > 1) in[i].c[1] = v[i];
  }
  forward_tangent<F, Tay<F, K>>(t, in.data(), buf);
  for (uint32_t j = 0; j < t.nout; ++j)
    for (int k = 0; k < K; ++k) out[j * K + k] = buf[t.outs[j]].c[k];
}

// WelfordAccumulator (src/stde/types.rs:44-113)
template <class F> struct Welford {
  F mean = F(0), m2 = F(0);
  size_t count = 0;
  void update(F s) {
    if (!std::isfinite(s)) return;
    count += 1;
    F k1 = (F)count;
    F delta = s - mean;
    mean = mean + delta / k1;
    F delta2 = s - mean;
    m2 = m2 + delta * delta2;
  }
  void finalize(F* est, F* var, F* se) const {
    if (count == 0) { *est = s_nan<F>(); *var = F(0); *se = F(0); return; }
    F nf = (F)count;
    if (count > 1) {
      F v = std::fmax(m2 / (nf - F(1)), F(0));  // Rust Float::max(0): maxNum
      *est = mean; *var = v; *se = std::sqrt(v / nf);
    } else {
      *est = mean; *var = F(0); *se = F(0);
    }
  }
};

template <class Fn> void parallel_for(uint64_t n, int nthreads, Fn fn) {
  if (nthreads <= 1 || n < 2) { fn(0, n, 0); return; }
  int nt = (int)std::min<uint64_t>((uint64_t)nthreads, n);
  std::vector<std::thread> th;
  uint64_t chunk = (n + nt - 1) / nt;
  for (int w = 0; w < nt; ++w) {
    uint64_t lo = w * chunk, hi = std::min<uint64_t>(n, lo + chunk);
    if (lo >= hi) break;
    th.emplace_back([=] { fn(lo, hi, w); });
  }
  for (auto& x : th) x.join();
}

template <class F, int K>
void taylor_batch_k(const Tape<F>& t, const F* P, const F* S, uint64_t B, F* coeffs, int nth) {
  parallel_for(B, nth, [&](uint64_t lo, uint64_t hi, int) {
    std::vector<Tay<F, K>> in, buf;
    std::vector<F> tmp(t.nout * K);
    for (uint64_t b = lo; b < hi; ++b) {
      taylor_point<F, K>(t, P + b * t.ni, S + b * t.ni, tmp.data(), in, buf);
      for (uint32_t j = 0; j < t.nout; ++j)
        for (int k = 0; k < K; ++k) coeffs[(uint64_t)k * B * t.nout + b * t.nout + j] = tmp[j * K + k];
    }
  });
}

template <class F>
int taylor_batch(const Tape<F>& t, int K, const F* P, const F* S, uint64_t B, F* coeffs, int nth) {
  switch (K) {
    case 1: taylor_batch_k<F, 1>(t, P, S, B, coeffs, nth); return 0;
    case 2: taylor_batch_k<F, 2>(t, P, S, B, coeffs, nth); return 0;
    case 3: taylor_batch_k<F, 3>(t, P, S, B, coeffs, nth); return 0;
    case 4: taylor_batch_k<F, 4>(t, P, S, B, coeffs, nth); return 0;
    case 5: taylor_batch_k<F, 5>(t, P, S, B, coeffs, nth); return 0;
    case 6: taylor_batch_k<F, 6>(t, P, S, B, coeffs, nth); return 0;
    case 7: taylor_batch_k<F, 7>(t, P, S, B, coeffs, nth); return 0;
    default: return -1;
  }
}

// Per-point Hutchinson Laplacian with statistics: estimate(&Laplacian, ...)
// (src/stde/pipeline.rs:19-38).  out = {value, estimate, variance, se, num_samples}.
template <class F> void laplacian_stats_point(const Tape<F>& t, const F* x, const F* dirs, uint32_t S, F* out,
                                              std::vector<Tay<F, 3>>& in, std::vector<Tay<F, 3>>& buf) {
  Welford<F> acc;
  F value = F(0);
  F jet[3 * 64];
  std::vector<F> jv;
  if (t.nout * 3 > 3 * 64) jv.resize(t.nout * 3);
  F* j = (t.nout * 3 > 3 * 64) ? jv.data() : jet;
  for (uint32_t s = 0; s < S; ++s) {
    taylor_point<F, 3>(t, x, dirs + (uint64_t)s * t.ni, j, in, buf);
    // taylor_jet_2nd reads buf[output_index]
    F c0 = buf[t.out_idx].c[0], c2 = buf[t.out_idx].c[2];
    value = c0;
    acc.update(F(2) * c2);
  }
  F est, var, se;
  acc.finalize(&est, &var, &se);
  out[0] = value; out[1] = est; out[2] = var; out[3] = se; out[4] = (F)acc.count;
}

// stde_sparse (src/stde/sparse.rs:37-78): per sampled entry e in order, input
// jets c0 = x_i with coefficient slots[q] of input vars[q] set to coefs[q]
// (seed_taylor_dyn_jets), one forward jet sweep, raw = c_{kout[e]} * pref[e],
// sample = sign[e] * Z * raw into a Welford accumulator; value = c0 of the
// primary output.  out = {value, estimate, variance, se, num_samples}.
template <class F, int K>
void stde_sparse_k(const Tape<F>& t, const F* x, const uint32_t* off, const uint32_t* vars, const uint32_t* slots,
                   const F* coefs, const uint32_t* kout, const F* pref, const F* sign, F z, const uint64_t* idx,
                   uint64_t nidx, F* out) {
  std::vector<Tay<F, K>> in(t.ni), buf;
  Welford<F> acc;
  F value = F(0);
  for (uint64_t s = 0; s < nidx; ++s) {
    const uint64_t e = idx[s];
    for (uint32_t i = 0; i < t.ni; ++i) {
      for (int k = 0; k < K; ++k) in[i].c[k] = F(0);
      in[i].c[0] = x[i];
    }
    for (uint32_t q = off[e]; q < off[e + 1]; ++q)
      if (slots[q] < (uint32_t)K) in[vars[q]].c[slots[q]] = coefs[q];
    forward_tangent<F, Tay<F, K>>(t, in.data(), buf);
    const Tay<F, K>& o = buf[t.out_idx];
    value = o.c[0];
    const F raw = o.c[kout[e]] * pref[e];
    const F sample = sign[e] * z * raw;
    acc.update(sample);
  }
  F est, var, se;
  acc.finalize(&est, &var, &se);
  out[0] = value; out[1] = est; out[2] = var; out[3] = se; out[4] = (F)acc.count;
}

template <class F>
int stde_sparse(const Tape<F>& t, int K, const F* x, const uint32_t* off, const uint32_t* vars, const uint32_t* slots,
                const F* coefs, const uint32_t* kout, const F* pref, const F* sign, F z, const uint64_t* idx,
                uint64_t nidx, F* out) {
  switch (K) {
#define ORC_SS(KK) \
  case KK: stde_sparse_k<F, KK>(t, x, off, vars, slots, coefs, kout, pref, sign, z, idx, nidx, out); return 0;
    ORC_SS(1) ORC_SS(2) ORC_SS(3) ORC_SS(4) ORC_SS(5) ORC_SS(6) ORC_SS(7) ORC_SS(8) ORC_SS(9) ORC_SS(10) ORC_SS(11)
#undef ORC_SS
    default: return -1;
  }
}

}  // namespace orc

// ───────────────────────── extern "C" surface ───────────────────────────────
extern "C" {

struct orc_tape_desc {
  const uint32_t* opcodes;
  const uint32_t* arg0;
  const uint32_t* arg1;
  const void* values;
  uint32_t num_variables;
  uint32_t num_inputs;
  uint32_t output_index;
  const uint32_t* output_indices;  // all_output_indices()
  uint32_t num_outputs;
};

}  // extern "C"

namespace {
template <class F> orc::Tape<F> mk(const orc_tape_desc* d) {
  return orc::Tape<F>{d->opcodes, d->arg0, d->arg1, (const F*)d->values, d->num_variables, d->num_inputs,
                      d->output_index, d->output_indices, d->num_outputs};
}

template <class F> void forward_batch(const orc_tape_desc* d, const F* X, uint64_t B, F* out, int nth) {
  auto t = mk<F>(d);
  orc::parallel_for(B, nth, [&](uint64_t lo, uint64_t hi, int) {
    std::vector<F> v;
    for (uint64_t b = lo; b < hi; ++b) {
      orc::forward_into<F>(t, X + b * t.ni, v);
      for (uint32_t j = 0; j < t.nout; ++j) out[b * t.nout + j] = v[t.outs[j]];
    }
  });
}

template <class F> void gradient_batch(const orc_tape_desc* d, const F* X, uint64_t B, F* out, F* grad, int nth) {
  auto t = mk<F>(d);
  orc::parallel_for(B, nth, [&](uint64_t lo, uint64_t hi, int) {
    std::vector<F> v, adj;
    for (uint64_t b = lo; b < hi; ++b) {
      orc::forward_into<F>(t, X + b * t.ni, v);
      for (uint32_t j = 0; j < t.nout; ++j) if (out) out[b * t.nout + j] = v[t.outs[j]];
      orc::reverse_from<F>(t, v, adj, t.out_idx);
      for (uint32_t i = 0; i < t.ni; ++i) grad[b * t.ni + i] = adj[i];
    }
  });
}

template <class F> void hvp_batch(const orc_tape_desc* d, const F* X, const F* V, uint64_t B, int x_per_point,
                                  F* grad, F* hv, int nth) {
  auto t = mk<F>(d);
  orc::parallel_for(B, nth, [&](uint64_t lo, uint64_t hi, int) {
    std::vector<orc::Dual<F>> din, dv, adj;
    for (uint64_t b = lo; b < hi; ++b)
      orc::hvp_point<F>(t, X + (x_per_point ? b * t.ni : 0), V + b * t.ni, grad + b * t.ni, hv + b * t.ni, din, dv, adj);
  });
}

template <class F> void jvp_batch(const orc_tape_desc* d, const F* X, const F* V, uint64_t B, F* val, F* tan, int nth) {
  auto t = mk<F>(d);
  orc::parallel_for(B, nth, [&](uint64_t lo, uint64_t hi, int) {
    std::vector<orc::Dual<F>> din(t.ni), dv;
    for (uint64_t b = lo; b < hi; ++b) {
      for (uint32_t i = 0; i < t.ni; ++i) din[i] = {X[b * t.ni + i], V[b * t.ni + i]};
      orc::forward_tangent<F, orc::Dual<F>>(t, din.data(), dv);
      for (uint32_t j = 0; j < t.nout; ++j) {
        if (val) val[b * t.nout + j] = dv[t.outs[j]].re;
        tan[b * t.nout + j] = dv[t.outs[j]].eps;
      }
    }
  });
}

template <class F> void hessian_full(const orc_tape_desc* d, const F* x, F* value, F* grad, F* hess) {
  // src/bytecode_tape/tangent.rs:334-376
  auto t = mk<F>(d);
  uint32_t n = t.ni;
  std::vector<orc::Dual<F>> din(n), dv, adj;
  for (uint32_t j = 0; j < n; ++j) {
    for (uint32_t i = 0; i < n; ++i) din[i] = {x[i], i == j ? F(1) : F(0)};
    orc::forward_tangent<F, orc::Dual<F>>(t, din.data(), dv);
    orc::reverse_tangent<F, orc::Dual<F>>(t, dv, adj);
    if (j == 0) {
      *value = dv[t.out_idx].re;
      for (uint32_t i = 0; i < n; ++i) grad[i] = adj[i].re;
    }
    for (uint32_t i = 0; i < n; ++i) hess[(uint64_t)i * n + j] = adj[i].eps;
  }
}

template <class F> void laplacian_stats_batch(const orc_tape_desc* d, const F* X, const F* dirs, uint64_t B, uint32_t S,
                                              int dirs_per_point, F* out, int nth) {
  auto t = mk<F>(d);
  orc::parallel_for(B, nth, [&](uint64_t lo, uint64_t hi, int) {
    std::vector<orc::Tay<F, 3>> in, buf;
    for (uint64_t b = lo; b < hi; ++b)
      orc::laplacian_stats_point<F>(t, X + b * t.ni, dirs + (dirs_per_point ? b * (uint64_t)S * t.ni : 0), S,
                                    out + b * 5, in, buf);
  });
}

// laplacian (plain mean, src/stde/laplacian.rs:28-41)
template <class F> void laplacian_plain(const orc_tape_desc* d, const F* x, const F* dirs, uint32_t S, F* value, F* lap) {
  auto t = mk<F>(d);
  std::vector<orc::Tay<F, 3>> in, buf;
  std::vector<F> tmp(t.nout * 3);
  F sum = F(0);
  F two = F(2);
  for (uint32_t s = 0; s < S; ++s) {
    orc::taylor_point<F, 3>(t, x, dirs + (uint64_t)s * t.ni, tmp.data(), in, buf);
    *value = buf[t.out_idx].c[0];
    sum = sum + two * buf[t.out_idx].c[2];
  }
  *lap = sum / (F)S;
}

// hessian_diagonal (src/stde/laplacian.rs:137-171)
template <class F> void hessian_diagonal(const orc_tape_desc* d, const F* x, F* value, F* diag) {
  auto t = mk<F>(d);
  std::vector<orc::Tay<F, 3>> in, buf;
  std::vector<F> e(t.ni, F(0)), tmp(t.nout * 3);
  for (uint32_t j = 0; j < t.ni; ++j) {
    e[j] = F(1);
    orc::taylor_point<F, 3>(t, x, e.data(), tmp.data(), in, buf);
    *value = buf[t.out_idx].c[0];
    diag[j] = F(2) * buf[t.out_idx].c[2];
    e[j] = F(0);
  }
}

// laplacian_with_control (src/stde/laplacian.rs:90-129)
template <class F> void laplacian_with_control(const orc_tape_desc* d, const F* x, const F* dirs, uint32_t S,
                                               const F* control, F* out) {
  auto t = mk<F>(d);
  std::vector<orc::Tay<F, 3>> in, buf;
  std::vector<F> tmp(t.nout * 3);
  F two = F(2);
  F trace = F(0);
  for (uint32_t j = 0; j < t.ni; ++j) trace = trace + control[j];
  orc::Welford<F> acc;
  F value = F(0);
  for (uint32_t s = 0; s < S; ++s) {
    const F* v = dirs + (uint64_t)s * t.ni;
    orc::taylor_point<F, 3>(t, x, v, tmp.data(), in, buf);
    value = buf[t.out_idx].c[0];
    F raw = two * buf[t.out_idx].c[2];
    F cv = F(0);
    for (uint32_t j = 0; j < t.ni; ++j) cv = cv + control[j] * v[j] * v[j];
    acc.update(raw - cv + trace);
  }
  F est, var, se;
  acc.finalize(&est, &var, &se);
  out[0] = value; out[1] = est; out[2] = var; out[3] = se; out[4] = (F)acc.count;
}

// estimate_weighted with the Laplacian estimator (src/stde/pipeline.rs:56-142)
template <class F> int estimate_weighted(const orc_tape_desc* d, const F* x, const F* dirs, uint32_t S, const F* w,
                                         F* out) {
  auto t = mk<F>(d);
  std::vector<orc::Tay<F, 3>> in, buf;
  std::vector<F> tmp(t.nout * 3);
  F value = F(0), w_sum = F(0), w_sum2 = F(0), mean = F(0), m2 = F(0);
  size_t skips = 0;
  for (uint32_t k = 0; k < S; ++k) {
    orc::taylor_point<F, 3>(t, x, dirs + (uint64_t)k * t.ni, tmp.data(), in, buf);
    value = buf[t.out_idx].c[0];
    F wk = w[k];
    if (!(wk >= F(0))) return -1;
    if (wk == F(0)) continue;
    F s = F(2) * buf[t.out_idx].c[2];
    if (!std::isfinite(s)) { skips++; continue; }
    w_sum = w_sum + wk;
    w_sum2 = w_sum2 + wk * wk;
    F delta = s - mean;
    mean = mean + (wk / w_sum) * delta;
    F delta2 = s - mean;
    m2 = m2 + wk * delta * delta2;
  }
  F denom = (w_sum > F(0)) ? w_sum - w_sum2 / w_sum : F(0);
  F var = F(0), se = F(0);
  if (S > 1 && denom > F(0)) {
    var = std::fmax(m2 / denom, F(0));
    F n_eff = w_sum * w_sum / w_sum2;
    se = std::sqrt(var / n_eff);
  }
  out[0] = value;
  out[1] = (w_sum > F(0) || skips == 0) ? mean : orc::s_nan<F>();
  out[2] = var; out[3] = se; out[4] = (F)(S - skips);
  return 0;
}

// diagonal_kth_order_stochastic (src/stde/higher_order.rs:173-227)
template <class F, int ORDER> void dks(const orc::Tape<F>& t, const F* x, const uint64_t* idx, uint64_t nidx, F* out) {
  F kf = F(1);
  for (int i = 2; i <= ORDER - 1; ++i) kf = kf * F(i);
  F nf = (F)t.ni;
  std::vector<orc::Tay<F, ORDER>> in(t.ni), buf;
  orc::Welford<F> acc;
  F value = F(0);
  for (uint64_t s = 0; s < nidx; ++s) {
    uint64_t j = idx[s];
    for (uint32_t i = 0; i < t.ni; ++i) {
      for (int k = 0; k < ORDER; ++k) in[i].c[k] = F(0);
      in[i].c[0] = x[i];
    }
    in[j].c[1] = F(1);
    orc::forward_tangent<F, orc::Tay<F, ORDER>>(t, in.data(), buf);
    value = buf[t.out_idx].c[0];
    acc.update(kf * buf[t.out_idx].c[ORDER - 1]);
  }
  F mean, var, se;
  acc.finalize(&mean, &var, &se);
  out[0] = value; out[1] = mean * nf; out[2] = var * nf * nf; out[3] = se * nf; out[4] = (F)acc.count;
}
}  // namespace

#define ORC_EXPORT extern "C" __attribute__((visibility("default")))

#define ORC_DEFINE(SUF, F)                                                                                          \
  ORC_EXPORT void orc_forward_##SUF(const orc_tape_desc* d, const F* X, uint64_t B, F* out, int nth) {              \
    forward_batch<F>(d, X, B, out, nth);                                                                            \
  }                                                                                                                 \
  ORC_EXPORT void orc_gradient_##SUF(const orc_tape_desc* d, const F* X, uint64_t B, F* out, F* grad, int nth) {    \
    gradient_batch<F>(d, X, B, out, grad, nth);                                                                     \
  }                                                                                                                 \
  ORC_EXPORT void orc_hvp_##SUF(const orc_tape_desc* d, const F* X, const F* V, uint64_t B, int x_per_point,       \
                                F* grad, F* hv, int nth) {                                                          \
    hvp_batch<F>(d, X, V, B, x_per_point, grad, hv, nth);                                                           \
  }                                                                                                                 \
  ORC_EXPORT void orc_jvp_##SUF(const orc_tape_desc* d, const F* X, const F* V, uint64_t B, F* val, F* tan,        \
                                int nth) {                                                                          \
    jvp_batch<F>(d, X, V, B, val, tan, nth);                                                                        \
  }                                                                                                                 \
  ORC_EXPORT int orc_taylor_##SUF(const orc_tape_desc* d, int K, const F* P, const F* S, uint64_t B, F* coeffs,     \
                                  int nth) {                                                                        \
    auto t = mk<F>(d);                                                                                              \
    return orc::taylor_batch<F>(t, K, P, S, B, coeffs, nth);                                                        \
  }                                                                                                                 \
  ORC_EXPORT int orc_stde_sparse_##SUF(const orc_tape_desc* d, int K, const F* x, const uint32_t* off,             \
                                       const uint32_t* vars, const uint32_t* slots, const F* coefs,                \
                                       const uint32_t* kout, const F* pref, const F* sign, F z,                    \
                                       const uint64_t* idx, uint64_t nidx, F* out) {                               \
    auto t = mk<F>(d);                                                                                              \
    return orc::stde_sparse<F>(t, K, x, off, vars, slots, coefs, kout, pref, sign, z, idx, nidx, out);              \
  }                                                                                                                 \
  ORC_EXPORT void orc_hessian_##SUF(const orc_tape_desc* d, const F* x, F* value, F* grad, F* hess) {              \
    hessian_full<F>(d, x, value, grad, hess);                                                                       \
  }                                                                                                                 \
  ORC_EXPORT void orc_laplacian_stats_batch_##SUF(const orc_tape_desc* d, const F* X, const F* dirs, uint64_t B,   \
                                                  uint32_t S, int dirs_per_point, F* out, int nth) {                \
    laplacian_stats_batch<F>(d, X, dirs, B, S, dirs_per_point, out, nth);                                           \
  }                                                                                                                 \
  ORC_EXPORT void orc_laplacian_##SUF(const orc_tape_desc* d, const F* x, const F* dirs, uint32_t S, F* value,     \
                                      F* lap) {                                                                     \
    laplacian_plain<F>(d, x, dirs, S, value, lap);                                                                  \
  }                                                                                                                 \
  ORC_EXPORT void orc_hessian_diagonal_##SUF(const orc_tape_desc* d, const F* x, F* value, F* diag) {              \
    hessian_diagonal<F>(d, x, value, diag);                                                                         \
  }                                                                                                                 \
  ORC_EXPORT void orc_laplacian_with_control_##SUF(const orc_tape_desc* d, const F* x, const F* dirs, uint32_t S,  \
                                                   const F* control, F* out) {                                      \
    laplacian_with_control<F>(d, x, dirs, S, control, out);                                                         \
  }                                                                                                                 \
  ORC_EXPORT int orc_estimate_weighted_##SUF(const orc_tape_desc* d, const F* x, const F* dirs, uint32_t S,        \
                                             const F* w, F* out) {                                                  \
    return estimate_weighted<F>(d, x, dirs, S, w, out);                                                             \
  }                                                                                                                 \
  ORC_EXPORT int orc_diagonal_kth_order_stochastic_##SUF(const orc_tape_desc* d, const F* x, uint32_t k,            \
                                                         const uint64_t* idx, uint64_t nidx, F* out) {              \
    auto t = mk<F>(d);                                                                                              \
    switch (k) {                                                                                                    \
      case 2: dks<F, 3>(t, x, idx, nidx, out); return 0;                                                            \
      case 3: dks<F, 4>(t, x, idx, nidx, out); return 0;                                                            \
      case 4: dks<F, 5>(t, x, idx, nidx, out); return 0;                                                            \
      case 5: dks<F, 6>(t, x, idx, nidx, out); return 0;                                                            \
      case 6: dks<F, 7>(t, x, idx, nidx, out); return 0;                                                            \
      case 7: dks<F, 8>(t, x, idx, nidx, out); return 0;                                                            \
      case 8: dks<F, 9>(t, x, idx, nidx, out); return 0;                                                            \
      default: return -1;                                                                                           \
    }                                                                                                               \
  }

ORC_DEFINE(f64, double)
ORC_DEFINE(f32, float)

ORC_EXPORT int orc_hardware_threads() { return (int)std::thread::hardware_concurrency(); }
