// dd.cuh -- double-double arithmetic for the magnetostatic tensor elements.
//
// A value is the unevaluated sum hi + lo of two doubles (|lo| <= ulp(hi)/2),
// about 106 significant bits.  The tensor's 64-corner sums
// (src/tensor_element.f90:78-100) subtract terms that grow like r^3 log r to
// leave a result of order 1/r^3: in FP64 an offset of r cells loses about
// (r / cell)^6 of the 2^-53 precision, so at a few hundred cells the far-field
// elements are rounding noise, and the demag field of a 1024 x 1024 grid
// differs from the exact convolution by ~1e-5 in relative L2.  Evaluating the
// same formula in double-double keeps those elements to ~1e-14 relative.
//
// Algorithms (published, written here from their descriptions): the
// error-free transformations two-sum (Knuth) and two-product by fused
// multiply-add; addition, multiplication, division by Newton correction and
// square root by one Newton step (Dekker 1971; Hida, Li and Bailey, "Algorithms
// for quad-double precision floating point arithmetic", 2001).  The logarithm
// reduces x = 2^k m (m in [1/sqrt 2, sqrt 2)), takes three square roots and
// sums the atanh series of s = (m^(1/8) - 1)/(m^(1/8) + 1); the arctangent
// reduces to |x| <= 1 (pi/2 - atan(1/x)), halves the angle three times
// (atan x = 2 atan(x / (1 + sqrt(1 + x^2)))) and sums the Taylor series.
// Host and device compile the same code (the host test checks it against
// quadruple precision).
#pragma once
#include <cmath>

#ifndef MRM_HD
#define MRM_HD __host__ __device__ __forceinline__
#endif

namespace mrm {

struct dd {
  double hi, lo;
};

MRM_HD dd dd_from(double a) { return dd{a, 0.0}; }

// s + e = a + b exactly
MRM_HD dd two_sum(double a, double b) {
  const double s = a + b;
  const double bb = s - a;
  return dd{s, (a - (s - bb)) + (b - bb)};
}
// s + e = a + b exactly, |a| >= |b|
MRM_HD dd quick_two_sum(double a, double b) {
  const double s = a + b;
  return dd{s, b - (s - a)};
}
// p + e = a * b exactly
MRM_HD dd two_prod(double a, double b) {
  const double p = a * b;
  return dd{p, fma(a, b, -p)};
}

MRM_HD dd dd_neg(dd a) { return dd{-a.hi, -a.lo}; }

MRM_HD dd dd_add(dd a, dd b) {
  dd s = two_sum(a.hi, b.hi);
  const dd t = two_sum(a.lo, b.lo);
  s.lo += t.hi;
  s = quick_two_sum(s.hi, s.lo);
  s.lo += t.lo;
  return quick_two_sum(s.hi, s.lo);
}
MRM_HD dd dd_sub(dd a, dd b) { return dd_add(a, dd_neg(b)); }
MRM_HD dd dd_add_d(dd a, double b) {
  dd s = two_sum(a.hi, b);
  s.lo += a.lo;
  return quick_two_sum(s.hi, s.lo);
}

MRM_HD dd dd_mul(dd a, dd b) {
  dd p = two_prod(a.hi, b.hi);
  p.lo += a.hi * b.lo + a.lo * b.hi;
  return quick_two_sum(p.hi, p.lo);
}
MRM_HD dd dd_mul_d(dd a, double b) {
  dd p = two_prod(a.hi, b);
  p.lo += a.lo * b;
  return quick_two_sum(p.hi, p.lo);
}
// multiplication by a power of two (exact)
MRM_HD dd dd_ldexp(dd a, int k) { return dd{ldexp(a.hi, k), ldexp(a.lo, k)}; }

MRM_HD dd dd_div(dd a, dd b) {
  const double q1 = a.hi / b.hi;
  dd r = dd_sub(a, dd_mul_d(b, q1));
  const double q2 = r.hi / b.hi;
  r = dd_sub(r, dd_mul_d(b, q2));
  const double q3 = r.hi / b.hi;
  return dd_add_d(quick_two_sum(q1, q2), q3);
}
// 1 / n for a small positive integer n
MRM_HD dd dd_recip_int(int n) {
  const double q = 1.0 / (double)n;
  const double r = fma(-q, (double)n, 1.0);  // exact residual
  return quick_two_sum(q, r / (double)n);
}

MRM_HD dd dd_sqrt(dd a) {
  if (!(a.hi > 0.0)) return dd{0.0, 0.0};
  const double x = 1.0 / sqrt(a.hi);
  const double ax = a.hi * x;
  // sqrt(a) ~ ax + (a - ax^2) x / 2
  const dd d = dd_sub(a, two_prod(ax, ax));
  return dd_add_d(dd{ax, 0.0}, d.hi * x * 0.5);
}

MRM_HD bool dd_lt(dd a, dd b) { return a.hi < b.hi || (a.hi == b.hi && a.lo < b.lo); }
MRM_HD dd dd_abs(dd a) { return (a.hi < 0.0 || (a.hi == 0.0 && a.lo < 0.0)) ? dd_neg(a) : a; }
MRM_HD dd dd_max_d(dd a, double b) { return dd_lt(a, dd_from(b)) ? dd_from(b) : a; }

// ln 2 and pi/2 to double-double precision
constexpr double kLn2Hi = 6.93147180559945286227e-01, kLn2Lo = 2.31904681384629955842e-17;
constexpr double kPi2Hi = 1.57079632679489655800e+00, kPi2Lo = 6.12323399573676603587e-17;

// natural logarithm of a > 0
MRM_HD dd dd_log(dd a) {
  int k = 0;
  const double f = frexp(a.hi, &k);  // a.hi = f 2^k, f in [0.5, 1)
  if (f < 0.70710678118654752440) --k;
  dd m = dd_ldexp(a, -k);  // in [1/sqrt 2, sqrt 2)
  m = dd_sqrt(dd_sqrt(dd_sqrt(m)));  // m^(1/8) in [0.957, 1.044]
  const dd s = dd_div(dd_add_d(m, -1.0), dd_add_d(m, 1.0));
  const dd s2 = dd_mul(s, s);  // <= 4.8e-4
  // atanh(s) = s sum_i s^(2i) / (2i + 1); 11 terms reach 1e-33
  dd p = dd_recip_int(21);
  for (int i = 9; i >= 0; --i) p = dd_add(dd_mul(p, s2), dd_recip_int(2 * i + 1));
  const dd lm = dd_ldexp(dd_mul(s, p), 4);  // 8 * 2 atanh(s)
  return dd_add(dd_mul_d(dd{kLn2Hi, kLn2Lo}, (double)k), lm);
}

// arctangent
MRM_HD dd dd_atan(dd a) {
  const bool neg = a.hi < 0.0;
  dd x = neg ? dd_neg(a) : a;
  const bool inv = x.hi > 1.0;
  if (inv) x = dd_div(dd_from(1.0), x);
  // three angle halvings: |x| <= tan(pi/32) ~ 0.0985
  for (int h = 0; h < 3; ++h) x = dd_div(x, dd_add_d(dd_sqrt(dd_add_d(dd_mul(x, x), 1.0)), 1.0));
  const dd q = dd_neg(dd_mul(x, x));  // -x^2, |q| <= 0.0097
  // atan(x) = x sum_i q^i / (2i + 1); 17 terms reach 1e-33
  dd p = dd_recip_int(33);
  for (int i = 15; i >= 0; --i) p = dd_add(dd_mul(p, q), dd_recip_int(2 * i + 1));
  dd r = dd_ldexp(dd_mul(x, p), 3);
  if (inv) r = dd_sub(dd{kPi2Hi, kPi2Lo}, r);
  return neg ? dd_neg(r) : r;
}

}  // namespace mrm
