// ddmath.h — pow and exp evaluated in double-double arithmetic and rounded once.
//
// CLEO evaluates its microphysics with the host libm (glibc), whose pow and exp return the
// correctly rounded result in all but very rare cases. Condensation near activation is
// ill-conditioned, so 1-2 ulp differences in pow/exp (the documented error of a GPU libm) grow to
// ~1e-10 relative in a few droplets. These functions remove that source of difference: the
// logarithm and exponential are computed to about 100 bits with Tang's table-driven argument
// reduction (P. T. P. Tang, ACM TOMS 15 (1989) 144-157 for exp; ACM TOMS 16 (1990) 378-400 for
// log), a Taylor series for exp(r), |r| <= ln2/128, and the series
// ln((1+t)/(1-t)) = 2 (t + t^3/3 + t^5/5 + ...), |t| <= 1/180, for the log, all in double-double
// arithmetic (Dekker's two-sum / two-product), followed by one rounding to double.
//
// The same code compiles for host and device, so the host build checks the device results bit
// for bit and the tests measure agreement with the host libm.
#pragma once

#include <cmath>
#include <cstdint>

#if defined(__CUDACC__)
#define CLEO_MATH_HD __host__ __device__ __forceinline__
#else
#define CLEO_MATH_HD static inline
#endif

// one copy of the tables for device code (global memory, read through the L1 cache: lanes index
// them divergently) and one for host code
#if defined(__CUDACC__)
#define CLEO_DD_TABLE __device__ static const
namespace cleo_dd_dev {
#include "dd_tables.h"
}
#undef CLEO_DD_TABLE
#endif
#define CLEO_DD_TABLE static const
namespace cleo_dd_host {
#include "dd_tables.h"
}
#undef CLEO_DD_TABLE

namespace cleo {

struct dd {
  double hi, lo;
};

CLEO_MATH_HD double dd_fma(double a, double b, double c) {
#if defined(__CUDA_ARCH__)
  return __fma_rn(a, b, c);
#else
  return std::fma(a, b, c);
#endif
}

CLEO_MATH_HD dd two_sum(double a, double b) {
  const double s = a + b;
  const double bb = s - a;
  const double e = (a - (s - bb)) + (b - bb);
  return {s, e};
}
CLEO_MATH_HD dd fast_two_sum(double a, double b) {  // |a| >= |b|
  const double s = a + b;
  const double e = b - (s - a);
  return {s, e};
}
CLEO_MATH_HD dd two_prod(double a, double b) {
  const double p = a * b;
  const double e = dd_fma(a, b, -p);
  return {p, e};
}
CLEO_MATH_HD dd dd_add(dd a, dd b) {
  dd s = two_sum(a.hi, b.hi);
  const dd t = two_sum(a.lo, b.lo);
  s.lo += t.hi;
  s = fast_two_sum(s.hi, s.lo);
  s.lo += t.lo;
  return fast_two_sum(s.hi, s.lo);
}
CLEO_MATH_HD dd dd_add_d(dd a, double b) {
  dd s = two_sum(a.hi, b);
  s.lo += a.lo;
  return fast_two_sum(s.hi, s.lo);
}
CLEO_MATH_HD dd dd_mul(dd a, dd b) {
  dd p = two_prod(a.hi, b.hi);
  p.lo += a.hi * b.lo + a.lo * b.hi;
  return fast_two_sum(p.hi, p.lo);
}
CLEO_MATH_HD dd dd_mul_d(dd a, double b) {
  dd p = two_prod(a.hi, b);
  p.lo += a.lo * b;
  return fast_two_sum(p.hi, p.lo);
}
CLEO_MATH_HD dd dd_div(dd a, dd b) {
  const double q1 = a.hi / b.hi;
  dd r = dd_add(a, dd_mul_d(b, -q1));
  const double q2 = r.hi / b.hi;
  r = dd_add(r, dd_mul_d(b, -q2));
  const double q3 = r.hi / b.hi;
  const dd q = fast_two_sum(q1, q2);
  return dd_add_d(q, q3);
}

// natural logarithm of a positive, finite, normal x as a double-double
CLEO_MATH_HD dd dd_log(double x) {
#if defined(__CUDA_ARCH__)
  using namespace cleo_dd_dev;
#else
  using namespace cleo_dd_host;
#endif
  int e = 0;
  double m = std::frexp(x, &e);  // x = m 2^e, m in [0.5, 1)
  if (m < 0.70710678118654752440) {
    m *= 2.0;
    e -= 1;
  }  // m in [sqrt(1/2), sqrt(2))
  const int k = (int)std::rint((m - 1.0) * 64.0);  // -19 .. 27
  const double c = 1.0 + (double)k * 0.015625;
  // ln(m/c) = 2 atanh(t), t = (m - c)/(m + c), |t| <= 1/180
  const dd t = dd_div(dd{m - c, 0.0}, two_sum(m, c));
  const dd t2 = dd_mul(t, t);
  const double u = t2.hi;
  const double tail = 1.0 / 9.0 + u * (1.0 / 11.0 + u * (1.0 / 13.0 + u * (1.0 / 15.0)));
  dd s = dd_add(dd{CLEO_DD_SEVENTH_HI, CLEO_DD_SEVENTH_LO}, dd_mul_d(t2, tail));
  s = dd_add(dd{CLEO_DD_FIFTH_HI, CLEO_DD_FIFTH_LO}, dd_mul(t2, s));
  s = dd_add(dd{CLEO_DD_THIRD_HI, CLEO_DD_THIRD_LO}, dd_mul(t2, s));
  s = dd_add_d(dd_mul(t2, s), 1.0);
  dd lnmc = dd_mul(t, s);
  lnmc.hi *= 2.0;
  lnmc.lo *= 2.0;
  const dd lnc{cleo_dd_log_tab[k + 20][0], cleo_dd_log_tab[k + 20][1]};
  const dd eln2 = dd_add_d(two_prod((double)e, CLEO_DD_LN2_HI), (double)e * CLEO_DD_LN2_LO);
  return dd_add(eln2, dd_add(lnc, lnmc));
}

// exp of a double-double a with |a.hi| < 708
CLEO_MATH_HD dd dd_exp(dd a) {
#if defined(__CUDA_ARCH__)
  using namespace cleo_dd_dev;
#else
  using namespace cleo_dd_host;
#endif
  const double nf = std::rint(a.hi * (64.0 * CLEO_DD_INV_LN2));
  const int n = (int)nf;
  const int j = ((n % 64) + 64 + 32) % 64 - 32;  // -32 .. 31, n = 64 k + j
  const int kk = (n - j) / 64;
  // r = a - n ln2/64 with ln2/64 = (LN2_HI + LN2_LO)/64 (exact scalings)
  const dd p = two_prod(nf, CLEO_DD_LN2_HI * 0.015625);
  dd r = dd_add(a, dd{-p.hi, -p.lo});
  r = dd_add_d(r, -nf * (CLEO_DD_LN2_LO * 0.015625));
  const double x = r.hi;
  const double tail =
      1.0 / 720.0 + x * (1.0 / 5040.0 + x * (1.0 / 40320.0 + x * (1.0 / 362880.0 + x * (1.0 / 3628800.0))));
  dd q = dd_add(dd{CLEO_DD_INV120_HI, CLEO_DD_INV120_LO}, dd_mul_d(r, tail));
  q = dd_add(dd{CLEO_DD_INV24_HI, CLEO_DD_INV24_LO}, dd_mul(r, q));
  q = dd_add(dd{CLEO_DD_INV6_HI, CLEO_DD_INV6_LO}, dd_mul(r, q));
  q = dd_add_d(dd_mul(r, q), 0.5);
  q = dd_add_d(dd_mul(r, q), 1.0);
  const dd em1 = dd_mul(r, q);  // exp(r) - 1
  const dd tj{cleo_dd_exp2_tab[j + 32][0], cleo_dd_exp2_tab[j + 32][1]};
  dd v = dd_add(tj, dd_mul(tj, em1));
  v.hi = std::ldexp(v.hi, kk);
  v.lo = std::ldexp(v.lo, kk);
  return v;
}

CLEO_MATH_HD double round_dd(dd v) {
  const dd s = fast_two_sum(v.hi, v.lo);
  return s.hi;
}

// exp(x), rounded once from a double-double evaluation
CLEO_MATH_HD double dexp(double x) {
  if (!(x > -707.0 && x < 707.0)) return std::exp(x);
  return round_dd(dd_exp(dd{x, 0.0}));
}

// pow(x, y) for the exponents CLEO uses, rounded once from a double-double evaluation
CLEO_MATH_HD double dpow(double x, double y) {
  if (y == 2.0) return x * x;
  if (y == 0.5 && x >= 0.0) return std::sqrt(x);
  if (!(x > 2.2250738585072014e-308) || !(x < 1.7976931348623157e308) || !(y == y) ||
      !(std::fabs(y) < 1e300))
    return std::pow(x, y);
  if (y == 1.0) return x;
  if (y == 3.0) {
    const dd x2 = two_prod(x, x);
    return round_dd(dd_mul_d(x2, x));
  }
  const dd z = dd_mul_d(dd_log(x), y);
  if (!(z.hi > -707.0 && z.hi < 707.0)) return std::pow(x, y);
  return round_dd(dd_exp(z));
}

}  // namespace cleo
