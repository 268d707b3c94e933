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
#include <cstring>

#if defined(__CUDACC__)
#define CLEO_MATH_HD __host__ __device__ __forceinline__
#define CLEO_MATH_SLOW static __host__ __device__ __noinline__  // the rarely taken accurate phase
#else
#define CLEO_MATH_HD static inline
#define CLEO_MATH_SLOW static
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
// a + b with one two-sum: absolute error below 2^-104 (|a| + |b|), all the first phase needs
// (its bound is 2^-72 relative, and none of its sums cancels more than a small factor except the
// reduction a - n ln2/512 of fast_exp, where the absolute error is what counts)
CLEO_MATH_HD dd dd_add_fast(dd a, dd b) {
  const dd s = two_sum(a.hi, b.hi);
  return fast_two_sum(s.hi, s.lo + (a.lo + b.lo));
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

// exp(x), rounded once from a double-double evaluation (the second, accurate phase)
CLEO_MATH_SLOW double dexp_dd(double x) {
  if (!(x > -707.0 && x < 707.0)) return std::exp(x);
  return round_dd(dd_exp(dd{x, 0.0}));
}

// pow(x, y) for x > 0 normal and y not special, rounded once from a double-double evaluation
CLEO_MATH_SLOW double dpow_dd(double x, double y) {
  const dd z = dd_mul_d(dd_log(x), y);
  if (!(z.hi > -707.0 && z.hi < 707.0)) return std::pow(x, y);
  return round_dd(dd_exp(z));
}

// ---- first phase (Ziv's strategy) ----
// A cheaper evaluation with relative error below 2^-72 (analysis beside each step), accepted
// only when that bound cannot move the value across a rounding midpoint; otherwise the accurate
// phase above decides. Either way the result is the double nearest the true value, so the two
// phases together return what the accurate phase alone returns.
constexpr double FAST_ERR = 0x1p-67;  // bound used by the rounding test (about 32x the estimate)

CLEO_MATH_HD uint64_t dbits(double x) {
#if defined(__CUDA_ARCH__)
  return (uint64_t)__double_as_longlong(x);
#else
  uint64_t b;
  std::memcpy(&b, &x, sizeof b);
  return b;
#endif
}
CLEO_MATH_HD double bitsd(uint64_t b) {
#if defined(__CUDA_ARCH__)
  return __longlong_as_double((long long)b);
#else
  double x;
  std::memcpy(&x, &b, sizeof x);
  return x;
#endif
}

// 2^k for -1022 <= k <= 1023, exactly: multiplying by it is ldexp(x, k) wherever the product is
// a normal double (both are the one correctly rounded value of x 2^k)
CLEO_MATH_HD double pow2i(int k) { return bitsd((uint64_t)(k + 1023) << 52); }

// ln x for positive normal finite x, relative error below 2^-70 (absolute below 2^-79 plus
// 2^-100 |exponent|): x = 2^e m, m in [sqrt(1/2), sqrt(2)); rc ~ 1/c for the nearest centre
// c = i/512, r = m rc - 1 exactly (|r| < 2^-9.4); ln m = -ln(rc) + log1p(r), the series
// truncated after r^8/8 (remainder below 2^-76 |r|).
CLEO_MATH_HD dd fast_log(double x) {
#if defined(__CUDA_ARCH__)
  using namespace cleo_dd_dev;
#else
  using namespace cleo_dd_host;
#endif
  // x = m 2^e, m in [0.5, 1) (frexp's split, read off the bits of the normal x)
  const uint64_t xb = dbits(x);
  int e = (int)((xb >> 52) & 0x7FF) - 1022;
  double m = bitsd((xb & 0x000FFFFFFFFFFFFFull) | 0x3FE0000000000000ull);
  if (m < 0.70710678118654752440) {
    m *= 2.0;
    e -= 1;
  }
  const int i = (int)std::rint(m * 512.0);  // 362 .. 724
  const double* t = cleo_fast_log_tab[i - 362];
  const dd p = two_prod(m, t[0]);
  const dd r = two_sum(p.hi - 1.0, p.lo);  // p.hi - 1 is exact (Sterbenz)
  const double rh = r.hi, rl = r.lo;
  const dd sq = two_prod(rh, rh);
  const dd s = two_sum(rh, -0.5 * sq.hi);
  // Horner's scheme with fused multiply-adds (each step rounds once, so no less accurately than
  // the separate product and sum)
  double q = dd_fma(rh, -0.125, CLEO_DD_SEVENTH_HI);
  q = dd_fma(rh, q, -CLEO_DD_INV6_HI);
  q = dd_fma(rh, q, CLEO_DD_FIFTH_HI);
  q = dd_fma(rh, q, -0.25);
  q = dd_fma(rh, q, CLEO_DD_THIRD_HI);
  // r^2/2 = rh^2/2 + rh rl + rl^2/2 (the last below 2^-115 |r|); r^3 q rounded: below 2^-72 |r|
  const double low = rl - 0.5 * sq.lo - rh * rl + (rh * sq.hi) * q;
  const dd l1p = fast_two_sum(s.hi, s.lo + low);
  dd eln2 = two_prod((double)e, CLEO_DD_LN2_HI);
  eln2.lo += (double)e * CLEO_DD_LN2_LO;
  return dd_add_fast(eln2, dd_add_fast(dd{t[1], t[2]}, l1p));
}

// exp of a double-double with |a.hi| < 600, relative error below 2^-72: a = n ln2/512 + r,
// |r| <= ln2/1024 (2^-10.5), exp(r) - 1 = r + r^2/2 + ... + r^5/120 (remainder below 2^-72).
CLEO_MATH_HD dd fast_exp(dd a) {
#if defined(__CUDA_ARCH__)
  using namespace cleo_dd_dev;
#else
  using namespace cleo_dd_host;
#endif
  const double nf = std::rint(a.hi * (512.0 * CLEO_DD_INV_LN2));
  const int n = (int)nf;
  const int j = n & 511;
  const int k = (n - j) / 512;
  const dd p = two_prod(nf, CLEO_DD_LN2_HI * 0x1p-9);
  dd r = dd_add_fast(a, dd{-p.hi, -p.lo});
  r = dd_add_d(r, -nf * (CLEO_DD_LN2_LO * 0x1p-9));
  const double rh = r.hi, rl = r.lo;
  double c = dd_fma(rh, CLEO_DD_INV120_HI, CLEO_DD_INV24_HI);  // Horner with fused steps
  c = dd_fma(rh, c, CLEO_DD_INV6_HI);
  c = dd_fma(rh, c, 0.5);
  const double poly = rh * rh * c;
  const dd em1 = fast_two_sum(rh, rl + rh * rl + poly);
  const dd tj{cleo_fast_exp2_tab[j][0], cleo_fast_exp2_tab[j][1]};
  dd v = dd_add_fast(tj, dd_mul(tj, em1));
  // |k| <= 866 and v.hi near [1, 2]: both products are normal, so exact (ldexp's values)
  const double sk = pow2i(k);
  v.hi *= sk;
  v.lo *= sk;
  return v;
}

// true when every value within FAST_ERR |v| of v.hi + v.lo (v positive, normalised, normal)
// rounds to v.hi
CLEO_MATH_HD bool fast_round_ok(dd v) {
  const uint64_t b = dbits(v.hi);
  const uint64_t ex = (b >> 52) & 0x7FF;
  if (ex <= 53 || ex >= 0x7FF) return false;
  const double u = bitsd((ex - 52) << 52);  // spacing of the doubles above v.hi
  const double d_up = 0.5 * u;
  const double d_down = ((b & 0xFFFFFFFFFFFFFull) == 0) ? 0.25 * u : 0.5 * u;
  const double err = FAST_ERR * v.hi;
  return (v.lo + err < d_up) && (v.lo - err > -d_down);
}

// exp(x), rounded once (first phase, then the double-double phase when needed)
CLEO_MATH_HD double dexp(double x) {
  if (x > -600.0 && x < 600.0) {
    const dd v = fast_exp(dd{x, 0.0});
    if (fast_round_ok(v)) return v.hi;
  }
  return dexp_dd(x);
}

// First phase for the exponents 1/6, 1/3 and 2/3 (as doubles: k/6 - eps with eps = 2^-57/3,
// 2^-56/3, 2^-55/3), for 2^-600 <= x <= 2^600, relative error below 2^-76:
//   x = 2^(3q) m with m in [1, 8); x^y = 2^(qk/2) m^(k/6) exp(-eps L), L = ln x, |eps L| <
//   2^-45.9, so exp(-eps L) = 1 - w + w^2/2 with w = eps L (remainder below 2^-136). w's
//   absolute error is eps times L's, so L from the exponent and a single-precision log2 of the
//   leading significand (absolute error below 2^-22) puts at most 2^-77 into the result;
//   m^(1/3): the inverse cube root y from a single-precision start (relative 2^-22) by two Newton
//   steps y (1 + (1 - m y^3) / 3) (error 2 e^2 each, so to the double's precision), c0 = m y^2
//   (within 2^-50), then one Newton step for the cube root with the exact residual: c0^2 = t + e1
//   and t c0 = u + ul exactly (fused multiply-adds), m - u exact (Sterbenz), the residual to
//   2^-102 m, the step res y^2 / 3 to 2^-99 c, the step's own truncation below 2^-99;
//   m^(2/3) the double-double square of it, m^(1/6) its double-double square root (one step from
//   the correctly rounded sqrt of the high part, whose residual fma is exact).
constexpr double Y16 = 1.0 / 6.0, Y13 = 1.0 / 3.0, Y23 = 2.0 / 3.0;
CLEO_MATH_HD dd fast_sixth_pow(double x, double yexp) {
  const uint64_t xb = dbits(x);
  const int e = (int)((xb >> 52) & 0x7FF) - 1023;
  const int q = e >= 0 ? e / 3 : -((2 - e) / 3);  // floor(e / 3)
  const double m = bitsd((xb & 0x000FFFFFFFFFFFFFull) | ((uint64_t)(1023 + e - 3 * q) << 52));
#if defined(__CUDA_ARCH__)
  double y = (double)rcbrtf((float)m);
#else
  double y = (double)(1.0f / std::cbrt((float)m));
#endif
  y = y + y * (1.0 - m * y * y * y) * (1.0 / 3.0);
  y = y + y * (1.0 - m * y * y * y) * (1.0 / 3.0);
  const double y2 = y * y;
  const double c0 = m * y2;
  const double t = c0 * c0;
  const double e1 = dd_fma(c0, c0, -t);
  const double u = t * c0;
  const double ul = dd_fma(t, c0, -u);
  const double res = ((m - u) - ul) - e1 * c0;
  dd c = fast_two_sum(c0, res * y2 * (1.0 / 3.0));
  double eps;
  int shift;  // x^(k/6) = 2^shift m^(k/6) with shift = q k / 2, q even where k = 1
  if (yexp == Y13) {
    eps = 0x1.5555555555555p-56;
    shift = q;
  } else if (yexp == Y23) {
    eps = 0x1.5555555555555p-55;
    shift = 2 * q;
    const dd s2 = two_prod(c.hi, c.hi);
    c = fast_two_sum(s2.hi, s2.lo + 2.0 * c.hi * c.lo);
  } else {  // 1/6: sqrt(2^q m^(1/3)), 2^q's odd part moved under the root
    eps = 0x1.5555555555555p-57;
    if (q & 1) {
      c.hi *= 2.0;
      c.lo *= 2.0;
    }
    shift = (q - (q & 1)) / 2;
    const double s0 = std::sqrt(c.hi);
    const double r = dd_fma(-s0, s0, c.hi) + c.lo;
    c = fast_two_sum(s0, r / (2.0 * s0));
  }
  const float mf = (float)bitsd((xb & 0x000FFFFFFFFFFFFFull) | 0x3FF0000000000000ull);
  const double w = eps * (((double)e + (double)std::log2(mf)) * 0.69314718055994530942);
  const double sk = pow2i(shift);
  return fast_two_sum(c.hi * sk, (c.lo - c.hi * (w - 0.5 * w * w)) * sk);
}

// pow(x, y) for the exponents CLEO uses, rounded once
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
  if ((y == Y13 || y == Y23 || y == Y16) && x >= 0x1p-600 && x <= 0x1p600) {
    const dd v = fast_sixth_pow(x, y);
    if (fast_round_ok(v)) return v.hi;
    return dpow_dd(x, y);
  }
  const dd z = dd_mul_d(fast_log(x), y);
  if (z.hi > -600.0 && z.hi < 600.0) {
    const dd v = fast_exp(z);
    if (fast_round_ok(v)) return v.hi;
  }
  return dpow_dd(x, y);
}

// dpow(x, y1) and dpow(x, y2) with one logarithm (same results as two dpow calls; for general
// exponents, i.e. not 0.5, 1, 2 or 3)
CLEO_MATH_HD void dpow2(double x, double y1, double y2, double& p1, double& p2) {
  if (!(x > 2.2250738585072014e-308) || !(x < 1.7976931348623157e308)) {
    p1 = dpow(x, y1);
    p2 = dpow(x, y2);
    return;
  }
  const dd lx = fast_log(x);
  const double ys[2] = {y1, y2};
  double out[2];
  for (int q = 0; q < 2; ++q) {
    const dd z = dd_mul_d(lx, ys[q]);
    out[q] = 0.0;
    bool done = false;
    if (z.hi > -600.0 && z.hi < 600.0) {
      const dd v = fast_exp(z);
      if (fast_round_ok(v)) {
        out[q] = v.hi;
        done = true;
      }
    }
    if (!done) out[q] = dpow_dd(x, ys[q]);
  }
  p1 = out[0];
  p2 = out[1];
}

}  // namespace cleo
