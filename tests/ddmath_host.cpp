// Host build of cleo_b200/csrc/ddmath.h for tests/test_ddmath.py.
#include <cstdint>

#include "../cleo_b200/csrc/ddmath.h"
extern "C" double dd_pow(double x, double y) { return cleo::dpow(x, y); }
extern "C" double dd_exp(double x) { return cleo::dexp(x); }
extern "C" double dd_pow_accurate(double x, double y) {
  if (y == 2.0 || y == 0.5 || y == 1.0 || y == 3.0) return cleo::dpow(x, y);
  return cleo::dpow_dd(x, y);
}
extern "C" double dd_exp_accurate(double x) { return cleo::dexp_dd(x); }

namespace {
uint64_t mix(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
double unit(uint64_t u) { return (double)(u >> 11) * 0x1p-53; }
}  // namespace

// n random pow arguments: x = 2^(uniform [lx0, lx1)) with random mantissa bits, y drawn from
// ys[0..nys) when nys > 0, else uniform in [y0, y1). Counts results of dpow that differ from the
// accurate phase alone, and how often the first phase deferred to it.
extern "C" void dd_compare_pow(uint64_t seed, uint64_t n, double lx0, double lx1, const double* ys,
                               int nys, double y0, double y1, uint64_t* mismatches,
                               uint64_t* deferred, double* bad) {
  uint64_t mm = 0, df = 0;
  for (uint64_t i = 0; i < n; ++i) {
    const double x = std::exp2(lx0 + (lx1 - lx0) * unit(mix(seed ^ (4 * i))));
    const double y =
        nys > 0 ? ys[mix(seed ^ (4 * i + 1)) % (uint64_t)nys] : y0 + (y1 - y0) * unit(mix(seed ^ (4 * i + 2)));
    const double a = cleo::dpow(x, y);
    const double b = dd_pow_accurate(x, y);
    if (cleo::dbits(a) != cleo::dbits(b)) {
      if (mm == 0) {
        bad[0] = x;
        bad[1] = y;
      }
      ++mm;
    }
    // the first phase dpow takes for (x, y)
    if ((y == cleo::Y13 || y == cleo::Y23 || y == cleo::Y16) && x >= 0x1p-600 && x <= 0x1p600) {
      if (!cleo::fast_round_ok(cleo::fast_sixth_pow(x, y))) ++df;
      continue;
    }
    const cleo::dd z = cleo::dd_mul_d(cleo::fast_log(x), y);
    if (!(z.hi > -600.0 && z.hi < 600.0) || !cleo::fast_round_ok(cleo::fast_exp(z))) ++df;
  }
  *mismatches = mm;
  *deferred = df;
}

extern "C" void dd_compare_exp(uint64_t seed, uint64_t n, double x0, double x1,
                               uint64_t* mismatches, uint64_t* deferred, double* bad) {
  uint64_t mm = 0, df = 0;
  for (uint64_t i = 0; i < n; ++i) {
    const double x = x0 + (x1 - x0) * unit(mix(seed ^ i));
    const double a = cleo::dexp(x), b = cleo::dexp_dd(x);
    if (cleo::dbits(a) != cleo::dbits(b)) {
      if (mm == 0) bad[0] = x;
      ++mm;
    }
    if (!cleo::fast_round_ok(cleo::fast_exp(cleo::dd{x, 0.0}))) ++df;
  }
  *mismatches = mm;
  *deferred = df;
}

// dpow2 against two dpow calls
extern "C" uint64_t dd_compare_pow2(uint64_t seed, uint64_t n, double y1, double y2) {
  uint64_t mm = 0;
  for (uint64_t i = 0; i < n; ++i) {
    const double x = std::exp2(-40.0 + 50.0 * unit(mix(seed ^ i)));
    double a, b;
    cleo::dpow2(x, y1, y2, a, b);
    if (cleo::dbits(a) != cleo::dbits(cleo::dpow(x, y1)) ||
        cleo::dbits(b) != cleo::dbits(cleo::dpow(x, y2)))
      ++mm;
  }
  return mm;
}

// largest relative difference between the first phase's double-double pow and the accurate
// phase's, over n random arguments (x = 2^U[lx0, lx1), y = U[y0, y1))
extern "C" double dd_fast_pow_maxerr(uint64_t seed, uint64_t n, double lx0, double lx1, double y0,
                                     double y1) {
  double worst = 0.0;
  for (uint64_t i = 0; i < n; ++i) {
    const double x = std::exp2(lx0 + (lx1 - lx0) * unit(mix(seed ^ (2 * i))));
    const double y = y0 + (y1 - y0) * unit(mix(seed ^ (2 * i + 1)));
    const cleo::dd z = cleo::dd_mul_d(cleo::fast_log(x), y);
    if (!(z.hi > -600.0 && z.hi < 600.0)) continue;
    const cleo::dd f = cleo::fast_exp(z);
    const cleo::dd a = cleo::dd_exp(cleo::dd_mul_d(cleo::dd_log(x), y));
    const cleo::dd d = cleo::dd_add(f, cleo::dd{-a.hi, -a.lo});
    const double rel = std::fabs(d.hi / a.hi);
    if (rel > worst) worst = rel;
  }
  return worst;
}

// largest relative difference between the first phase for the exponents 1/6, 1/3, 2/3 and the
// accurate double-double pow, over n random x = 2^U[lx0, lx1) (within the phase's range)
extern "C" double dd_fast_sixth_maxerr(uint64_t seed, uint64_t n, double lx0, double lx1) {
  const double ys[3] = {cleo::Y16, cleo::Y13, cleo::Y23};
  double worst = 0.0;
  for (uint64_t i = 0; i < n; ++i) {
    const double x = std::exp2(lx0 + (lx1 - lx0) * unit(mix(seed ^ (2 * i))));
    const double y = ys[mix(seed ^ (2 * i + 1)) % 3];
    const cleo::dd f = cleo::fast_sixth_pow(x, y);
    const cleo::dd a = cleo::dd_exp(cleo::dd_mul_d(cleo::dd_log(x), y));
    const cleo::dd d = cleo::dd_add(f, cleo::dd{-a.hi, -a.lo});
    const double rel = std::fabs(d.hi / a.hi);
    if (rel > worst) worst = rel;
  }
  return worst;
}

// out[i] = dpow(x[i], y[i]), or dexp(x[i]) when y is null (the host side of the device check)
extern "C" void dd_eval_array(const double* x, const double* y, double* out, uint64_t n) {
  for (uint64_t i = 0; i < n; ++i) out[i] = y ? cleo::dpow(x[i], y[i]) : cleo::dexp(x[i]);
}

// the ventilation factor (impliciteuler.cpp:131-145) with the correctly rounded powers, radius in
// CLEO's units (1e-6 m)
extern "C" void dd_vent_array(const double* radius, double* out, uint64_t n) {
  for (uint64_t i = 0; i < n; ++i) {
    double pa, pb;
    cleo::dpow2(radius[i] * 1e-6, 1.963, 0.702, pa, pb);
    const double a = 1.0 / (6.954e+7 * pa);
    const double b = 1.0 / (1.069e+3 * pb);
    out[i] = std::fmin(1.0 + 1.0 / (a + b), 20.0);
  }
}
