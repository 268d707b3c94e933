// physics.cuh — device implementations of CLEO's per-droplet and per-pair microphysics.
//
// Each function follows the reference function named beside it with the same floating-point
// association (compiled with -fmad=false, so no contraction), so results match the reference up
// to the difference between CUDA's and the host libm's pow/exp. Abort sites of the reference
// record a status in the device error word instead of trapping.
#pragma once

#include <cstdint>

#include "../../include/cleo_b200.h"
#include "../../include/cleo_b200_rng.h"
#include "ddmath.h"

namespace cleo {

// ---- constants: libs/cleoconstants.hpp:32-118 ----
constexpr double PI = 3.141592653589793238462643383279502884;
constexpr double DC_RGAS_UNIV = 8.314462618;
constexpr double DC_MR_WATER = 0.01801528;
constexpr double DC_MR_DRY = 0.028966216;
constexpr double DC_RGAS_DRY = DC_RGAS_UNIV / DC_MR_DRY;
constexpr double DC_RGAS_V = DC_RGAS_UNIV / DC_MR_WATER;
constexpr double DC_LATENT_V = 2500930.0;
constexpr double DC_CP_DRY = 1004.64;
constexpr double DC_CP_V = 1865.01;
constexpr double DC_C_L = 4192.664;
constexpr double DC_RHO_L = 998.203;
constexpr double DC_RHO_SOL = 2016.5;
constexpr double DC_MR_SOL = 0.05844277;
constexpr double DC_SURFSIGMA = 7.28e-2;
constexpr double W0 = 1.0;
constexpr double TIME0 = 1000.0;
constexpr double COORD0 = TIME0 * W0;
constexpr double VOL0 = COORD0 * COORD0 * COORD0;
constexpr double CP0 = DC_CP_DRY;
constexpr double MR0 = DC_MR_DRY;
constexpr double R0 = 1e-6;
constexpr double P0 = 100000.0;
constexpr double TEMP0 = 273.15;
constexpr double RHO0 = P0 / (CP0 * TEMP0);
constexpr double MASS0 = R0 * R0 * R0 * RHO0;
constexpr double MASS0grams = MASS0 * 1000;
constexpr double F0 = TIME0 / (RHO0 * R0 * R0);
constexpr double Mr_ratio = DC_MR_WATER / DC_MR_DRY;
constexpr double Cp_dry = DC_CP_DRY / CP0;
constexpr double Cp_v = DC_CP_V / CP0;
constexpr double C_l = DC_C_L / CP0;
constexpr double Latent_v = DC_LATENT_V / (TEMP0 * CP0);
constexpr double Rgas_dry = DC_RGAS_DRY / CP0;
constexpr double Rgas_v = DC_RGAS_V / CP0;
constexpr double Rho_l = DC_RHO_L / RHO0;
constexpr double Rho_sol = DC_RHO_SOL / RHO0;
constexpr double Mr_sol = DC_MR_SOL / MR0;
constexpr double IONIC = 2.0;
constexpr double surfconst = 4.0 * DC_SURFSIGMA * PI * R0 * R0;
constexpr uint32_t OOB = 0xFFFFFFFFu;
constexpr double DBLMAX = 1.7976931348623157e308;

// ---- device error word ----
struct DevError {
  int32_t code;
  uint32_t gbx;
  unsigned long long index;
};

__device__ __forceinline__ void record_error(DevError* e, int code, uint32_t gbx, uint64_t index) {
  if (atomicCAS(&e->code, 0, code) == 0) {
    e->gbx = gbx;
    e->index = index;
  }
}

// context for error attribution of one droplet / pair; `failed`, where set, also marks this
// droplet's own failure (the batch solves report which droplets the reference would abort on)
struct Where {
  DevError* err;
  uint32_t gbx;
  uint64_t index;
  uint32_t* failed = nullptr;
  __device__ void fail(int code) const {
    if (failed) *failed = 1u;
    record_error(err, code, gbx, index);
  }
};

// ---- SuperdropAttrs: superdrop_attrs.hpp:61-259, superdrop_attrs.cpp:34-62 ----
__device__ __forceinline__ double dryradius(double msol) {  // :227-231
  const double vconst = 3.0 / (4.0 * PI);
  const double dryrcubed = vconst * msol / Rho_sol;
  return dpow(dryrcubed, 1.0 / 3.0);
}
__device__ __forceinline__ double rcubed(double r) { return r * r * r; }       // :238
__device__ __forceinline__ double vol(double r) { return 4.0 / 3.0 * PI * rcubed(r); }  // :247
__device__ __forceinline__ double sd_mass(double r, double msol) {  // superdrop_attrs.cpp:54-62
  const double massconst = 4.0 / 3.0 * PI * Rho_l;
  const double density_factor = 1.0 - Rho_l / Rho_sol;
  double m = msol * density_factor;
  m += massconst * rcubed(r);
  return m;
}
__device__ __forceinline__ double condensate_mass(double r, double msol, const Where& w) {  // :208-218
  double m_cond = sd_mass(r, msol) - msol;
  if (m_cond <= -0.0001 * msol) w.fail(CLEO_ERR_NEG_CONDENSATE);
  return fmax(0.0, m_cond);
}
// set_radius: superdrop_attrs.hpp:175-182 (the check; the caller stores)
__device__ __forceinline__ void check_radius(double r, double msol, const Where& w) {
  if (r - dryradius(msol) <= -1e-12 / R0) w.fail(CLEO_ERR_RADIUS_BELOW_DRY);
}
__device__ __forceinline__ void check_xi(uint64_t xi, const Where& w) {  // set_xi :156-163
  if (xi <= 0) w.fail(CLEO_ERR_XI_ZERO);
}

// ---- terminal velocities: terminalvelocity.cpp:32-147 ----
__device__ __forceinline__ double tv_simmel(double radius) {  // :57-85
  const double r1 = 6.7215e-5 / R0;
  const double r2 = 7.5582e-4 / R0;
  const double r3 = 1.73892e-3 / R0;
  const double VELCONST = (100.0 * W0);
  const double a1 = 457950 / VELCONST;
  const double a2 = 4962 / VELCONST;
  const double a3 = 1732 / VELCONST;
  const double a4 = 917 / VELCONST;
  if (radius >= r3) return a4;
  const double massconst = 4.0 / 3.0 * PI * Rho_l;  // watermass :32-40
  const double MASS = (massconst * radius * radius * radius) * MASS0grams;
  // the three branches' a * MASS^y with one inlined pow (the same values)
  const bool big = radius >= r2, mid = radius >= r1;
  const double a = big ? a3 : (mid ? a2 : a1);
  const double y = big ? 1.0 / 6.0 : (mid ? 1.0 / 3.0 : 2.0 / 3.0);
  return a * dpow(MASS, y);
}
__device__ __forceinline__ double tv_rogersyau(double radius) {  // :95-117
  const double r1 = 3e-5 / R0;
  const double r2 = 6e-4 / R0;
  const double r3 = 2e-3 / R0;
  const double k1 = 1.19e8 * R0 * R0 / W0;
  const double k2 = 8000 * R0 / W0;
  const double k3 = 201 / W0;
  const double k4 = 9 / W0;
  if (radius < r1) return k1 * dpow(radius, 2.0);
  if (radius < r2) return k2 * radius;
  if (radius < r3) return k3 * dpow((radius * R0), 0.5);
  return k4;
}
__device__ __forceinline__ double tv_rogersgk(double radius) {  // :127-147
  const double radius0 = 3.725 * 1e-4 / R0;
  const double kcaps = 2.0 * 4.0 * 1000 * R0 / W0;
  const double smallk = -1.0 * 2.0 * 12.0 * 1000 * R0;
  const double acaps = 9.65 / W0;
  const double bcaps = 10.43 / W0;
  const double ccaps = -1.0 * 2.0 * 0.6 * 1000 * R0;
  const bool small = radius < radius0;  // both branches with one inlined exp (same values)
  const double e = dexp((small ? smallk : ccaps) * radius);
  if (small) {
    const double term = 1.0 - e;
    return term * kcaps * radius;
  }
  return acaps - bcaps * e;
}
__device__ __forceinline__ double terminalv(int kind, double radius) {
  switch (kind) {
    case CLEO_TV_SIMMEL: return tv_simmel(radius);
    case CLEO_TV_ROGERSYAU: return tv_rogersyau(radius);
    case CLEO_TV_ROGERSGK: return tv_rogersgk(radius);
    default: return 0.0;
  }
}

// ---- collision probabilities ----
__device__ __forceinline__ double prob_golovin(double r1, double r2, double DELT, double VOLUME) {
  const double prob_jk_const = 1.5e3 * R0 * R0 * R0;  // golovinprob.hpp:40
  const double DELT_DELVOL = DELT / VOLUME;            // golovinprob.cpp:31-43
  const double golovins_kernel = prob_jk_const * (vol(r1) + vol(r2));
  return golovins_kernel * DELT_DELVOL;
}
__device__ __forceinline__ double long_kerneleff(double ra, double rb, double coaleff) {
  const double k1 = 4.5e4 * R0 * R0 * 100 * 100;  // longhydroprob.cpp:29-48
  const double k2 = 3e-4 / R0 / 100;
  const double rlim = 5e-5 / R0;
  const double colleff_min = 0.001;
  const double rsmall = fmin(ra, rb);
  const double rbig = fmax(ra, rb);
  double colleff = 1.0;
  if (rbig < rlim) {
    colleff = k1 * rbig * rbig * (1 - (k2 / rsmall));
    colleff = fmax(colleff, colleff_min);
  }
  return colleff * coaleff;
}
// tv1, tv2: the Simmel terminal velocities of r1, r2 (computed by the caller, possibly once per
// droplet for all its pairs: the same function of the same radius)
__device__ __forceinline__ double prob_hydrodynamic(double r1, double r2, double tv1, double tv2,
                                                    double eff, double DELT,
                                                    double VOLUME) {  // hydrodynamicprob.hpp:49-66
  const double prob_jk_const = PI * R0 * R0 * W0;
  const double DELT_DELVOL = DELT / VOLUME;
  const double sumr = r1 + r2;
  const double sumrsqrd = sumr * sumr;
  const double vdiff = fabs(tv1 - tv2);
  const double hydro_kernel = prob_jk_const * eff * sumrsqrd * vdiff;
  return hydro_kernel * DELT_DELVOL;
}
// pair probability; tv1, tv2 = tv_simmel(r1), tv_simmel(r2) when p.coll_prob is CLEO_PROB_LONG
__device__ __forceinline__ double pair_prob_tv(const cleo_b200_params& p, double r1, double r2,
                                               double tv1, double tv2, double VOLUME) {
  switch (p.coll_prob) {
    case CLEO_PROB_GOLOVIN: return prob_golovin(r1, r2, p.coll_delt, VOLUME);
    case CLEO_PROB_LONG:
      return prob_hydrodynamic(r1, r2, tv1, tv2, long_kerneleff(r1, r2, p.coaleff), p.coll_delt,
                               VOLUME);
    default: return p.const_kernel * p.coll_delt / VOLUME;  // constprob.hpp:44-48
  }
}
// the pair-probability terminal velocity of one droplet (0 when the kernel needs none)
__device__ __forceinline__ double pair_tv(const cleo_b200_params& p, double r) {
  return p.coll_prob == CLEO_PROB_LONG ? tv_simmel(r) : 0.0;
}
__device__ __forceinline__ double pair_prob(const cleo_b200_params& p, double r1, double r2,
                                            double VOLUME) {
  return pair_prob_tv(p, r1, r2, pair_tv(p, r1), pair_tv(p, r2), VOLUME);
}

// ---- collision kinetics: collisionkinetics.cpp:31-67, coalescence_efficiency.cpp:27-38 ----
__device__ __forceinline__ double collision_kinetic_energy(double r1, double r2, double tv1,
                                                          double tv2) {
  const double R0cubed = R0 * R0 * R0;
  const double ckeconst = R0cubed * 2.0 / 3.0 * DC_RHO_L * PI * W0 * W0;
  const double r1cubed = r1 * r1 * r1;
  const double r1_r2cubed = (r1 / r2) * (r1 / r2) * (r1 / r2);
  const double rratio = r1cubed / (1 + r1_r2cubed);
  const double vdiff = tv1 - tv2;
  return ckeconst * rratio * vdiff * vdiff;
}
__device__ __forceinline__ double coal_surfenergy(double r1, double r2) {
  const double r1cubed = r1 * r1 * r1;
  const double r2cubed = r2 * r2 * r2;
  const double rcubedsum = r1cubed + r2cubed;
  return surfconst * dpow(rcubedsum, 2.0 / 3.0);
}
__device__ __forceinline__ double surfenergy(double radius) { return surfconst * (radius * radius); }
__device__ __forceinline__ double ecoal_straub2010(double r1, double r2, double cke) {
  const double beta = -1.15;
  const double surf_c = coal_surfenergy(r1, r2);
  const double weber = cke / surf_c;
  return dexp(beta * weber);
}
__device__ __forceinline__ double nfrags_of(const cleo_b200_params& p, double r1, double r2) {
  if (p.nfrags_kind == CLEO_NFRAGS_CONST) return p.nfrags;  // breakup_nfrags.hpp:40-50
  const double alpha = 1.5;                                   // :54-92
  const double beta = 0.135;
  const double ckemax = 16.49789599 / 1000000;
  const double epsilon = 11.0 / 6.0;
  const double cke = collision_kinetic_energy(r1, r2, terminalv(p.nfrags_tv, r1),
                                              terminalv(p.nfrags_tv, r2));
  const double cke_cap = fmin(ckemax, cke);
  const double gamma = dpow(cke_cap * 1e6, beta);
  return 1.0 / (alpha - gamma) + epsilon;
}
// The outcomes of a collision (flag, coalescence, breakup) run only for the pairs that collide;
// kept out of line, they stay out of the collision kernels' hot loops and instruction caches.
// tv1, tv2: terminalv(p.flag_tv, r1) and terminalv(p.flag_tv, r2) when tv_known (a caller that
// already holds them), else evaluated here
static __device__ __noinline__ unsigned coalbure_flag(const cleo_b200_params& p, double phi,
                                                      double r1, double r2, bool tv_known,
                                                      double tv1, double tv2) {  // coalbure_flag.hpp:42-198
  if (!tv_known && p.flag_kind != CLEO_FLAG_CONST) {
    tv1 = terminalv(p.flag_tv, r1);
    tv2 = terminalv(p.flag_tv, r2);
  }
  switch (p.flag_kind) {
    case CLEO_FLAG_STRAUB: {
      const double cke = collision_kinetic_energy(r1, r2, tv1, tv2);
      return (phi < ecoal_straub2010(r1, r2, cke)) ? 1u : 2u;
    }
    case CLEO_FLAG_TESTIKSTRAUB: {
      const double cke = collision_kinetic_energy(r1, r2, tv1, tv2);
      if (cke < surfenergy(fmin(r1, r2))) return (phi < ecoal_straub2010(r1, r2, cke)) ? 1u : 0u;
      if (cke < surfenergy(fmax(r1, r2))) return (phi < ecoal_straub2010(r1, r2, cke)) ? 1u : 2u;
      return 2u;
    }
    case CLEO_FLAG_SZAKALLURBICH: {
      const double cke = collision_kinetic_energy(r1, r2, tv1, tv2);
      if (cke < surfenergy(fmin(r1, r2))) return 0u;
      if (cke < coal_surfenergy(r1, r2)) return 1u;
      return 2u;
    }
    default: return (phi < p.flag_coaleff) ? 1u : 2u;
  }
}

// one superdroplet's attributes while it takes part in a collision
struct Drop {
  uint64_t xi;
  double r, msol;
};

// ---- coalescence: coalescence.cpp:39-196 ----
__device__ __forceinline__ uint64_t coalescence_gamma(uint64_t xi1, uint64_t xi2, double prob,
                                                      double phi) {  // :68-79
  uint64_t gamma = (uint64_t)floor(prob);
  if (phi < (prob - (double)gamma)) ++gamma;
  if (gamma == 0) return 0;  // fmin(0, maxgamma) is 0: the 64-bit division only when it matters
  const uint64_t maxgamma = xi1 / xi2;
  return (uint64_t)fmin((double)gamma, (double)maxgamma);
}
__device__ __forceinline__ void twin_coalescence(uint64_t gamma, Drop& d1, Drop& d2,
                                                 const Where& w) {  // :131-162
  if (d1.xi != gamma * d2.xi) w.fail(CLEO_ERR_COALESCENCE);
  const uint64_t old_xi = d2.xi;
  const uint64_t new_xi = old_xi / 2;
  if (new_xi >= old_xi) w.fail(CLEO_ERR_COALESCENCE);
  const double new_rcubed = rcubed(d2.r) + (double)gamma * rcubed(d1.r);
  const double new_r = dpow(new_rcubed, (1.0 / 3.0));
  const double new_msol = d2.msol + (double)gamma * d1.msol;
  if (new_xi == 0) {
    d1.xi = 0;  // set_null
  } else {
    check_xi(new_xi, w);
    d1.xi = new_xi;
  }
  check_xi(old_xi - new_xi, w);
  d2.xi = old_xi - new_xi;
  check_radius(new_r, d1.msol, w);
  d1.r = new_r;
  check_radius(new_r, d2.msol, w);
  d2.r = new_r;
  d1.msol = new_msol;
  d2.msol = new_msol;
}
__device__ __forceinline__ void different_coalescence(uint64_t gamma, Drop& d1, Drop& d2,
                                                      const Where& w) {  // :177-196
  if (d1.xi <= gamma * d2.xi) w.fail(CLEO_ERR_COALESCENCE);
  const uint64_t new_xi = d1.xi - gamma * d2.xi;
  if (new_xi >= d1.xi) w.fail(CLEO_ERR_COALESCENCE);
  check_xi(new_xi, w);
  d1.xi = new_xi;
  const double new_rcubed = rcubed(d2.r) + (double)gamma * rcubed(d1.r);
  const double nr = dpow(new_rcubed, (1.0 / 3.0));
  check_radius(nr, d2.msol, w);
  d2.r = nr;
  d2.msol = d2.msol + (double)gamma * d1.msol;
}
static __device__ __noinline__ uint32_t coalesce_pair(uint64_t gamma, Drop& d1, Drop& d2,
                                                  const Where& w) {  // :92-113
  const uint64_t xi1 = d1.xi, xi2 = d2.xi;
  if (xi1 - gamma * xi2 > 0) {
    different_coalescence(gamma, d1, d2, w);
    return 0;
  } else if (xi1 - gamma * xi2 == 0) {
    twin_coalescence(gamma, d1, d2, w);
    return d1.xi == 0 ? 1u : 0u;
  }
  return 0;
}

// ---- breakup: breakup.hpp:140-268 ----
__device__ __forceinline__ void twin_breakup(const cleo_b200_params& p, Drop& d1, Drop& d2,
                                             const Where& w) {  // :193-228
  const uint64_t old_xi = d2.xi;
  const double totnfrags = nfrags_of(p, d1.r, d2.r) * (double)old_xi;
  if ((totnfrags / (double)old_xi) <= 2.5) w.fail(CLEO_ERR_BREAKUP);
  const uint64_t new_xi1 = (uint64_t)round(totnfrags / 2);
  const uint64_t new_xi2 = (uint64_t)round(totnfrags - (double)new_xi1);
  const uint64_t new_xitot = new_xi1 + new_xi2;
  if (new_xi2 <= old_xi) w.fail(CLEO_ERR_BREAKUP);
  if (new_xitot <= (old_xi * 2)) w.fail(CLEO_ERR_BREAKUP);
  const double sum_rcubed = rcubed(d1.r) + rcubed(d2.r);
  const double new_rcubed = sum_rcubed * (double)old_xi / (double)new_xitot;
  const double new_r = dpow(new_rcubed, (1.0 / 3.0));
  const double sum_msol = d1.msol + d2.msol;
  const double new_msol = sum_msol * (double)old_xi / (double)new_xitot;
  check_xi(new_xi1, w);
  d1.xi = new_xi1;
  check_xi(new_xi2, w);
  d2.xi = new_xi2;
  check_radius(new_r, d1.msol, w);
  d1.r = new_r;
  check_radius(new_r, d2.msol, w);
  d2.r = new_r;
  d1.msol = new_msol;
  d2.msol = new_msol;
}
__device__ __forceinline__ void different_breakup(const cleo_b200_params& p, Drop& d1, Drop& d2,
                                                  const Where& w) {  // :235-268
  const uint64_t old_xi1 = d1.xi;
  const uint64_t old_xi2 = d2.xi;
  const uint64_t new_xi1 = old_xi1 - old_xi2;
  check_xi(new_xi1, w);
  d1.xi = new_xi1;
  const double totnfrags = nfrags_of(p, d1.r, d2.r) * (double)old_xi2;
  const uint64_t new_xi2 = (uint64_t)round(totnfrags);
  if ((totnfrags / (double)old_xi2) <= 2.5) w.fail(CLEO_ERR_BREAKUP);
  if (new_xi2 <= old_xi2) w.fail(CLEO_ERR_BREAKUP);
  if ((new_xi1 + new_xi2) <= (old_xi1 + old_xi2)) w.fail(CLEO_ERR_BREAKUP);
  const double sum_rcubed = rcubed(d1.r) + rcubed(d2.r);
  const double new_rcubed = sum_rcubed * (double)old_xi2 / (double)new_xi2;
  const double new_r = dpow(new_rcubed, (1.0 / 3.0));
  const double sum_msol = d1.msol + d2.msol;
  const double new_msol = sum_msol * (double)old_xi2 / (double)new_xi2;
  check_xi(new_xi2, w);
  d2.xi = new_xi2;
  check_radius(new_r, d2.msol, w);
  d2.r = new_r;
  d2.msol = new_msol;
}
static __device__ __noinline__ uint32_t breakup_pair(const cleo_b200_params& p, Drop& d1, Drop& d2,
                                                 const Where& w) {  // :176-186
  if (d1.xi == d2.xi) {
    twin_breakup(p, d1, d2, w);
  } else {
    different_breakup(p, d1, d2, w);
  }
  return 0;
}

// Enact the collision of a pair (already ordered so that d1.xi >= d2.xi): returns the number of
// superdroplets made null. coalescence.cpp:39-54, breakup.hpp:140-166, coalbure.hpp:207-256.
// tv_known, tv1, tv2: the flag's terminal velocities of d1 and d2 when the caller holds them
__device__ __forceinline__ uint32_t enact_collision(const cleo_b200_params& p, Drop& d1, Drop& d2,
                                                   double prob, double phi_coll, double phi_out,
                                                   const Where& w, bool tv_known = false,
                                                   double tv1 = 0.0, double tv2 = 0.0) {
  if (p.coll_enact == CLEO_ENACT_COALESCENCE) {
    const uint64_t gamma = coalescence_gamma(d1.xi, d2.xi, prob, phi_coll);
    if (gamma != 0) return coalesce_pair(gamma, d1, d2, w);
    return 0;
  }
  if (p.coll_enact == CLEO_ENACT_BREAKUP) {
    if (phi_coll < (prob - floor(prob))) return breakup_pair(p, d1, d2, w);
    return 0;
  }
  const uint64_t gamma = coalescence_gamma(d1.xi, d2.xi, prob, phi_coll);
  if (gamma != 0) {
    const unsigned flag = coalbure_flag(p, phi_out, d1.r, d2.r, tv_known, tv1, tv2);
    if (flag == 1u) return coalesce_pair(gamma, d1, d2, w);
    if (flag == 2u) return breakup_pair(p, d1, d2, w);
  }
  return 0;
}

// ---- thermodynamic equations: thermodynamic_equations.{hpp:44-107, cpp:38-145} ----
__device__ __forceinline__ double dry_air_density(double press, double temp, double qvap) {
  const double rgas_equiv = Rgas_dry + Rgas_v * qvap;
  return press / (rgas_equiv * temp);
}
__device__ __forceinline__ double moist_specifc_heat(double qvap, double qcond) {
  return Cp_dry + Cp_v * (qvap) + C_l * (qcond);
}
__device__ __forceinline__ double supersaturation_ratio(double press, double qvap, double psat) {
  return (press * qvap) / ((Mr_ratio + qvap) * psat);
}
__device__ __forceinline__ double saturation_pressure(double temp, const Where& w) {
  if (temp <= 0) w.fail(CLEO_ERR_TEMPERATURE);
  const double A = 17.4146;
  const double B = 33.639;
  const double TREF = 273.16;
  const double PREF = 611.655;
  const double T = temp * TEMP0;
  return (PREF * dexp(A * (T - TREF) / (T - B))) / P0;
}
__device__ __forceinline__ double diffusion_factor(double press, double temp, double psat) {
  const double A = 7.11756e-5;
  const double B = 4.38127686e-3;
  const double LATENT_RGAS_V = DC_LATENT_V / DC_RGAS_V;
  const double D = 4.012182971e-5;
  const double TEMP = temp * TEMP0;
  const double PRESS = press * P0;
  const double PSAT = psat * P0;
  const double THERMK = A * dpow(TEMP, 2.0) + TEMP * B;
  const double DIFFUSE_V = (D / PRESS * dpow(TEMP, 1.94)) / DC_RGAS_V;
  const double fkl = (LATENT_RGAS_V / TEMP - 1.0) * DC_LATENT_V / (THERMK * F0);
  const double fdl = TEMP / (DIFFUSE_V * PSAT) / F0;
  return Rho_l * (fkl + fdl);
}
// ventilation_factor (impliciteuler.cpp:131-145) with the correctly rounded powers
__device__ __forceinline__ double ventilation_factor_cr(double radius) {
  const double vent_factor_max = 20;
  const double C1 = 6.954e+7;
  const double A = 1.963;
  const double C2 = 1.069e+3;
  const double B = 0.702;
  double pa, pb;  // pow(radius * R0, A) and pow(radius * R0, B), one logarithm
  dpow2(radius * R0, A, B, pa, pb);
  const double a = 1.0 / (C1 * pa);
  const double b = 1.0 / (C2 * pb);
  const double vent_factor = 1.0 + 1.0 / (a + b);
  return fmin(vent_factor, vent_factor_max);
}
// x^y for 2^-60 <= x < 1 (x = 2^e m, m in [1, 2)) from the library's log2 and exp2, relative
// error below 2^-50: log2 m to 2^-53 absolute (1 ulp documented, |log2 m| < 1), so y log2 m to
// 2^-51 with its rounding (y < 2); y e exact as a double-double; exp2 of the sum's high part
// (2 ulp documented) times 1 + lo ln2 (lo below 2^-46, so the omitted term is below 2^-93)
__device__ __forceinline__ double vent_pow(double y, int e, double lm) {
  const dd ye = two_prod(y, (double)e);
  dd z = two_sum(ye.hi, y * lm);
  z = fast_two_sum(z.hi, z.lo + ye.lo);
  return exp2(z.hi) * (1.0 + z.lo * 0.69314718055994530942);
}
// The same doubles as ventilation_factor_cr, from powers good to 2^-50 where they decide it.
// The result is 1 + d, d = 1 / (a + b), rounded once. With the powers off by at most eps
// (relative) from the correctly rounded ones, each of the five rounded steps up to d adds at most
// 2^-52, so d is within (eps + 2^-50) d of the reference's; when 1 + d lies farther than that
// from the rounding boundaries around RN(1 + d) (two_sum gives its exact remainder), the
// reference rounds to the same double. eps is taken as 2^-48 (the analysis gives 2^-49.6 with the
// correctly rounded value's half ulp). The check fails in about 2^6 d of the cases, so a warp
// tries this form only when all its droplets are below 1.5 um (d below about 2e-4); otherwise,
// and when the check fails, the correctly rounded powers decide.
__device__ __forceinline__ double ventilation_factor(double radius) {
  const double x = radius * R0;
  const bool quick = x >= 0x1p-60 && x < 1.5e-6;
  if (__all_sync(__activemask(), quick)) {
    const uint64_t xb = dbits(x);
    const int e = (int)((xb >> 52) & 0x7FF) - 1023;
    const double lm = log2(bitsd((xb & 0x000FFFFFFFFFFFFFull) | 0x3FF0000000000000ull));
    const double pa = vent_pow(1.963, e, lm), pb = vent_pow(0.702, e, lm);
    const double a = 1.0 / (6.954e+7 * pa);
    const double b = 1.0 / (1.069e+3 * pb);
    const double d = 1.0 / (a + b);
    const dd v = two_sum(1.0, d);  // v.hi = RN(1 + d), v.lo = 1 + d - v.hi exactly
    const double bound = d * 0x1p-47;
    const uint64_t vb = dbits(v.hi);
    const double u = bitsd(vb & 0x7FF0000000000000ull) * 0x1p-52;  // ulp of v.hi in [1, 20)
    const double d_up = 0.5 * u;
    const double d_down = (vb & 0x000FFFFFFFFFFFFFull) == 0 ? 0.25 * u : 0.5 * u;
    if (v.hi < 19.0 && v.lo + bound < d_up && v.lo - bound > -d_down) return v.hi;
  }
  return ventilation_factor_cr(radius);
}
__device__ __forceinline__ double kohler_a(double temp) {
  const double akoh_constant = 3.3e-7 / (TEMP0 * R0);
  return akoh_constant / temp;
}
__device__ __forceinline__ double kohler_b(double msol) {
  const double bkoh_constant = 4.3e-6 * RHO0 / MR0;
  return bkoh_constant * msol * IONIC / Mr_sol;
}
__device__ __forceinline__ void kohler_factors(double msol, double temp, double& akoh,
                                               double& bkoh) {
  akoh = kohler_a(temp);
  bkoh = kohler_b(msol);
}

// ---- ImplicitEuler: impliciteuler.{hpp:41-345, cpp:35-301} ----
struct OdeConsts {
  double s_ratio, akoh, bkoh, ffactor_fv;
};
struct NewtonCfg {
  uint32_t maxniters;
  double rtol, atol;
};
// Upper bound on the Newton iterations of one solve (all sub-steps). Legitimate solves need at
// most (delt / minsubdelt) * (2 + maxniters); this bound only stops a runaway solve, reported as
// CLEO_ERR_TIMEOUT, so that no thread can spin for long.
constexpr uint32_t NR_ITER_CAP = 4u << 20;

// ode_gfunc (:270-281) at one iterate z = r^2, keeping the terms that ode_gfuncderivative
// (:291-301) shares at the same z. The reference evaluates g at each new iterate twice (as the
// convergence check of one iteration and as the numerator of the next) and recomputes sqrt(z),
// z^(3/2) and akoh/r for g'; one evaluation per iterate gives the same doubles, because each
// value is the same expression of the same inputs.
// g's beta is (2 subdelt) / (z F) and g''s is subdelt / (z F) with the same rounded product z F;
// scaling by 2 commutes with rounding to nearest (no overflow or underflow at these magnitudes),
// so the first is exactly twice the second and one division serves both.
struct GEval {
  double z, radius, akr, r3, q, g;
};
__device__ __forceinline__ GEval eval_g(const OdeConsts& o, double subdelt, double rprev,
                                        double rsqrd) {
  GEval e;
  e.z = rsqrd;
  e.radius = sqrt(rsqrd);
  e.akr = o.akoh / e.radius;
  e.r3 = dpow(e.radius, 3.0);
  const double alpha = o.s_ratio - 1 - e.akr + o.bkoh / e.r3;
  e.q = subdelt / (rsqrd * o.ffactor_fv);
  const double beta = 2.0 * e.q;
  const double gamma = dpow(rprev / e.radius, 2.0);
  e.g = 1 - gamma - alpha * beta;
  return e;
}
__device__ __forceinline__ double eval_gprime(const OdeConsts& o, const GEval& e) {
  const double alpha = e.akr - 3.0 * o.bkoh / e.r3;
  return 1 - alpha * e.q;
}
// iterate_rootfinding_algorithm: impliciteuler.cpp:239-255 (+ check_for_convergence, hpp:213-219)
__device__ __forceinline__ GEval nr_iterate(const NewtonCfg& c, const OdeConsts& o,
                                            double subdelt, double rprev, const GEval& e,
                                            bool& converged, uint32_t& niters) {
  const double numerator = e.g;
  const double denominator = eval_gprime(o, e);
  double ziter = e.z * (1 - numerator / denominator);
  ziter = fmax(ziter, 1e-8);
  const GEval next = eval_g(o, subdelt, rprev, ziter);
  const double conv = c.rtol * fabs(next.g) + c.atol;
  converged = fabs(next.g - numerator) < conv;
  ++niters;
  return next;
}
// integrate_condensation_ode: impliciteuler.cpp:128-141 with newtonraphson_niterations (:181-194)
// and newtonraphson_untilconverged (:207-227). e0 is g at the initial guess. Returns 0 or the
// failure code; z receives the last iterate either way.
__device__ __forceinline__ int integrate_ode_core(const NewtonCfg& c, const OdeConsts& o,
                                                  double subdelt, double rprev, const GEval& e0,
                                                  uint32_t& niters, double& z) {
  bool conv = false;
  GEval e = nr_iterate(c, o, subdelt, rprev, e0, conv, niters);
  const bool conv1 = conv;
  const double z1 = e.z;
  e = nr_iterate(c, o, subdelt, rprev, e, conv, niters);
  if (conv) {
    z = e.z;
    return 0;
  }
  // the restart from e0 (newtonraphson_untilconverged): its first two iterations repeat the two
  // above exactly, so they are taken from them, each behind the checks the restart makes before it
  if (1 > c.maxniters) {
    z = e0.z;
    return CLEO_ERR_NR_NOCONVERGE;
  }
  if (niters >= NR_ITER_CAP) {
    z = e0.z;
    return CLEO_ERR_TIMEOUT;
  }
  niters += 1;
  if (conv1) {
    z = z1;
    return 0;
  }
  if (2 > c.maxniters) {
    z = z1;
    return CLEO_ERR_NR_NOCONVERGE;
  }
  if (niters >= NR_ITER_CAP) {
    z = z1;
    return CLEO_ERR_TIMEOUT;
  }
  niters += 1;
  conv = false;  // as after the second iteration above
  uint32_t niter = 3;
  int code = 0;
  while (!conv) {
    if (niter > c.maxniters) {
      code = CLEO_ERR_NR_NOCONVERGE;
      break;
    }
    if (niters >= NR_ITER_CAP) {
      code = CLEO_ERR_TIMEOUT;
      break;
    }
    e = nr_iterate(c, o, subdelt, rprev, e, conv, niters);
    niter += 1;
  }
  z = e.z;
  return code;
}
// The restart of integrate_ode_core (newtonraphson_untilconverged from the initial guess,
// impliciteuler.cpp:131-132, 207-227) when the two iterations before it have already been done:
// the restart's first two iterations repeat them exactly, so it can continue from them. zres is
// -z1 when the first iteration passed the convergence test (the restart stops after it) and z2
// otherwise (the second did not pass it, or there would be no restart). Adds the restart's
// iterations, the repeated ones included, to niters; needs maxniters >= 2.
__device__ __forceinline__ int resume_restart(const NewtonCfg& c, const OdeConsts& o,
                                              double subdelt, double rprev, double zres,
                                              uint32_t& niters, double& z) {
  if (zres < 0.0) {
    niters += 1;
    z = -zres;
    return 0;
  }
  niters += 2;
  GEval e = eval_g(o, subdelt, rprev, zres);
  bool conv = false;
  uint32_t niter = 3;
  int code = 0;
  while (!conv) {
    if (niter > c.maxniters) {
      code = CLEO_ERR_NR_NOCONVERGE;
      break;
    }
    if (niters >= NR_ITER_CAP) {
      code = CLEO_ERR_TIMEOUT;
      break;
    }
    e = nr_iterate(c, o, subdelt, rprev, e, conv, niters);
    niter += 1;
  }
  z = e.z;
  return code;
}
__device__ __forceinline__ double integrate_ode(const NewtonCfg& c, const OdeConsts& o,
                                                double subdelt, double rprev, const GEval& e0,
                                                uint32_t& niters, const Where& w) {
  double z;
  const int code = integrate_ode_core(c, o, subdelt, rprev, e0, niters, z);
  if (code) w.fail(code);
  return z;
}
// a usable seed: finite and positive (NaN compares false)
__device__ __forceinline__ bool seed_ok(double seed_rsqrd) {
  return seed_rsqrd > 0.0 && seed_rsqrd <= DBLMAX;
}
// Newton iterations from a seed, the convergence test (check_for_convergence) after every one,
// at most SEED_MAXITERS: a good seed converges in one or two, a poor one is abandoned early
// (the caller then starts from the reference guess). Returns true when converged.
constexpr uint32_t SEED_MAXITERS = 6;
__device__ __forceinline__ bool integrate_seeded(const NewtonCfg& c, const OdeConsts& o,
                                                 double subdelt, double rprev, GEval e,
                                                 uint32_t& niters, double& z) {
  bool conv = false;
  for (uint32_t k = 0; k < SEED_MAXITERS; ++k) {
    e = nr_iterate(c, o, subdelt, rprev, e, conv, niters);
    if (conv) break;
  }
  z = e.z;
  return conv;
}
// Whether a root reached from a seed is the root the reference's guess leads to. With
// h(z) = z g(z) = z - rprev^2 - (2 delt / F)(s - 1 - a/r + b/r^3), h'(z) = 1 - (delt/F) f'(r)/r
// with f'(r) = a/r^2 - 3b/r^4, whose largest value over r (at r^2 = 5b/a) keeps h' > 0 exactly
// when delt < 2.5 F/a (5b/a)^1.5, the critical timestep: then the root is unique. Otherwise the
// direct branch was taken for an unactivated droplet (ucrit1), and h is increasing only on
// (0, 3b/a], where f' < 0; a seeded root is accepted there, where it is the only one.
__device__ __forceinline__ bool seeded_root_ok(const OdeConsts& o, bool ucrit1, double z) {
  return !ucrit1 || z <= 3.0 * o.bkoh / o.akoh;
}
// The factors of initialguess and first_unique_criteria that depend on akoh alone, i.e. on the
// gridbox's temperature: the batched schedule evaluates them once per gridbox (same expressions,
// so the same doubles). The two differ in rounding (a correctly rounded cube against a product).
__device__ __forceinline__ double activation_a3(double akoh) { return 4.0 * dpow(akoh, 3.0) / 27; }
__device__ __forceinline__ double unique_a3(double akoh) { return 4.0 * akoh * akoh * akoh / 27.0; }
// initialguess (:156-170) given a3 = activation_a3(o.akoh)
__device__ __forceinline__ double initialguess_a3(const OdeConsts& o, double rprev, double a3) {
  const double s_act = 1 + sqrt(a3 / o.bkoh);
  if (o.s_ratio > s_act) {
    const double bigr = 1e-3 / R0;
    const double maxradius = fmax(bigr, rprev);
    return maxradius * maxradius;
  }
  return rprev * rprev;
}
__device__ __forceinline__ double initialguess(const OdeConsts& o, double rprev) {  // :156-170
  return initialguess_a3(o, rprev, activation_a3(o.akoh));
}
// first_unique_criteria (:69-83) given a3 = unique_a3(o.akoh)
__device__ __forceinline__ bool first_unique_a3(const OdeConsts& o, double rprev, double ziter,
                                                double a3) {
  const double akoh = o.akoh;
  const double bkoh = o.bkoh;
  const double rcritsqrd = 3.0 * bkoh / akoh;
  const bool is_ziter_unactivated = ziter < rcritsqrd;
  const bool is_unactivated = (rprev * rprev < rcritsqrd && is_ziter_unactivated);
  const double sqrdval = a3 / bkoh;
  const bool is_subactivated_saturation = (o.s_ratio <= 1.0 + dpow(sqrdval, 0.5));
  return (is_unactivated && is_subactivated_saturation);
}
__device__ __forceinline__ bool first_unique_criteria(const OdeConsts& o, double rprev,
                                                      double ziter) {  // :69-83
  return first_unique_a3(o, rprev, ziter, unique_a3(o.akoh));
}
__device__ __forceinline__ double critical_timestep(const OdeConsts& o) {  // hpp:266-269
  const double cuberoot = dpow(5.0 * o.bkoh / o.akoh, 1.5);
  return 2.5 * o.ffactor_fv / o.akoh * cuberoot;
}
// delt <= critical_timestep(o), decided from x sqrt(x) in place of the correctly rounded
// pow(x, 1.5): the two estimates of the timestep differ by a few units in the last place, so
// outside a band of 1e-12 relative around the estimate the answer is the same, and inside it
// the exact timestep decides. `crit` receives the timestep used (the estimate outside the band).
__device__ __forceinline__ bool below_critical_timestep(const OdeConsts& o, double delt,
                                                        double& crit) {
  const double x = 5.0 * o.bkoh / o.akoh;
  crit = 2.5 * o.ffactor_fv / o.akoh * (x * sqrt(x));
  const double band = 1e-12 * fabs(crit);
  if (delt <= crit - band) return true;
  if (delt > crit + band) return false;
  crit = critical_timestep(o);  // also where the estimate is not finite
  return delt <= crit;
}
// fmax(r, dryradius(msol)) (change_radius, superdrop.hpp) without the cube root where r is
// plainly the larger: r^3 Rho_sol > vconst msol (1 + 1e-13) gives r > dryradius(msol), the
// margin being about 100 times the rounding of both sides and of the cube root; fmax then
// returns r, as it does after the cube root. Otherwise (and for NaN) the cube root decides.
__device__ __forceinline__ double max_dryradius(double r, double msol) {
  const double vconst = 3.0 / (4.0 * PI);
  if (r * r * r * Rho_sol > vconst * msol * (1.0 + 1e-13)) return r;
  return fmax(r, dryradius(msol));
}
// solve_condensation: impliciteuler.cpp:35-54 (+ substepping :98-113). A usable seed_rsqrd
// replaces the Newton start of the direct branch (not the branch decision) by a predicted r^2.
// solve_condensation_fv takes the diffusion factor already divided by the ventilation factor of
// rprev (what solve_condensation computes first), for a caller that holds it
__device__ __forceinline__ double solve_condensation_fv(const NewtonCfg& c, double delt,
                                                        double minsubdelt, double s_ratio,
                                                        double akoh, double bkoh,
                                                        double ffactor_fv, double rprev,
                                                        double seed_rsqrd, uint32_t& niters,
                                                        const Where& w) {
  const OdeConsts o{s_ratio, akoh, bkoh, ffactor_fv};
  double ziter = initialguess(o, rprev);
  // ucrit1 || ucrit2: the critical timestep (a general pow) is only needed when ucrit1 fails
  const bool ucrit1 = first_unique_criteria(o, rprev, ziter);
  double crit;  // the sub-stepping branch below takes the exact timestep
  const bool direct = ucrit1 || below_critical_timestep(o, delt, crit);
  double rsqrd;
  if (direct) {
    const GEval e0 = eval_g(o, delt, rprev, ziter);
    // a seed is used when its residual is smaller than the reference guess's; a seeded solve
    // that does not converge within SEED_MAXITERS, or ends on another root, restarts from the
    // reference's guess
    bool done = false;
    if (seed_ok(seed_rsqrd)) {
      const GEval es = eval_g(o, delt, rprev, seed_rsqrd);
      if (fabs(es.g) < fabs(e0.g) && integrate_seeded(c, o, delt, rprev, es, niters, rsqrd) &&
          seeded_root_ok(o, ucrit1, rsqrd))
        done = true;
    }
    if (!done) rsqrd = integrate_ode(c, o, delt, rprev, e0, niters, w);
  } else {
    const double critdelt = critical_timestep(o);
    const double mindelt = fmax(critdelt, minsubdelt);
    double remdelt = delt;
    while (remdelt > 0.0) {
      if (niters >= NR_ITER_CAP) {
        w.fail(CLEO_ERR_TIMEOUT);
        break;
      }
      const double subdelt = fmin(mindelt, remdelt);
      ziter = integrate_ode(c, o, subdelt, rprev, eval_g(o, subdelt, rprev, ziter), niters, w);
      rprev = dpow(ziter, 0.5);
      remdelt -= subdelt;
    }
    rsqrd = ziter;
  }
  return sqrt(rsqrd);
}
__device__ __forceinline__ double solve_condensation(const NewtonCfg& c, double delt,
                                                     double minsubdelt, double s_ratio,
                                                     double akoh, double bkoh, double ffactor,
                                                     double rprev, double seed_rsqrd,
                                                     uint32_t& niters, const Where& w) {
  return solve_condensation_fv(c, delt, minsubdelt, s_ratio, akoh, bkoh,
                               ffactor / ventilation_factor(rprev), rprev, seed_rsqrd, niters, w);
}

// ---- scheduling: microphysicalprocess.hpp:222-248 ----
__host__ __device__ __forceinline__ bool on_step(uint32_t interval, uint32_t t) {
  return (t % interval == 0) && (interval != CLEO_STEP_OFF);
}
__host__ __device__ __forceinline__ uint32_t next_step(uint32_t interval, uint32_t t) {
  if (interval == CLEO_STEP_OFF) return CLEO_STEP_OFF;
  return ((t / interval) + 1) * interval;
}

}  // namespace cleo
