/*
 * cleo_oracle.c — CPU restatement of CLEO's super-droplet hot path (TEST INFRASTRUCTURE ONLY).
 *
 * The checker for the CUDA path: restates, in C and with the reference's operation order, the
 * functions on CLEO v0.69.0's SDM hot path (paths below are relative to the CLEO project root).
 * Every function names the reference lines it follows. Floating-point expressions keep the
 * reference's association and use the same libm calls (pow, exp, sqrt, floor, round, fmin, fmax),
 * so results differ from the reference only where libm does. Compile without FMA contraction.
 * Aborts of the reference become error codes (the first one is kept).
 *
 * Two builds (oracle/Makefile):
 *   liboracle.so     pow and exp from the host libm, as the reference calls them: this build is
 *                    pinned bit for bit to CLEO's own sources compiled here;
 *   liboracle_cr.so  the same code with pow and exp correctly rounded (ORACLE_CR_LIBM, see
 *                    oracle/crlibm.cpp), the arithmetic the CUDA path documents: there the CUDA
 *                    path must agree bit for bit, and the two builds differ only where the host
 *                    libm misrounds.
 * The loops over gridboxes of one SDM step can run on OpenMP threads (oc_set_num_threads); every
 * gridbox's work is independent of the others' within a loop, so results are the same doubles
 * for any number of threads.
 */
#include "cleo_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifdef ORACLE_CR_LIBM
/* correctly rounded pow and exp (oracle/crlibm.cpp) in place of the host libm's */
double oc_cr_pow(double x, double y);
double oc_cr_exp(double x);
#define pow(x, y) oc_cr_pow((x), (y))
#define exp(x) oc_cr_exp((x))
#endif

#include "../include/cleo_b200_rng.h"

/* ------------------------------------------------------------------------------------------ */
/* constants: libs/cleoconstants.hpp:32-118                                                   */
/* ------------------------------------------------------------------------------------------ */
#define PI 3.141592653589793238462643383279502884 /* std::numbers::pi */
/* dimmed_constants (cleoconstants.hpp:32-66) */
#define DC_RGAS_UNIV 8.314462618
#define DC_MR_WATER 0.01801528
#define DC_MR_DRY 0.028966216
#define DC_RGAS_DRY (DC_RGAS_UNIV / DC_MR_DRY)
#define DC_RGAS_V (DC_RGAS_UNIV / DC_MR_WATER)
#define DC_LATENT_V 2500930.0
#define DC_CP_DRY 1004.64
#define DC_CP_V 1865.01
#define DC_C_L 4192.664
#define DC_RHO_L 998.203
#define DC_RHO_SOL 2016.5
#define DC_MR_SOL 0.05844277
#define DC_SURFSIGMA 7.28e-2
/* dimless_constants (cleoconstants.hpp:68-104) */
static const double W0 = 1.0;
static const double TIME0 = 1000.0;
#define COORD0 (1000.0 * 1.0)
#define VOL0 (COORD0 * COORD0 * COORD0)
#define CP0 DC_CP_DRY
#define MR0 DC_MR_DRY
#define R0 1e-6
#define P0 100000.0
#define TEMP0 273.15
#define RHO0 (P0 / (CP0 * TEMP0))
#define MASS0 (R0 * R0 * R0 * RHO0)
#define MASS0grams (MASS0 * 1000)
#define F0 (1000.0 / (RHO0 * R0 * R0))
#define Mr_ratio (DC_MR_WATER / DC_MR_DRY)
#define Cp_dry (DC_CP_DRY / CP0)
#define Cp_v (DC_CP_V / CP0)
#define C_l (DC_C_L / CP0)
#define Latent_v (DC_LATENT_V / (TEMP0 * CP0))
#define Rgas_dry (DC_RGAS_DRY / CP0)
#define Rgas_v (DC_RGAS_V / CP0)
#define Rho_l (DC_RHO_L / RHO0)
#define Rho_sol (DC_RHO_SOL / RHO0)
#define Mr_sol (DC_MR_SOL / MR0)
#define IONIC 2.0
#define surfconst (4.0 * DC_SURFSIGMA * PI * R0 * R0)
#define OOB 0xFFFFFFFFu /* LIMITVALUES::oob_gbxindex */
#define LLIM (-1.0 * DBL_MAX)
#define ULIM (DBL_MAX)

/* ------------------------------------------------------------------------------------------ */
/* context and error recording                                                                */
/* ------------------------------------------------------------------------------------------ */
typedef struct {
  uint32_t gbx;
  double c3, c1, c2;
  uint64_t xi;
  double r, msol;
  uint64_t id;
} sd_t; /* Superdrop (superdrop.hpp:36-48), AoS like the reference */

struct oc_ctx {
  cleo_b200_params p;
  uint32_t ngbxs;
  uint32_t ndims[3];
  double *b3lo, *b3hi, *b1lo, *b1hi, *b2lo, *b2hi;
  uint32_t *back3, *fwd3, *back1, *fwd1, *back2, *fwd2;
  /* gridbox states */
  double *volume, *press, *temp, *qvap, *qcond, *wlo, *whi, *ulo, *uhi, *vlo, *vhi;
  double* cond_mass;
  uint64_t* nr_iters;
  /* superdroplets */
  size_t capacity, ntot, ndomain;
  sd_t* sd;
  sd_t* tmp;
  size_t* refs0; /* SupersInGbx refs per gridbox, relative to the domain start */
  size_t* refs1;
  size_t* counts;
  /* SDMMonitor members (params.monitors): [0] all droplets, [1] raindrops; changes after
   * microphysics ([.][0]) and after motion ([.][1]); the previous moments; precipitation */
  double* gbxarea;
  uint64_t* mm0[2][2];
  float *mm1[2][2], *mm2[2][2];
  uint64_t* prev0[2];
  float *prev1[2], *prev2[2];
  double* precip;
  /* errors */
  cleo_b200_error err;
};

/* per thread: the error slot of the context being stepped (or of this thread's share of a
 * parallel loop) and the Newton iteration counter of the current solve */
static _Thread_local cleo_b200_error* g_err;
static _Thread_local uint64_t* g_iters;
static int g_nthreads = 1; /* threads of the gridbox loops (oc_set_num_threads) */

/* set by every abort of the current thread's work, cleared by the batch solves per droplet */
static _Thread_local int g_failed;

static void set_error(int code, uint32_t gbx, uint64_t index) {
  g_failed = 1;
  if (g_err && g_err->code == CLEO_OK) {
    g_err->code = code;
    g_err->gbxindex = gbx;
    g_err->index = index;
  }
}

/* the superdroplet being processed (for error attribution) */
static _Thread_local uint32_t g_cur_gbx = OOB;
static _Thread_local uint64_t g_cur_sd = 0;

/* A loop over gridboxes on several threads: each thread records its first error, that is the one
 * of the lowest gridbox it visits (OpenMP hands a thread its iterations in increasing order), and
 * the error of the lowest gridbox over all threads is the one the sequential loop meets first. */
static void merge_error(cleo_b200_error* into, const cleo_b200_error* e) {
  if (e->code == CLEO_OK) return;
  if (into->code == CLEO_OK || e->gbxindex < into->gbxindex ||
      (e->gbxindex == into->gbxindex && e->index < into->index))
    *into = *e;
}

/* ------------------------------------------------------------------------------------------ */
/* SuperdropAttrs: superdrop_attrs.hpp:61-259, superdrop_attrs.cpp:34-62                      */
/* ------------------------------------------------------------------------------------------ */
/* dryradius(): superdrop_attrs.hpp:227-231 */
static double dryradius(double msol) {
  const double vconst = 3.0 / (4.0 * PI);
  const double dryrcubed = vconst * msol / Rho_sol;
  return pow(dryrcubed, 1.0 / 3.0);
}
/* rcubed(): superdrop_attrs.hpp:238 */
static double rcubed(double r) { return r * r * r; }
/* vol(): superdrop_attrs.hpp:247 */
static double vol(double r) { return 4.0 / 3.0 * PI * rcubed(r); }
/* mass(): superdrop_attrs.cpp:54-62 */
static double sd_mass(double r, double msol) {
  const double massconst = 4.0 / 3.0 * PI * Rho_l;
  const double density_factor = 1.0 - Rho_l / Rho_sol;
  double m = msol * density_factor;
  m += massconst * rcubed(r);
  return m;
}
/* condensate_mass(): superdrop_attrs.hpp:208-218 */
static double condensate_mass(double r, double msol) {
  double m_cond = sd_mass(r, msol) - msol;
  if (m_cond <= -0.0001 * msol) set_error(CLEO_ERR_NEG_CONDENSATE, g_cur_gbx, g_cur_sd);
  m_cond = fmax(0.0, m_cond);
  return m_cond;
}
/* set_xi(): superdrop_attrs.hpp:156-163 */
static void set_xi(sd_t* d, uint64_t xi) {
  if (xi <= 0) set_error(CLEO_ERR_XI_ZERO, g_cur_gbx, g_cur_sd);
  d->xi = xi;
}
/* set_radius(): superdrop_attrs.hpp:175-182 */
static void set_radius(sd_t* d, double r) {
  if (r - dryradius(d->msol) <= -1e-12 / R0) set_error(CLEO_ERR_RADIUS_BELOW_DRY, g_cur_gbx, g_cur_sd);
  d->r = r;
}
/* set_null(): superdrop.hpp (Superdrop::set_null) + superdrop_attrs.hpp:147 */
static void set_null(sd_t* d) {
  d->xi = 0;
  d->gbx = OOB;
}
/* change_radius(): superdrop_attrs.cpp:34-44 */
static double change_radius(sd_t* d, double newr) {
  const double oldradius = d->r;
  const double dryr = dryradius(d->msol);
  d->r = fmax(newr, dryr);
  return d->r - oldradius;
}

/* ------------------------------------------------------------------------------------------ */
/* terminal velocities: terminalvelocity.cpp:32-147                                           */
/* ------------------------------------------------------------------------------------------ */
/* SimmelTerminalVelocity::watermass: terminalvelocity.cpp:32-40 */
static double simmel_watermass(double radius) {
  const double massconst = 4.0 / 3.0 * PI * Rho_l;
  const double mass = massconst * radius * radius * radius;
  return mass * MASS0grams;
}
/* SimmelTerminalVelocity::operator(): terminalvelocity.cpp:57-85 */
static double tv_simmel(double radius) {
  const double r1 = 6.7215e-5 / R0;
  const double r2 = 7.5582e-4 / R0;
  const double r3 = 1.73892e-3 / R0;
  const double VELCONST = (100.0 * W0);
  const double a1 = 457950 / VELCONST;
  const double a2 = 4962 / VELCONST;
  const double a3 = 1732 / VELCONST;
  const double a4 = 917 / VELCONST;
  if (radius >= r3) {
    return a4;
  } else {
    const double MASS = simmel_watermass(radius);
    if (radius >= r2) {
      return a3 * pow(MASS, 1.0 / 6.0);
    } else if (radius >= r1) {
      return a2 * pow(MASS, 1.0 / 3.0);
    } else {
      return a1 * pow(MASS, 2.0 / 3.0);
    }
  }
}
/* RogersYauTerminalVelocity::operator(): terminalvelocity.cpp:95-117 */
static double tv_rogersyau(double radius) {
  const double r1 = 3e-5 / R0;
  const double r2 = 6e-4 / R0;
  const double r3 = 2e-3 / R0;
  const double k1 = 1.19e8 * R0 * R0 / W0;
  const double k2 = 8000 * R0 / W0;
  const double k3 = 201 / W0;
  const double k4 = 9 / W0;
  if (radius < r1) {
    return k1 * pow(radius, 2.0);
  } else if (radius < r2) {
    return k2 * radius;
  } else if (radius < r3) {
    return k3 * pow((radius * R0), 0.5);
  } else {
    return k4;
  }
}
/* RogersGKTerminalVelocity::operator(): terminalvelocity.cpp:127-147 */
static double tv_rogersgk(double radius) {
  const double radius0 = 3.725 * 1e-4 / R0;
  const double kcaps = 2.0 * 4.0 * 1000 * R0 / W0;
  const double smallk = -1.0 * 2.0 * 12.0 * 1000 * R0;
  const double acaps = 9.65 / W0;
  const double bcaps = 10.43 / W0;
  const double ccaps = -1.0 * 2.0 * 0.6 * 1000 * R0;
  if (radius < radius0) {
    const double term = 1.0 - exp(smallk * radius);
    return term * kcaps * radius;
  } else {
    return acaps - bcaps * exp(ccaps * radius);
  }
}
static double terminalv(int kind, double radius) {
  switch (kind) {
    case CLEO_TV_SIMMEL: return tv_simmel(radius);
    case CLEO_TV_ROGERSYAU: return tv_rogersyau(radius);
    case CLEO_TV_ROGERSGK: return tv_rogersgk(radius);
    default: return 0.0; /* NullTerminalVelocity, terminalvelocity.hpp:44-53 */
  }
}
double oc_terminal_velocity(int kind, double radius) { return terminalv(kind, radius); }

/* ------------------------------------------------------------------------------------------ */
/* collision probabilities                                                                    */
/* ------------------------------------------------------------------------------------------ */
/* GolovinProb: golovinprob.hpp:40, golovinprob.cpp:31-43 */
static double prob_golovin(const sd_t* d1, const sd_t* d2, double DELT, double VOLUME) {
  const double prob_jk_const = 1.5e3 * R0 * R0 * R0;
  const double DELT_DELVOL = DELT / VOLUME;
  const double golovins_kernel = prob_jk_const * (vol(d1->r) + vol(d2->r));
  return golovins_kernel * DELT_DELVOL;
}
/* LongHydroProb::kerneleff: longhydroprob.cpp:29-48 */
static double long_kerneleff(const sd_t* d1, const sd_t* d2, double coaleff) {
  const double k1 = 4.5e4 * R0 * R0 * 100 * 100;
  const double k2 = 3e-4 / R0 / 100;
  const double rlim = 5e-5 / R0;
  const double colleff_min = 0.001;
  const double rsmall = fmin(d1->r, d2->r);
  const double rbig = fmax(d1->r, d2->r);
  double colleff = 1.0;
  if (rbig < rlim) {
    colleff = k1 * rbig * rbig * (1 - (k2 / rsmall));
    colleff = fmax(colleff, colleff_min);
  }
  return colleff * coaleff;
}
/* HydrodynamicProb<SimmelTerminalVelocity>::operator(): hydrodynamicprob.hpp:38-66 */
static double prob_hydrodynamic(const sd_t* d1, const sd_t* d2, double eff, double DELT,
                                double VOLUME) {
  const double prob_jk_const = PI * R0 * R0 * W0;
  const double DELT_DELVOL = DELT / VOLUME;
  const double sumr = d1->r + d2->r;
  const double sumrsqrd = sumr * sumr;
  const double vdiff = fabs(tv_simmel(d1->r) - tv_simmel(d2->r));
  const double hydro_kernel = prob_jk_const * eff * sumrsqrd * vdiff;
  return hydro_kernel * DELT_DELVOL;
}
/* ConstProb: constprob.hpp:34-49 */
static double prob_const(double kernel, double DELT, double VOLUME) {
  return kernel * DELT / VOLUME;
}
static double pair_prob(const cleo_b200_params* p, const sd_t* d1, const sd_t* d2, double VOLUME) {
  switch (p->coll_prob) {
    case CLEO_PROB_GOLOVIN: return prob_golovin(d1, d2, p->coll_delt, VOLUME);
    case CLEO_PROB_LONG:
      /* LongHydroProb::operator(), longhydroprob.hpp:61-65 */
      return prob_hydrodynamic(d1, d2, long_kerneleff(d1, d2, p->coaleff), p->coll_delt, VOLUME);
    default: return prob_const(p->const_kernel, p->coll_delt, VOLUME);
  }
}

/* ------------------------------------------------------------------------------------------ */
/* collision kinetics: collisionkinetics.{hpp:71-93, cpp:31-67}                               */
/* ------------------------------------------------------------------------------------------ */
static double collision_kinetic_energy(double r1, double r2, double tv1, double tv2) {
  const double R0cubed = R0 * R0 * R0;
  const double ckeconst = R0cubed * 2.0 / 3.0 * DC_RHO_L * PI * W0 * W0;
  const double r1cubed = r1 * r1 * r1;
  const double r1_r2cubed = (r1 / r2) * (r1 / r2) * (r1 / r2);
  const double rratio = r1cubed / (1 + r1_r2cubed);
  const double vdiff = tv1 - tv2;
  return ckeconst * rratio * vdiff * vdiff;
}
static double coal_surfenergy(double r1, double r2) {
  const double r1cubed = r1 * r1 * r1;
  const double r2cubed = r2 * r2 * r2;
  const double rcubedsum = r1cubed + r2cubed;
  return surfconst * pow(rcubedsum, 2.0 / 3.0);
}
static double surfenergy(double radius) {
  const double rsqrd = radius * radius;
  return surfconst * rsqrd;
}
/* coalescence_efficiency_straub2010: coalescence_efficiency.cpp:27-38 */
static double ecoal_straub2010(const sd_t* d1, const sd_t* d2, double cke) {
  const double beta = -1.15;
  const double surf_c = coal_surfenergy(d1->r, d2->r);
  const double weber = cke / surf_c;
  return exp(beta * weber);
}
/* NFragments: breakup_nfrags.hpp:40-92 */
static double nfrags_of(const cleo_b200_params* p, const sd_t* d1, const sd_t* d2) {
  if (p->nfrags_kind == CLEO_NFRAGS_CONST) return p->nfrags;
  const double alpha = 1.5;
  const double beta = 0.135;
  const double ckemax = 16.49789599 / 1000000;
  const double epsilon = 11.0 / 6.0;
  const double cke = collision_kinetic_energy(d1->r, d2->r, terminalv(p->nfrags_tv, d1->r),
                                              terminalv(p->nfrags_tv, d2->r));
  const double cke_cap = fmin(ckemax, cke);
  const double gamma = pow(cke_cap * 1e6, beta);
  return 1.0 / (alpha - gamma) + epsilon;
}
/* CoalBuReFlag models: coalbure_flag.hpp:42-198 */
static unsigned coalbure_flag(const cleo_b200_params* p, double phi, const sd_t* d1,
                              const sd_t* d2) {
  const double r1 = d1->r, r2 = d2->r;
  switch (p->flag_kind) {
    case CLEO_FLAG_STRAUB: { /* StraubCoalBuReFlag: coalbure_flag.hpp:162-176 */
      const double cke = collision_kinetic_energy(r1, r2, terminalv(p->flag_tv, r1),
                                                  terminalv(p->flag_tv, r2));
      const double ecoal = ecoal_straub2010(d1, d2, cke);
      return (phi < ecoal) ? 1u : 2u;
    }
    case CLEO_FLAG_TESTIKSTRAUB: { /* TSCoalBuReFlag: coalbure_flag.hpp:87-145 */
      const double cke = collision_kinetic_energy(r1, r2, terminalv(p->flag_tv, r1),
                                                  terminalv(p->flag_tv, r2));
      if (cke < surfenergy(fmin(r1, r2))) {
        return (phi < ecoal_straub2010(d1, d2, cke)) ? 1u : 0u;
      } else if (cke < surfenergy(fmax(r1, r2))) {
        return (phi < ecoal_straub2010(d1, d2, cke)) ? 1u : 2u;
      } else {
        return 2u;
      }
    }
    case CLEO_FLAG_SZAKALLURBICH: { /* SUCoalBuReFlag: coalbure_flag.hpp:53-77 */
      const double cke = collision_kinetic_energy(r1, r2, terminalv(p->flag_tv, r1),
                                                  terminalv(p->flag_tv, r2));
      if (cke < surfenergy(fmin(r1, r2))) {
        return 0u;
      } else if (cke < coal_surfenergy(r1, r2)) {
        return 1u;
      } else {
        return 2u;
      }
    }
    default: /* ConstCoalBuReFlag: coalbure_flag.hpp:190-197 */
      return (phi < p->flag_coaleff) ? 1u : 2u;
  }
}

/* ------------------------------------------------------------------------------------------ */
/* coalescence: coalescence.cpp:39-196                                                        */
/* ------------------------------------------------------------------------------------------ */
/* coalescence_gamma: coalescence.cpp:68-79 (same as DoCoalBuRe::collision_gamma, coalbure.hpp:73-84) */
static uint64_t coalescence_gamma(uint64_t xi1, uint64_t xi2, double prob, double phi) {
  uint64_t gamma = (uint64_t)floor(prob);
  if (phi < (prob - (double)gamma)) {
    ++gamma;
  }
  const uint64_t maxgamma = xi1 / xi2;
  return (uint64_t)fmin((double)gamma, (double)maxgamma);
}
/* twin_superdroplet_coalescence: coalescence.cpp:131-162 */
static void twin_coalescence(uint64_t gamma, sd_t* d1, sd_t* d2) {
  if (d1->xi != gamma * d2->xi) set_error(CLEO_ERR_COALESCENCE, g_cur_gbx, g_cur_sd);
  const uint64_t old_xi = d2->xi;
  const uint64_t new_xi = old_xi / 2;
  if (new_xi >= old_xi) set_error(CLEO_ERR_COALESCENCE, g_cur_gbx, g_cur_sd);
  const double new_rcubed = rcubed(d2->r) + (double)gamma * rcubed(d1->r);
  const double new_r = pow(new_rcubed, (1.0 / 3.0));
  const double new_msol = d2->msol + (double)gamma * d1->msol;
  if (new_xi == 0) {
    set_null(d1);
  } else {
    set_xi(d1, new_xi);
  }
  set_xi(d2, old_xi - new_xi);
  set_radius(d1, new_r);
  set_radius(d2, new_r);
  d1->msol = new_msol;
  d2->msol = new_msol;
}
/* different_superdroplet_coalescence: coalescence.cpp:177-196 */
static void different_coalescence(uint64_t gamma, sd_t* d1, sd_t* d2) {
  if (d1->xi <= gamma * d2->xi) set_error(CLEO_ERR_COALESCENCE, g_cur_gbx, g_cur_sd);
  const uint64_t new_xi = d1->xi - gamma * d2->xi;
  if (new_xi >= d1->xi) set_error(CLEO_ERR_COALESCENCE, g_cur_gbx, g_cur_sd);
  set_xi(d1, new_xi);
  const double new_rcubed = rcubed(d2->r) + (double)gamma * rcubed(d1->r);
  set_radius(d2, pow(new_rcubed, (1.0 / 3.0)));
  d2->msol = d2->msol + (double)gamma * d1->msol;
}
/* coalesce_superdroplet_pair: coalescence.cpp:92-113 */
static size_t coalesce_pair(uint64_t gamma, sd_t* d1, sd_t* d2) {
  const uint64_t xi1 = d1->xi;
  const uint64_t xi2 = d2->xi;
  if (xi1 - gamma * xi2 > 0) {
    different_coalescence(gamma, d1, d2);
    return 0;
  } else if (xi1 - gamma * xi2 == 0) {
    twin_coalescence(gamma, d1, d2);
    return (size_t)(d1->xi == 0);
  }
  return 0;
}

/* ------------------------------------------------------------------------------------------ */
/* breakup: breakup.hpp:140-268                                                               */
/* ------------------------------------------------------------------------------------------ */
/* twin_superdroplet_breakup: breakup.hpp:193-228 */
static void twin_breakup(const cleo_b200_params* p, sd_t* d1, sd_t* d2) {
  const uint64_t old_xi = d2->xi;
  const double totnfrags = nfrags_of(p, d1, d2) * (double)old_xi;
  if ((totnfrags / (double)old_xi) <= 2.5) set_error(CLEO_ERR_BREAKUP, g_cur_gbx, g_cur_sd);
  const uint64_t new_xi1 = (uint64_t)round(totnfrags / 2);
  const uint64_t new_xi2 = (uint64_t)round(totnfrags - (double)new_xi1);
  const uint64_t new_xitot = new_xi1 + new_xi2;
  if (new_xi2 <= old_xi) set_error(CLEO_ERR_BREAKUP, g_cur_gbx, g_cur_sd);
  if (new_xitot <= (old_xi * 2)) set_error(CLEO_ERR_BREAKUP, g_cur_gbx, g_cur_sd);
  const double sum_rcubed = rcubed(d1->r) + rcubed(d2->r);
  const double new_rcubed = sum_rcubed * (double)old_xi / (double)new_xitot;
  const double new_r = pow(new_rcubed, (1.0 / 3.0));
  const double sum_msol = d1->msol + d2->msol;
  const double new_msol = sum_msol * (double)old_xi / (double)new_xitot;
  set_xi(d1, new_xi1);
  set_xi(d2, new_xi2);
  set_radius(d1, new_r);
  set_radius(d2, new_r);
  d1->msol = new_msol;
  d2->msol = new_msol;
}
/* different_superdroplet_breakup: breakup.hpp:235-268 */
static void different_breakup(const cleo_b200_params* p, sd_t* d1, sd_t* d2) {
  const uint64_t old_xi1 = d1->xi;
  const uint64_t old_xi2 = d2->xi;
  const uint64_t new_xi1 = old_xi1 - old_xi2;
  set_xi(d1, new_xi1);
  const double totnfrags = nfrags_of(p, d1, d2) * (double)old_xi2;
  const uint64_t new_xi2 = (uint64_t)round(totnfrags);
  if ((totnfrags / (double)old_xi2) <= 2.5) set_error(CLEO_ERR_BREAKUP, g_cur_gbx, g_cur_sd);
  if (new_xi2 <= old_xi2) set_error(CLEO_ERR_BREAKUP, g_cur_gbx, g_cur_sd);
  if ((new_xi1 + new_xi2) <= (old_xi1 + old_xi2)) set_error(CLEO_ERR_BREAKUP, g_cur_gbx, g_cur_sd);
  const double sum_rcubed = rcubed(d1->r) + rcubed(d2->r);
  const double new_rcubed = sum_rcubed * (double)old_xi2 / (double)new_xi2;
  const double new_r = pow(new_rcubed, (1.0 / 3.0));
  const double sum_msol = d1->msol + d2->msol;
  const double new_msol = sum_msol * (double)old_xi2 / (double)new_xi2;
  set_xi(d2, new_xi2);
  set_radius(d2, new_r);
  d2->msol = new_msol;
}
/* breakup_superdroplet_pair: breakup.hpp:176-186 */
static size_t breakup_pair(const cleo_b200_params* p, sd_t* d1, sd_t* d2) {
  if (d1->xi == d2->xi) {
    twin_breakup(p, d1, d2);
  } else {
    different_breakup(p, d1, d2);
  }
  return 0;
}

/* ------------------------------------------------------------------------------------------ */
/* pair enactment: coalescence.cpp:39-54, breakup.hpp:140-166, coalbure.hpp:207-256            */
/* ------------------------------------------------------------------------------------------ */
static size_t enact_collision(const cleo_b200_params* p, sd_t* d1, sd_t* d2, double prob,
                              double phi_coll, double phi_out) {
  switch (p->coll_enact) {
    case CLEO_ENACT_COALESCENCE: {
      const uint64_t gamma = coalescence_gamma(d1->xi, d2->xi, prob, phi_coll);
      if (gamma != 0) return coalesce_pair(gamma, d1, d2);
      return 0;
    }
    case CLEO_ENACT_BREAKUP: { /* breakup_gamma: breakup.hpp:158-166 */
      if (phi_coll < (prob - floor(prob))) return breakup_pair(p, d1, d2);
      return 0;
    }
    default: {
      const uint64_t gamma = coalescence_gamma(d1->xi, d2->xi, prob, phi_coll);
      if (gamma != 0) { /* coalesce_breakup_or_rebound: coalbure.hpp:240-256 */
        const unsigned flag = coalbure_flag(p, phi_out, d1, d2);
        if (flag == 1u) return coalesce_pair(gamma, d1, d2);
        if (flag == 2u) return breakup_pair(p, d1, d2);
      }
      return 0;
    }
  }
}

/* ------------------------------------------------------------------------------------------ */
/* DoCollisions: collisions.hpp:74-327, shuffle.cpp:38-53, shuffle.hpp:80-87                  */
/* ------------------------------------------------------------------------------------------ */
/* Collide the n superdroplets of one gridbox; returns the number of superdroplets left. Draws
 * come from the injected stream at slots starting at *slot. */
static size_t do_collisions(const cleo_b200_params* p, sd_t* supers, size_t nsupers, double volume,
                            uint64_t key, uint64_t* slot, uint32_t gbx, size_t sd_base) {
  /* shuffle_supers / fisher_yates_shuffle: shuffle.cpp:38-53, shuffle.hpp:80-87 */
  if (nsupers >= 2) {
    for (size_t iter = nsupers - 1; iter > 0; --iter) {
      const uint64_t u = cleo_rng_u64(key, (*slot)++);
      const uint64_t randiter = cleo_rng_range(u, 0, (uint64_t)iter + 1);
      const sd_t c = supers[iter];
      supers[iter] = supers[randiter];
      supers[randiter] = c;
    }
  }
  /* collide_supers: collisions.hpp:215-229 */
  const size_t npairs = nsupers / 2;
  const double scale_p = (double)nsupers * ((double)nsupers - 1.0) / (2.0 * (double)npairs);
  const double VOLUME = volume * VOL0;
  size_t oob_nsupers = 0;
  for (size_t jj = 0; jj < npairs; ++jj) {
    sd_t* dA = &supers[2 * jj];
    sd_t* dB = &supers[2 * jj + 1];
    g_cur_gbx = gbx;
    g_cur_sd = sd_base + 2 * jj;
    /* assign_drops: collisions.hpp:94-101 */
    sd_t* d1 = dA;
    sd_t* d2 = dB;
    if (dA->xi < dB->xi) {
      d1 = dB;
      d2 = dA;
    }
    /* scaled_probability: collisions.hpp:117-126 */
    const double prob_jk = pair_prob(p, d1, d2, VOLUME);
    const double large_xi = (double)d1->xi;
    const double prob = scale_p * large_xi * prob_jk;
    /* draws: collisions.hpp:152-155 */
    const double phi_coll = cleo_rng_to_unit(cleo_rng_u64(key, (*slot)++));
    const double phi_out = cleo_rng_to_unit(cleo_rng_u64(key, (*slot)++));
    oob_nsupers += enact_collision(p, d1, d2, prob, phi_coll, phi_out);
  }
  if (oob_nsupers == 0) return nsupers;
  /* remove_null_supers: collisions.hpp:240-248, a stable sort by sdgbxindex of the gridbox's
   * subview; null superdroplets (sdgbxindex = oob) move to the end. */
  size_t w = 0;
  sd_t* nulls = (sd_t*)malloc(sizeof(sd_t) * oob_nsupers);
  size_t nn = 0;
  for (size_t k = 0; k < nsupers; ++k) {
    if (supers[k].gbx == OOB) {
      nulls[nn++] = supers[k];
    } else {
      supers[w++] = supers[k];
    }
  }
  memcpy(&supers[w], nulls, sizeof(sd_t) * nn);
  free(nulls);
  return nsupers - oob_nsupers;
}

/* ------------------------------------------------------------------------------------------ */
/* thermodynamic equations: thermodynamic_equations.{hpp:44-107, cpp:38-145}                  */
/* ------------------------------------------------------------------------------------------ */
static double dry_air_density(double press, double temp, double qvap) {
  const double rgas_equiv = Rgas_dry + Rgas_v * qvap;
  return press / (rgas_equiv * temp);
}
static double moist_specifc_heat(double qvap, double qcond) {
  return Cp_dry + Cp_v * (qvap) + C_l * (qcond);
}
static double supersaturation_ratio(double press, double qvap, double psat) {
  return (press * qvap) / ((Mr_ratio + qvap) * psat);
}
static double saturation_pressure(double temp) {
  if (temp <= 0) set_error(CLEO_ERR_TEMPERATURE, g_cur_gbx, g_cur_sd);
  const double A = 17.4146;
  const double B = 33.639;
  const double TREF = 273.16;
  const double PREF = 611.655;
  const double T = temp * TEMP0;
  return (PREF * exp(A * (T - TREF) / (T - B))) / P0;
}
static double diffusion_factor(double press, double temp, double psat) {
  const double A = 7.11756e-5;
  const double B = 4.38127686e-3;
  const double LATENT_RGAS_V = DC_LATENT_V / DC_RGAS_V;
  const double D = 4.012182971e-5;
  const double TEMP = temp * TEMP0;
  const double PRESS = press * P0;
  const double PSAT = psat * P0;
  const double THERMK = A * pow(TEMP, 2.0) + TEMP * B;
  const double DIFFUSE_V = (D / PRESS * pow(TEMP, 1.94)) / DC_RGAS_V;
  const double fkl = (LATENT_RGAS_V / TEMP - 1.0) * DC_LATENT_V / (THERMK * F0);
  const double fdl = TEMP / (DIFFUSE_V * PSAT) / F0;
  return Rho_l * (fkl + fdl);
}
static double ventilation_factor(double radius) {
  const double vent_factor_max = 20;
  const double C1 = 6.954e+7;
  const double A = 1.963;
  const double C2 = 1.069e+3;
  const double B = 0.702;
  const double a = 1.0 / (C1 * pow(radius * R0, A));
  const double b = 1.0 / (C2 * pow(radius * R0, B));
  const double vent_factor = 1.0 + 1.0 / (a + b);
  return fmin(vent_factor, vent_factor_max);
}
/* kohler_factors: thermodynamic_equations.hpp:95-107 */
static void kohler_factors(double msol, double temp, double* akoh, double* bkoh) {
  const double akoh_constant = 3.3e-7 / (TEMP0 * R0);
  *akoh = akoh_constant / temp;
  const double bkoh_constant = 4.3e-6 * RHO0 / MR0;
  *bkoh = bkoh_constant * msol * IONIC / Mr_sol;
}

/* ------------------------------------------------------------------------------------------ */
/* ImplicitEuler / ImplicitIterations: impliciteuler.{hpp:41-345, cpp:35-301}                 */
/* ------------------------------------------------------------------------------------------ */
typedef struct {
  double s_ratio, akoh, bkoh, ffactor_fv;
} odeconsts_t;
typedef struct {
  size_t maxniters;
  double rtol, atol;
} implit_t;

/* ode_gfunc: impliciteuler.cpp:270-281 */
static double ode_gfunc(const odeconsts_t* o, double subdelt, double rprev, double rsqrd) {
  const double radius = sqrt(rsqrd);
  const double alpha = o->s_ratio - 1 - o->akoh / radius + o->bkoh / pow(radius, 3.0);
  const double beta = 2.0 * subdelt / (rsqrd * o->ffactor_fv);
  const double gamma = pow(rprev / radius, 2.0);
  return 1 - gamma - alpha * beta;
}
/* ode_gfuncderivative: impliciteuler.cpp:291-301 */
static double ode_gfuncderivative(const odeconsts_t* o, double subdelt, double rsqrd) {
  const double radius = sqrt(rsqrd);
  const double alpha = o->akoh / radius - 3.0 * o->bkoh / pow(radius, 3.0);
  const double beta = subdelt / (rsqrd * o->ffactor_fv);
  return 1 - alpha * beta;
}
/* check_for_convergence: impliciteuler.hpp:213-219 */
static int check_for_convergence(const implit_t* it, double gfunciter, double gfuncprev) {
  const double converged = it->rtol * fabs(gfunciter) + it->atol;
  const double currentvalue = fabs(gfunciter - gfuncprev);
  return (currentvalue < converged);
}
/* iterate_rootfinding_algorithm: impliciteuler.cpp:239-255 */
static double iterate_rootfinding(const implit_t* it, const odeconsts_t* o, double subdelt,
                                  double rprev, double ziter, int* is_converged) {
  const double numerator = ode_gfunc(o, subdelt, rprev, ziter);
  const double denominator = ode_gfuncderivative(o, subdelt, ziter);
  ziter = ziter * (1 - numerator / denominator);
  ziter = fmax(ziter, 1e-8);
  const double newnumerator = ode_gfunc(o, subdelt, rprev, ziter);
  *is_converged = check_for_convergence(it, newnumerator, numerator);
  if (g_iters) ++(*g_iters);
  return ziter;
}
/* newtonraphson_niterations: impliciteuler.cpp:181-194 */
static double nr_niterations(const implit_t* it, const odeconsts_t* o, double subdelt,
                             double rprev, double ziter, size_t niters, int* is_converged) {
  *is_converged = 0;
  for (size_t iter = 0; iter < niters; ++iter) {
    ziter = iterate_rootfinding(it, o, subdelt, rprev, ziter, is_converged);
  }
  return ziter;
}
/* newtonraphson_untilconverged: impliciteuler.cpp:207-227 */
static double nr_untilconverged(const implit_t* it, const odeconsts_t* o, size_t niterslimit,
                                double subdelt, double rprev, double ziter, int* failed) {
  int is_converged = 0;
  size_t niter = 1;
  while (!is_converged) {
    if (niter > niterslimit) {
      if (failed)
        *failed = 1; /* a seeded attempt: the caller restarts from the reference guess */
      else
        set_error(CLEO_ERR_NR_NOCONVERGE, g_cur_gbx, g_cur_sd);
      break;
    }
    ziter = iterate_rootfinding(it, o, subdelt, rprev, ziter, &is_converged);
    niter += 1;
  }
  return ziter;
}
/* integrate_condensation_ode: impliciteuler.cpp:128-141 */
static double integrate_ode_ex(const implit_t* it, const odeconsts_t* o, double subdelt,
                               double rprev, double ziter, int* failed) {
  const size_t niters = 2;
  int conv = 0;
  const double res = nr_niterations(it, o, subdelt, rprev, ziter, niters, &conv);
  if (conv) {
    return res;
  } else {
    return nr_untilconverged(it, o, it->maxniters, subdelt, rprev, ziter, failed);
  }
}
static double integrate_condensation_ode(const implit_t* it, const odeconsts_t* o, double subdelt,
                                         double rprev, double ziter) {
  return integrate_ode_ex(it, o, subdelt, rprev, ziter, NULL);
}
/* initialguess: impliciteuler.cpp:156-170 */
static double initialguess(const odeconsts_t* o, double rprev) {
  const double s_act = 1 + sqrt(4.0 * pow(o->akoh, 3.0) / 27 / o->bkoh);
  if (o->s_ratio > s_act) {
    const double bigr = 1e-3 / R0;
    const double maxradius = fmax(bigr, rprev);
    return maxradius * maxradius;
  }
  return rprev * rprev;
}
/* first_unique_criteria: impliciteuler.cpp:69-83 */
static int first_unique_criteria(const odeconsts_t* o, double rprev, double ziter) {
  const double akoh = o->akoh;
  const double bkoh = o->bkoh;
  const double rcritsqrd = 3.0 * bkoh / akoh;
  const int is_ziter_unactivated = ziter < rcritsqrd;
  const int is_unactivated = (rprev * rprev < rcritsqrd && is_ziter_unactivated);
  const double sqrdval = 4.0 * akoh * akoh * akoh / 27.0 / bkoh;
  const int is_subactivated_saturation = (o->s_ratio <= 1.0 + pow(sqrdval, 0.5));
  return (is_unactivated && is_subactivated_saturation);
}
/* critial_timestep: impliciteuler.hpp:266-269 */
static double critical_timestep(const odeconsts_t* o) {
  const double cuberoot = pow(5.0 * o->bkoh / o->akoh, 1.5);
  return 2.5 * o->ffactor_fv / o->akoh * cuberoot;
}
/* solve_with_adaptive_subtimestepping: impliciteuler.cpp:98-113 */
static double solve_substepping(const implit_t* it, const odeconsts_t* o, double delt,
                                double minsubdelt, double rprev, double ziter) {
  const double critdelt = critical_timestep(o);
  const double mindelt = fmax(critdelt, minsubdelt);
  double remdelt = delt;
  while (remdelt > 0.0) {
    const double subdelt = fmin(mindelt, remdelt);
    ziter = integrate_condensation_ode(it, o, subdelt, rprev, ziter);
    rprev = pow(ziter, 0.5);
    remdelt -= subdelt;
  }
  return ziter;
}
/* solve_condensation: impliciteuler.cpp:35-54. A finite positive seed_rsqrd starts the Newton
 * iteration of the direct branch (not the branch decision) instead of the reference initial
 * guess; a seeded iteration that does not converge within maxniters restarts from that guess. */
static double solve_condensation(const implit_t* it, double delt, double minsubdelt,
                                 double s_ratio, double akoh, double bkoh, double ffactor,
                                 double rprev, double seed_rsqrd) {
  const double ffactor_fv = ffactor / ventilation_factor(rprev);
  const odeconsts_t o = {s_ratio, akoh, bkoh, ffactor_fv};
  double ziter = initialguess(&o, rprev);
  const int ucrit1 = first_unique_criteria(&o, rprev, ziter);
  const int ucrit2 = (delt <= critical_timestep(&o)); /* second_unique_criteria, impliciteuler.hpp:283-286 */
  double rsqrd = 0.0;
  if (ucrit1 || ucrit2) {
    /* a seed with a smaller residual than the reference guess starts the iteration; its root is
     * kept when it is the reference's root: unique when delt <= critical timestep, else (an
     * unactivated droplet) only in (0, 3b/a] where z g(z) increases */
    if (seed_rsqrd > 0.0 && seed_rsqrd <= DBL_MAX &&
        fabs(ode_gfunc(&o, delt, rprev, seed_rsqrd)) < fabs(ode_gfunc(&o, delt, rprev, ziter))) {
      /* Newton from the seed with the convergence test after every iteration, at most 6 */
      int conv = 0;
      double z = seed_rsqrd;
      for (int k = 0; k < 6 && !conv; ++k) z = iterate_rootfinding(it, &o, delt, rprev, z, &conv);
      if (conv && (!ucrit1 || z <= 3.0 * bkoh / akoh)) return sqrt(z);
    }
    rsqrd = integrate_condensation_ode(it, &o, delt, rprev, ziter);
  } else {
    rsqrd = solve_substepping(it, &o, delt, minsubdelt, rprev, ziter);
  }
  return sqrt(rsqrd);
}

/* ------------------------------------------------------------------------------------------ */
/* DoCondensation: condensation.cpp:43-138                                                    */
/* ------------------------------------------------------------------------------------------ */
static double do_condensation(oc_ctx* c, uint32_t g, sd_t* supers, size_t nsupers, size_t sd_base) {
  const cleo_b200_params* p = &c->p;
  const implit_t it = {p->maxniters, p->rtol, p->atol};
  g_cur_gbx = g;
  g_cur_sd = sd_base;
  /* superdroplets_change: condensation.cpp:43-59 */
  const double psat = saturation_pressure(c->temp[g]);
  const double s_ratio = supersaturation_ratio(c->press[g], c->qvap[g], psat);
  const double ffactor = diffusion_factor(c->press[g], c->temp[g], psat);
  double totmass_condensed = 0.0;
  g_iters = &c->nr_iters[g];
  for (size_t kk = 0; kk < nsupers; ++kk) {
    sd_t* drop = &supers[kk];
    g_cur_sd = sd_base + kk;
    /* superdrop_mass_change: condensation.cpp:98-112 */
    const double old_m_cond = condensate_mass(drop->r, drop->msol);
    double akoh, bkoh;
    kohler_factors(drop->msol, c->temp[g], &akoh, &bkoh);
    const double newr = solve_condensation(&it, p->cond_delt, p->cond_minsubdelt, s_ratio, akoh,
                                           bkoh, ffactor, drop->r, 0.0);
    change_radius(drop, newr);
    const double mass_condensed = (condensate_mass(drop->r, drop->msol) - old_m_cond) * (double)drop->xi;
    totmass_condensed += mass_condensed;
  }
  g_iters = NULL;
  /* effect_on_thermodynamic_state: condensation.cpp:72-80, state_change :126-138 */
  if (p->do_alter_thermo) {
    const double R0cubed_VOL0 = R0 * R0 * R0 / VOL0;
    const double totrho_condensed = totmass_condensed / c->volume[g] * R0cubed_VOL0;
    const double rho_dry = dry_air_density(c->press[g], c->temp[g], c->qvap[g]);
    const double delta_qcond = totrho_condensed / rho_dry;
    c->qvap[g] -= delta_qcond;
    c->qcond[g] += delta_qcond;
    const double delta_temp = (Latent_v / moist_specifc_heat(c->qvap[g], c->qcond[g])) * delta_qcond;
    c->temp[g] += delta_temp;
  }
  /* monitor_condensation (condensation.hpp:149): cumulative budget */
  c->cond_mass[g] += totmass_condensed;
  return totmass_condensed;
}

/* ------------------------------------------------------------------------------------------ */
/* motion: predcorr.{hpp:50-172, cpp:30-42}, predcorrmotion.hpp:40-107, cfl_criteria.hpp,      */
/* cartesianmaps.cpp:93-286, domainboundaries.hpp, doubly_periodic_domain.hpp                  */
/* ------------------------------------------------------------------------------------------ */
typedef struct {
  double lo, hi;
} bounds_t;
static bounds_t b3(const oc_ctx* c, uint32_t i) {
  bounds_t b = {LLIM, ULIM};
  if (i < c->ngbxs) { b.lo = c->b3lo[i]; b.hi = c->b3hi[i]; }
  return b;
}
static bounds_t b1(const oc_ctx* c, uint32_t i) {
  bounds_t b = {LLIM, ULIM};
  if (i < c->ngbxs) { b.lo = c->b1lo[i]; b.hi = c->b1hi[i]; }
  return b;
}
static bounds_t b2(const oc_ctx* c, uint32_t i) {
  bounds_t b = {LLIM, ULIM};
  if (i < c->ngbxs) { b.lo = c->b2lo[i]; b.hi = c->b2hi[i]; }
  return b;
}
static uint32_t nb(const uint32_t* arr, const oc_ctx* c, uint32_t i) {
  return (i < c->ngbxs) ? arr[i] : OOB; /* nullnghbrs(oob) = {oob, oob} */
}
/* interpolation: predcorr.cpp:30-42 */
static double interpolation(bounds_t bounds, double vlo, double vhi, double sdcoord) {
  const double coord = fmin(bounds.hi, fmax(bounds.lo, sdcoord));
  const double alpha = (coord - bounds.lo) / (bounds.hi - bounds.lo);
  return alpha * vhi + (1 - alpha) * vlo;
}
/* beyond_domainboundary: domainboundaries.hpp:34-37 */
static int beyond_domainboundary(uint32_t gbxindex, uint32_t increment, size_t ndim) {
  return (gbxindex / increment) % ndim == 0;
}
/* flag_sdgbxindex: cartesianmaps.cpp:93-107 */
static int flag_sdgbxindex(uint32_t idx, bounds_t bounds, double coord) {
  if (idx == OOB) return 0;
  else if (coord < bounds.lo) return 1;
  else if (coord >= bounds.hi) return 2;
  return 0;
}
/* change_if_coord3nghbr + forwards/backwards: cartesianmaps.cpp:184-213, 264-276 (z finite) */
static uint32_t change_if_coord3nghbr(const oc_ctx* c, uint32_t idx, double* coord3) {
  const int flag = flag_sdgbxindex(idx, b3(c, idx), *coord3);
  if (flag == 1) {
    const uint32_t nghbr = nb(c->back3, c, idx);
    if (beyond_domainboundary(idx, 1u, c->ndims[0])) {
      /* boundarycond_coord3 = coordbeyond_finitedomain: coord unchanged */
    }
    idx = nghbr;
  } else if (flag == 2) {
    const uint32_t nghbr = nb(c->fwd3, c, idx);
    idx = nghbr;
  }
  return idx;
}
/* change_if_coord1nghbr + forwards/backwards: cartesianmaps.cpp:148-179, 243-255 (x periodic) */
static uint32_t change_if_coord1nghbr(const oc_ctx* c, uint32_t idx, double* coord1) {
  const int flag = flag_sdgbxindex(idx, b1(c, idx), *coord1);
  const uint32_t incre = c->ndims[0];
  if (flag == 1) {
    const uint32_t nghbr = nb(c->back1, c, idx);
    if (beyond_domainboundary(idx, incre, c->ndims[1])) {
      const double lim1 = b1(c, nghbr).hi;
      const double lim2 = b1(c, idx).lo;
      *coord1 = *coord1 + lim1 - lim2; /* coordbeyond_periodicdomain, domainboundaries.hpp:106-109 */
    }
    idx = nghbr;
  } else if (flag == 2) {
    const uint32_t nghbr = nb(c->fwd1, c, idx);
    if (beyond_domainboundary(idx + incre, incre, c->ndims[1])) {
      const double lim1 = b1(c, nghbr).lo;
      const double lim2 = b1(c, idx).hi;
      *coord1 = *coord1 + lim1 - lim2;
    }
    idx = nghbr;
  }
  return idx;
}
/* change_if_coord2nghbr + forwards/backwards: cartesianmaps.cpp:112-143, 222-234 (y periodic) */
static uint32_t change_if_coord2nghbr(const oc_ctx* c, uint32_t idx, double* coord2) {
  const int flag = flag_sdgbxindex(idx, b2(c, idx), *coord2);
  const uint32_t incre = c->ndims[0] * c->ndims[1];
  if (flag == 1) {
    const uint32_t nghbr = nb(c->back2, c, idx);
    if (beyond_domainboundary(idx, incre, c->ndims[2])) {
      const double lim1 = b2(c, nghbr).hi;
      const double lim2 = b2(c, idx).lo;
      *coord2 = *coord2 + lim1 - lim2;
    }
    idx = nghbr;
  } else if (flag == 2) {
    const uint32_t nghbr = nb(c->fwd2, c, idx);
    if (beyond_domainboundary(idx + incre, incre, c->ndims[2])) {
      const double lim1 = b2(c, nghbr).lo;
      const double lim2 = b2(c, idx).hi;
      *coord2 = *coord2 + lim1 - lim2;
    }
    idx = nghbr;
  }
  return idx;
}
/* PredCorr::operator() and PredCorrMotion::superdrop_gbx for one superdroplet in gridbox g. */
static void move_superdrop(const oc_ctx* c, uint32_t g, sd_t* drop) {
  const double delt = c->p.motion_delt;
  const bounds_t bz = b3(c, g), bx = b1(c, g), by = b2(c, g);
  /* delta_coord3: predcorr.hpp:83-105 */
  double coord3 = drop->c3;
  const double terminal = terminalv(c->p.motion_tv, drop->r);
  double vel3 = interpolation(bz, c->wlo[g], c->whi[g], coord3);
  vel3 -= terminal;
  coord3 += vel3 * delt;
  double corrvel3 = interpolation(bz, c->wlo[g], c->whi[g], coord3);
  corrvel3 -= terminal;
  const double delta3 = (vel3 + corrvel3) * (delt / 2);
  /* delta_coord1: predcorr.hpp:107-125 */
  double coord1 = drop->c1;
  const double vel1 = interpolation(bx, c->ulo[g], c->uhi[g], coord1);
  coord1 += vel1 * delt;
  const double corrvel1 = interpolation(bx, c->ulo[g], c->uhi[g], coord1);
  const double delta1 = (vel1 + corrvel1) * (delt / 2);
  /* delta_coord2: predcorr.hpp:127-145 */
  double coord2 = drop->c2;
  const double vel2 = interpolation(by, c->vlo[g], c->vhi[g], coord2);
  coord2 += vel2 * delt;
  const double corrvel2 = interpolation(by, c->vlo[g], c->vhi[g], coord2);
  const double delta2 = (vel2 + corrvel2) * (delt / 2);
  /* cfl_criteria: cfl_criteria.hpp:30-57 */
  int cfl = (fabs(delta3) <= fabs(bz.hi - bz.lo));
  cfl = (fabs(delta1) <= fabs(bx.hi - bx.lo)) && cfl;
  cfl = (fabs(delta2) <= fabs(by.hi - by.lo)) && cfl;
  if (!cfl) set_error(CLEO_ERR_CFL, g_cur_gbx, g_cur_sd);
  /* increment_coords: superdrop.hpp */
  drop->c3 += delta3;
  drop->c1 += delta1;
  drop->c2 += delta2;
  /* monitor_precipitation: monitor_precipitation_observer.hpp:97-107 */
  if ((c->p.monitors & CLEO_MONITOR_PRECIPITATION) && drop->c3 < bz.lo) {
    const double m = condensate_mass(drop->r, drop->msol) * (double)drop->xi / Rho_l / c->gbxarea[g];
    c->precip[g] += m;
  }
  /* superdrop_gbx: predcorrmotion.hpp:85-106 -> get_no_decomposition_bounding_gridbox,
   * cartesianmaps.cpp:278-286 */
  double n3 = drop->c3, n1 = drop->c1, n2 = drop->c2;
  uint32_t idx = change_if_coord3nghbr(c, g, &n3);
  idx = change_if_coord1nghbr(c, idx, &n1);
  idx = change_if_coord2nghbr(c, idx, &n2);
  drop->c3 = n3;
  drop->c1 = n1;
  drop->c2 = n2;
  drop->gbx = idx;
  if (idx >= c->ngbxs) return;
  /* CartesianCheckBounds: cartesian_motion.hpp:38-54 */
  const bounds_t nz = b3(c, idx), nx = b1(c, idx), ny = b2(c, idx);
  int bad = (drop->c3 < nz.lo) | (drop->c3 >= nz.hi);
  bad |= (drop->c1 < nx.lo) | (drop->c1 >= nx.hi);
  bad |= (drop->c2 < ny.lo) | (drop->c2 >= ny.hi);
  if (bad) set_error(CLEO_ERR_OUT_OF_BOX, g_cur_gbx, g_cur_sd);
}

/* ------------------------------------------------------------------------------------------ */
/* sorting: sortsupers.hpp:44-226, findrefs.hpp:54-179, supersindomain.hpp:46-92               */
/* ------------------------------------------------------------------------------------------ */
/* Stable counting sort of all superdroplets by sdgbxindex; keys > ngbxs share the last bucket
 * (_get_count_position, sortsupers.hpp:44-48). Equivalent to the Serial execution of
 * create_cumlcounts + counting_sort (the team variant visits gridbox refs in order, which
 * partition the domain, then the out-of-domain tail). Then sets domain and gridbox refs. */
static void sort_and_set_refs(oc_ctx* c) {
  const size_t nb_ = (size_t)c->ngbxs + 1;
  memset(c->counts, 0, sizeof(size_t) * nb_);
  for (size_t k = 0; k < c->ntot; ++k) {
    const uint32_t key = c->sd[k].gbx;
    const size_t pos = !(key <= c->ngbxs) ? (nb_ - 1) : key;
    c->counts[pos]++;
  }
  size_t acc = 0;
  for (size_t b = 0; b < nb_; ++b) {
    const size_t cnt = c->counts[b];
    c->counts[b] = acc;
    acc += cnt;
  }
  for (size_t k = 0; k < c->ntot; ++k) {
    const uint32_t key = c->sd[k].gbx;
    const size_t pos = !(key <= c->ngbxs) ? (nb_ - 1) : key;
    c->tmp[c->counts[pos]++] = c->sd[k];
  }
  sd_t* t = c->sd;
  c->sd = c->tmp;
  c->tmp = t;
  /* find_domainrefs: first superdrop with sdgbxindex > gbxindex_max (= ngbxs) */
  size_t nd = 0;
  while (nd < c->ntot && c->sd[nd].gbx <= c->ngbxs) ++nd;
  c->ndomain = nd;
  /* set_refs for each gridbox: find_refs by partition point (findrefs.hpp:54-61) */
  size_t k = 0;
  for (uint32_t g = 0; g < c->ngbxs; ++g) {
    while (k < nd && c->sd[k].gbx < g) ++k;
    c->refs0[g] = k;
    size_t e = k;
    while (e < nd && c->sd[e].gbx <= g) ++e;
    c->refs1[g] = e;
    k = e;
  }
}

/* effect_on_hydrometeor_states: movesupersindomain.hpp:95-136, 259-267 */
static int effect_on_qcond(oc_ctx* c, uint32_t g, const void* arg) {
  (void)arg;
  double totmass_cond = 0.0;
  for (size_t k = c->refs0[g]; k < c->refs1[g]; ++k) {
    g_cur_gbx = g;
    g_cur_sd = k;
    totmass_cond += condensate_mass(c->sd[k].r, c->sd[k].msol) * (double)c->sd[k].xi;
  }
  const double R0cubed_VOL0 = R0 * R0 * R0 / VOL0;
  const double rho_cond = totmass_cond / c->volume[g] * R0cubed_VOL0;
  const double rho_dry = dry_air_density(c->press[g], c->temp[g], c->qvap[g]);
  c->qcond[g] = rho_cond / rho_dry;
  return 0;
}

/* ------------------------------------------------------------------------------------------ */
/* scheduling: microphysicalprocess.hpp:222-248, predcorrmotion.hpp:52-68                     */
/* ------------------------------------------------------------------------------------------ */
static int on_step(uint32_t interval, uint32_t t) {
  return (t % interval == 0) && (interval != CLEO_STEP_OFF);
}
static uint32_t next_step(uint32_t interval, uint32_t t) {
  if (interval == CLEO_STEP_OFF) return CLEO_STEP_OFF; /* Null processes, microphysicalprocess.hpp:150 */
  return ((t / interval) + 1) * interval;
}

/* ------------------------------------------------------------------------------------------ */
/* the SDM step: sdmmethods.hpp:54-93, 184-230, 319-332; movesupersindomain.hpp:234-301         */
/* ------------------------------------------------------------------------------------------ */
/* ------------------------------------------------------------------------------------------ */
/* SDMMonitor members: monitor_massmoments_change.hpp, monitor_precipitation_observer.hpp     */
/* ------------------------------------------------------------------------------------------ */
/* calculate_massmoments / calculate_rainmassmoments: massmoments_observer.cpp:38-113, the
 * reduction in the superdroplets' order (Kokkos' serial order) */
static void massmoments(const sd_t* supers, size_t n, int rain, uint64_t* m0, float* m1,
                        float* m2) {
  const double rlim = 40e-6 / R0;
  uint64_t a0 = 0;
  float a1 = 0.0f, a2 = 0.0f;
  for (size_t kk = 0; kk < n; ++kk) {
    const sd_t* drop = &supers[kk];
    const int binary = rain ? (drop->r >= rlim) : 1;
    a0 += (uint64_t)(drop->xi * (uint64_t)binary);
    const double mass = sd_mass(drop->r, drop->msol);
    const double xi = (double)drop->xi;
    a1 += (float)(xi * mass * (double)binary);
    a2 += (float)(xi * mass * mass * (double)binary);
  }
  *m0 = a0;
  *m1 = a1;
  *m2 = a2;
}
/* fetch_delta_massmoments: monitor_massmoments_change.hpp:99-121 (which = 0 after microphysics,
 * 1 after motion) */
static void monitor_massmoments(oc_ctx* c, uint32_t g, const sd_t* supers, size_t n, int which) {
  for (int rain = 0; rain < 2; ++rain) {
    if (!(c->p.monitors & (rain ? CLEO_MONITOR_RAINMASSMOMENTS : CLEO_MONITOR_MASSMOMENTS)))
      continue;
    uint64_t m0;
    float m1, m2;
    massmoments(supers, n, rain, &m0, &m1, &m2);
    c->mm0[rain][which][g] += m0 - c->prev0[rain][g];
    c->mm1[rain][which][g] += m1 - c->prev1[rain][g];
    c->mm2[rain][which][g] += m2 - c->prev2[rain][g];
    c->prev0[rain][g] = m0;
    c->prev1[rain][g] = m1;
    c->prev2[rain][g] = m2;
  }
}
/* MonitorMassMomentsChange::monitor_motion :295-305, for gridbox g */
static int monitor_motion(oc_ctx* c, uint32_t g, const void* arg) {
  (void)arg;
  monitor_massmoments(c, g, &c->sd[c->refs0[g]], c->refs1[g] - c->refs0[g], 1);
  return 0;
}

int oc_monitors_begin(oc_ctx* c) { /* before_timestepping: :75-82, reset_monitor */
  for (int rain = 0; rain < 2; ++rain) {
    for (uint32_t g = 0; g < c->ngbxs; ++g) {
      massmoments(&c->sd[c->refs0[g]], c->refs1[g] - c->refs0[g], rain, &c->prev0[rain][g],
                  &c->prev1[rain][g], &c->prev2[rain][g]);
      for (int w = 0; w < 2; ++w) {
        c->mm0[rain][w][g] = 0;
        c->mm1[rain][w][g] = 0.0f;
        c->mm2[rain][w][g] = 0.0f;
      }
    }
  }
  memset(c->precip, 0, sizeof(double) * (c->ngbxs ? c->ngbxs : 1));
  return CLEO_OK;
}

int oc_download_monitors(oc_ctx* c, cleo_b200_monitors* o, int reset) {
  const size_t n = c->ngbxs;
  uint64_t* d0[2][2] = {{o->mom0_micro, o->mom0_motion}, {o->rain_mom0_micro, o->rain_mom0_motion}};
  float* d1[2][2] = {{o->mom1_micro, o->mom1_motion}, {o->rain_mom1_micro, o->rain_mom1_motion}};
  float* d2[2][2] = {{o->mom2_micro, o->mom2_motion}, {o->rain_mom2_micro, o->rain_mom2_motion}};
  for (int r = 0; r < 2; ++r)
    for (int w = 0; w < 2; ++w) {
      if (d0[r][w]) memcpy(d0[r][w], c->mm0[r][w], n * 8);
      if (d1[r][w]) memcpy(d1[r][w], c->mm1[r][w], n * 4);
      if (d2[r][w]) memcpy(d2[r][w], c->mm2[r][w], n * 4);
      if (reset) {
        memset(c->mm0[r][w], 0, n * 8);
        memset(c->mm1[r][w], 0, n * 4);
        memset(c->mm2[r][w], 0, n * 4);
      }
    }
  if (o->precip) memcpy(o->precip, c->precip, n * 8);
  if (reset) memset(c->precip, 0, n * 8);
  return CLEO_OK;
}

/* One step of a loop over all gridboxes (the reference's league of gridbox teams), on
 * g_nthreads threads; returns the OR of f's results. Errors keep the sequential loop's order
 * (merge_error) and never replace one the context already holds. */
typedef int (*gbx_fn)(oc_ctx* c, uint32_t g, const void* arg);
int oc_set_num_threads(int n) {
  g_nthreads = n < 1 ? 1 : n;
  return g_nthreads;
}
static int for_each_gridbox(oc_ctx* c, gbx_fn f, const void* arg) {
  cleo_b200_error first = {CLEO_OK, OOB, 0};
  int any = 0;
  const long ng = (long)c->ngbxs;
#pragma omp parallel num_threads(g_nthreads) if (g_nthreads > 1) reduction(| : any)
  {
    cleo_b200_error mine = {CLEO_OK, OOB, 0};
    g_err = &mine;
#pragma omp for schedule(dynamic, 64)
    for (long g = 0; g < ng; ++g) any |= f(c, (uint32_t)g, arg);
#pragma omp critical(oc_first_error)
    merge_error(&first, &mine);
    g_err = NULL;
  }
  g_err = &c->err;
  if (c->err.code == CLEO_OK && first.code != CLEO_OK) c->err = first;
  return any;
}

/* movesupersindomain.hpp:47-93: every superdroplet of gridbox g moved */
static int move_gridbox(oc_ctx* c, uint32_t g, const void* arg) {
  (void)arg;
  for (size_t k = c->refs0[g]; k < c->refs1[g]; ++k) {
    g_cur_gbx = g;
    g_cur_sd = k;
    move_superdrop(c, g, &c->sd[k]);
  }
  return 0;
}

/* the SDM microphysics of gridbox g between t_sdm and t_sdm_next: run_subtimestepping
 * (sdmmethods.hpp:70-84) with Condensation >> Collisions, then monitor_microphysics
 * (sdmmethods.hpp:76); returns 1 if collisions left null superdroplets */
typedef struct {
  uint32_t t_sdm, t_sdm_next;
} micro_span;
static int micro_gridbox(oc_ctx* c, uint32_t g, const void* arg) {
  const micro_span* sp = (const micro_span*)arg;
  const cleo_b200_params* p = &c->p;
  sd_t* supers = &c->sd[c->refs0[g]];
  size_t n = c->refs1[g] - c->refs0[g];
  const size_t nbefore = n;
  const uint64_t key = cleo_rng_key(p->seed, sp->t_sdm, g);
  uint64_t slot = 0;
  uint32_t subt = sp->t_sdm;
  while (subt < sp->t_sdm_next) {
    if (on_step(p->condstep, subt)) do_condensation(c, g, supers, n, c->refs0[g]);
    if (on_step(p->collstep, subt)) {
      n = do_collisions(p, supers, n, c->volume[g], key, &slot, g, c->refs0[g]);
    }
    const uint32_t a = next_step(p->condstep, subt);
    const uint32_t b = next_step(p->collstep, subt);
    subt = (a < b) ? a : b;
  }
  monitor_massmoments(c, g, supers, n, 0);
  return n != nbefore;
}

int oc_step(oc_ctx* c, uint32_t t_mdl, uint32_t t_next) {
  const cleo_b200_params* p = &c->p;
  g_err = &c->err;
  uint32_t t_sdm = t_mdl;
  while (t_sdm < t_next) {
    /* next_sdmstep: sdmmethods.hpp:131-139 */
    const uint32_t next_move = next_step(p->motionstep, t_sdm);
    const uint32_t t_sdm_next = (t_next < next_move) ? t_next : next_move;

    /* superdrops_movement -> MoveSupersInDomain::run_step (movesupersindomain.hpp:292-301) */
    if (on_step(p->motionstep, t_sdm)) {
      for_each_gridbox(c, move_gridbox, NULL);
      sort_and_set_refs(c); /* CartesianTransportAcrossDomain on 1 process: sort_totsupers */
      for_each_gridbox(c, effect_on_qcond, NULL);
      for_each_gridbox(c, monitor_motion, NULL); /* movesupersindomain.hpp:297 */
    }

    /* sdm_microphysics: sdmmethods.hpp:184-230 */
    const micro_span sp = {t_sdm, t_sdm_next};
    if (for_each_gridbox(c, micro_gridbox, &sp)) sort_and_set_refs(c);

    t_sdm = t_sdm_next;
  }
  g_err = NULL;
  return c->err.code;
}

/* ------------------------------------------------------------------------------------------ */
/* context management                                                                         */
/* ------------------------------------------------------------------------------------------ */
static double* dup_d(const double* src, size_t n) {
  double* d = (double*)malloc(sizeof(double) * (n ? n : 1));
  if (src) memcpy(d, src, sizeof(double) * n);
  else memset(d, 0, sizeof(double) * (n ? n : 1));
  return d;
}
static uint32_t* dup_u(const uint32_t* src, size_t n) {
  uint32_t* d = (uint32_t*)malloc(sizeof(uint32_t) * (n ? n : 1));
  if (src) memcpy(d, src, sizeof(uint32_t) * n);
  return d;
}

int oc_create(const cleo_b200_params* p, const cleo_b200_grid* g, size_t capacity, oc_ctx** out) {
  if (!p || !g || !out) return CLEO_ERR_ARGUMENT;
  if (p->cond_delt < p->cond_minsubdelt && p->condstep != CLEO_STEP_OFF) return CLEO_ERR_SUBDELT;
  oc_ctx* c = (oc_ctx*)calloc(1, sizeof(oc_ctx));
  c->p = *p;
  c->ngbxs = g->ngbxs;
  memcpy(c->ndims, g->ndims, sizeof(c->ndims));
  const size_t n = g->ngbxs;
  c->b3lo = dup_d(g->coord3lo, n); c->b3hi = dup_d(g->coord3hi, n);
  c->b1lo = dup_d(g->coord1lo, n); c->b1hi = dup_d(g->coord1hi, n);
  c->b2lo = dup_d(g->coord2lo, n); c->b2hi = dup_d(g->coord2hi, n);
  c->back3 = dup_u(g->back3, n); c->fwd3 = dup_u(g->fwd3, n);
  c->back1 = dup_u(g->back1, n); c->fwd1 = dup_u(g->fwd1, n);
  c->back2 = dup_u(g->back2, n); c->fwd2 = dup_u(g->fwd2, n);
  c->volume = dup_d(NULL, n); c->press = dup_d(NULL, n); c->temp = dup_d(NULL, n);
  c->qvap = dup_d(NULL, n); c->qcond = dup_d(NULL, n);
  c->wlo = dup_d(NULL, n); c->whi = dup_d(NULL, n); c->ulo = dup_d(NULL, n);
  c->uhi = dup_d(NULL, n); c->vlo = dup_d(NULL, n); c->vhi = dup_d(NULL, n);
  c->cond_mass = dup_d(NULL, n);
  c->nr_iters = (uint64_t*)calloc(n ? n : 1, sizeof(uint64_t));
  c->capacity = capacity;
  c->sd = (sd_t*)calloc(capacity ? capacity : 1, sizeof(sd_t));
  c->tmp = (sd_t*)calloc(capacity ? capacity : 1, sizeof(sd_t));
  c->refs0 = (size_t*)calloc(n ? n : 1, sizeof(size_t));
  c->refs1 = (size_t*)calloc(n ? n : 1, sizeof(size_t));
  c->counts = (size_t*)calloc(n + 1, sizeof(size_t));
  c->gbxarea = (double*)calloc(n ? n : 1, sizeof(double));
  for (size_t i = 0; i < n; ++i)
    c->gbxarea[i] = g->gbxarea ? g->gbxarea[i]
                               : (g->coord1hi[i] - g->coord1lo[i]) * (g->coord2hi[i] - g->coord2lo[i]);
  for (int r = 0; r < 2; ++r) {
    for (int w = 0; w < 2; ++w) {
      c->mm0[r][w] = (uint64_t*)calloc(n ? n : 1, 8);
      c->mm1[r][w] = (float*)calloc(n ? n : 1, 4);
      c->mm2[r][w] = (float*)calloc(n ? n : 1, 4);
    }
    c->prev0[r] = (uint64_t*)calloc(n ? n : 1, 8);
    c->prev1[r] = (float*)calloc(n ? n : 1, 4);
    c->prev2[r] = (float*)calloc(n ? n : 1, 4);
  }
  c->precip = (double*)calloc(n ? n : 1, sizeof(double));
  c->err.code = CLEO_OK;
  c->err.gbxindex = OOB;
  *out = c;
  return CLEO_OK;
}

void oc_destroy(oc_ctx* c) {
  if (!c) return;
  double* dd[] = {c->b3lo, c->b3hi, c->b1lo, c->b1hi, c->b2lo, c->b2hi, c->volume, c->press,
                  c->temp, c->qvap, c->qcond, c->wlo, c->whi, c->ulo, c->uhi, c->vlo, c->vhi,
                  c->cond_mass};
  for (size_t i = 0; i < sizeof(dd) / sizeof(dd[0]); ++i) free(dd[i]);
  uint32_t* uu[] = {c->back3, c->fwd3, c->back1, c->fwd1, c->back2, c->fwd2};
  for (size_t i = 0; i < sizeof(uu) / sizeof(uu[0]); ++i) free(uu[i]);
  free(c->nr_iters); free(c->sd); free(c->tmp); free(c->refs0); free(c->refs1); free(c->counts);
  free(c->gbxarea); free(c->precip);
  for (int r = 0; r < 2; ++r) {
    for (int w = 0; w < 2; ++w) {
      free(c->mm0[r][w]); free(c->mm1[r][w]); free(c->mm2[r][w]);
    }
    free(c->prev0[r]); free(c->prev1[r]); free(c->prev2[r]);
  }
  free(c);
}

int oc_upload_supers(oc_ctx* c, const cleo_b200_supers* h, size_t n) {
  if (n > c->capacity) return CLEO_ERR_CAPACITY;
  for (size_t k = 0; k < n; ++k) {
    sd_t* d = &c->sd[k];
    d->gbx = h->sdgbxindex[k];
    d->c3 = h->coord3[k]; d->c1 = h->coord1[k]; d->c2 = h->coord2[k];
    d->xi = h->xi[k]; d->r = h->radius[k]; d->msol = h->msol[k];
    d->id = h->sdid ? h->sdid[k] : k;
  }
  c->ntot = n;
  sort_and_set_refs(c); /* SupersInDomain ctor: supersindomain.hpp:55-62 */
  return CLEO_OK;
}

int oc_upload_state(oc_ctx* c, const cleo_b200_gbx_state* h) {
  const size_t n = c->ngbxs;
  memcpy(c->volume, h->volume, n * 8); memcpy(c->press, h->press, n * 8);
  memcpy(c->temp, h->temp, n * 8); memcpy(c->qvap, h->qvap, n * 8);
  memcpy(c->qcond, h->qcond, n * 8);
  memcpy(c->wlo, h->wvel_lo, n * 8); memcpy(c->whi, h->wvel_hi, n * 8);
  memcpy(c->ulo, h->uvel_lo, n * 8); memcpy(c->uhi, h->uvel_hi, n * 8);
  memcpy(c->vlo, h->vvel_lo, n * 8); memcpy(c->vhi, h->vvel_hi, n * 8);
  return CLEO_OK;
}

int oc_status(oc_ctx* c, cleo_b200_error* err) {
  if (err) *err = c->err;
  return c->err.code;
}

int oc_download_supers(oc_ctx* c, cleo_b200_supers* h, size_t* n_domain, size_t* n_total) {
  for (size_t k = 0; k < c->ntot; ++k) {
    const sd_t* d = &c->sd[k];
    h->sdgbxindex[k] = d->gbx;
    h->coord3[k] = d->c3; h->coord1[k] = d->c1; h->coord2[k] = d->c2;
    h->xi[k] = d->xi; h->radius[k] = d->r; h->msol[k] = d->msol;
    if (h->sdid) h->sdid[k] = d->id;
  }
  if (n_domain) *n_domain = c->ndomain;
  if (n_total) *n_total = c->ntot;
  return CLEO_OK;
}

int oc_download_state(oc_ctx* c, cleo_b200_gbx_state* h) {
  const size_t n = c->ngbxs;
  memcpy(h->volume, c->volume, n * 8); memcpy(h->press, c->press, n * 8);
  memcpy(h->temp, c->temp, n * 8); memcpy(h->qvap, c->qvap, n * 8);
  memcpy(h->qcond, c->qcond, n * 8);
  memcpy(h->wvel_lo, c->wlo, n * 8); memcpy(h->wvel_hi, c->whi, n * 8);
  memcpy(h->uvel_lo, c->ulo, n * 8); memcpy(h->uvel_hi, c->uhi, n * 8);
  memcpy(h->vvel_lo, c->vlo, n * 8); memcpy(h->vvel_hi, c->vhi, n * 8);
  return CLEO_OK;
}

int oc_download_budgets(oc_ctx* c, double* cond_mass, uint64_t* nr_iters) {
  if (cond_mass) memcpy(cond_mass, c->cond_mass, sizeof(double) * c->ngbxs);
  if (nr_iters) memcpy(nr_iters, c->nr_iters, sizeof(uint64_t) * c->ngbxs);
  return CLEO_OK;
}

/* ------------------------------------------------------------------------------------------ */
/* batch condensation solves (independent droplets; superdrop_mass_change without the xi sum)  */
/* ------------------------------------------------------------------------------------------ */
static int solve_batch(const cleo_b200_params* p, size_t n, const double* radius,
                       const double* msol, const double* temp, const double* press,
                       const double* s_ratio, const double* delt, const double* seed,
                       double* radius_out, uint32_t* niters_out) {
  const implit_t it = {p->maxniters, p->rtol, p->atol};
  cleo_b200_error first = {CLEO_OK, OOB, 0};
  const long nn = (long)n;
  /* droplets are independent: any number of threads, the first error by droplet index */
#pragma omp parallel num_threads(g_nthreads) if (g_nthreads > 1)
  {
    cleo_b200_error mine = {CLEO_OK, OOB, 0};
    g_err = &mine;
#pragma omp for schedule(dynamic, 256)
    for (long ii = 0; ii < nn; ++ii) {
      const size_t i = (size_t)ii;
      uint64_t iters = 0;
      g_iters = &iters;
      g_failed = 0;
      g_cur_gbx = OOB;
      g_cur_sd = i;
      const double psat = saturation_pressure(temp[i]);
      const double ffactor = diffusion_factor(press[i], temp[i], psat);
      double akoh, bkoh;
      kohler_factors(msol[i], temp[i], &akoh, &bkoh);
      sd_t d = {0, 0, 0, 0, 1, radius[i], msol[i], 0};
      const double newr = solve_condensation(&it, delt[i], p->cond_minsubdelt, s_ratio[i], akoh,
                                             bkoh, ffactor, radius[i], seed ? seed[i] : 0.0);
      change_radius(&d, newr);
      radius_out[i] = d.r;
      /* the droplets the reference would abort on are marked (CLEO_NITERS_FAILED) */
      if (niters_out) niters_out[i] = (uint32_t)iters | (g_failed ? CLEO_NITERS_FAILED : 0u);
    }
    g_iters = NULL;
#pragma omp critical(oc_first_error)
    merge_error(&first, &mine);
    g_err = NULL;
  }
  return first.code;
}

int oc_condensation_solve(const cleo_b200_params* p, size_t n, const double* radius,
                          const double* msol, const double* temp, const double* press,
                          const double* s_ratio, const double* delt, double* radius_out,
                          uint32_t* niters_out) {
  return solve_batch(p, n, radius, msol, temp, press, s_ratio, delt, NULL, radius_out, niters_out);
}

int oc_condensation_solve_seeded(const cleo_b200_params* p, size_t n, const double* radius,
                                 const double* msol, const double* temp, const double* press,
                                 const double* s_ratio, const double* delt,
                                 const double* seed_rsqrd, double* radius_out,
                                 uint32_t* niters_out) {
  return solve_batch(p, n, radius, msol, temp, press, s_ratio, delt, seed_rsqrd, radius_out,
                     niters_out);
}

/* ------------------------------------------------------------------------------------------ */
/* unit-check exports                                                                         */
/* ------------------------------------------------------------------------------------------ */
uint64_t oc_rng_u64(uint64_t seed, uint32_t t_sdm, uint32_t gbxindex, uint64_t slot) {
  return cleo_rng_u64(cleo_rng_key(seed, t_sdm, gbxindex), slot);
}
double oc_rng_drand(uint64_t seed, uint32_t t_sdm, uint32_t gbxindex, uint64_t slot) {
  return cleo_rng_to_unit(oc_rng_u64(seed, t_sdm, gbxindex, slot));
}
uint64_t oc_rng_urand(uint64_t seed, uint32_t t_sdm, uint32_t gbxindex, uint64_t slot,
                      uint64_t start, uint64_t end) {
  return cleo_rng_range(oc_rng_u64(seed, t_sdm, gbxindex, slot), start, end);
}
double oc_pair_probability(const cleo_b200_params* p, double r1, uint64_t xi1, double msol1,
                           double r2, uint64_t xi2, double msol2, double volume) {
  const sd_t a = {0, 0, 0, 0, xi1, r1, msol1, 0};
  const sd_t b = {0, 0, 0, 0, xi2, r2, msol2, 0};
  return pair_prob(p, &a, &b, volume * VOL0);
}
