/*
 * cleo_b200.h — C ABI of the B200 super-droplet microphysics hot path.
 *
 * One context owns the device structure-of-arrays (SoA) superdroplet state, the per-gridbox
 * thermodynamic state, the Cartesian gridbox maps and all scratch memory for one domain on one
 * GPU. Every entry point takes plain pointers and sizes; no C++ or torch types cross this
 * boundary. All quantities are CLEO's non-dimensional ones (cleoconstants.hpp:72-102): radii in
 * units of R0 = 1e-6 m, coordinates in COORD0 = 1000 m, volumes in VOL0 = 1e9 m^3, time in
 * TIME0 = 1000 s, pressure in P0, temperature in TEMP0.
 *
 * Reference interfaces replaced (paths relative to the CLEO project root):
 *   cleo_b200_create        ~ SDMMethods ctor + create_supers/create_gbxs
 *                             (libs/runcleo/sdmmethods.hpp:244-250, libs/runcleo/createsupers.hpp:111-138,
 *                              libs/runcleo/creategbxs.hpp:170-351)
 *   cleo_b200_step          ~ SDMMethods::run_step (libs/runcleo/sdmmethods.hpp:319-332), i.e.
 *                             MoveSupersInDomain::run_step (libs/gridboxes/movesupersindomain.hpp:292-301)
 *                             then sdm_microphysics (libs/runcleo/sdmmethods.hpp:184-230) with
 *                             Condensation >> CollCoal/CoalBuRe/CollBu (libs/superdrops/condensation.hpp:242-253,
 *                             libs/superdrops/collisions/coalescence.hpp:133-160,
 *                             libs/superdrops/collisions/coalbure.hpp:156-185, breakup.hpp:97-123)
 *   cleo_b200_upload_* /    ~ the DualView host<->device syncs RunCLEO does around coupling and
 *   cleo_b200_download_*      observation steps (libs/runcleo/runcleo.hpp:163-175)
 *   cleo_b200_status        ~ Kokkos::abort sites of the hot path, reported as status codes
 *   cleo_b200_condensation_solve ~ ImplicitEuler::solve_condensation applied to a batch of
 *                             independent droplets (libs/superdrops/impliciteuler.cpp:35-54)
 *
 * Threading: one context per host thread; calls on a context are serialised on its CUDA stream.
 * Errors: every function returns a cleo_status. Device-side failures (the reference's abort
 * sites) are recorded in a device error word and surface from cleo_b200_status(), which
 * synchronises the context's stream. Kernels never trap.
 */
#ifndef CLEO_B200_H_
#define CLEO_B200_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes: 0 = ok, one code per reference abort site ---- */
typedef enum cleo_status {
  CLEO_OK = 0,
  CLEO_ERR_XI_ZERO = 1,          /* superdrop_attrs.hpp:157-163  xi < 1 */
  CLEO_ERR_RADIUS_BELOW_DRY = 2, /* superdrop_attrs.hpp:176-182  r < r_dry - 1e-6 */
  CLEO_ERR_NEG_CONDENSATE = 3,   /* superdrop_attrs.hpp:208-218 */
  CLEO_ERR_COALESCENCE = 4,      /* coalescence.cpp:109-111,134-143,180-188 */
  CLEO_ERR_BREAKUP = 5,          /* breakup.hpp:198-256 */
  CLEO_ERR_NR_NOCONVERGE = 6,    /* impliciteuler.cpp:213-217 */
  CLEO_ERR_SUBDELT = 7,          /* impliciteuler.hpp:323-325 */
  CLEO_ERR_CFL = 8,              /* cfl_criteria.hpp:52-54 */
  CLEO_ERR_OUT_OF_BOX = 9,       /* cartesian_motion.hpp:44-52 */
  CLEO_ERR_TEMPERATURE = 10,     /* thermodynamic_equations.cpp:40-42 */
  CLEO_ERR_CAPACITY = 11,        /* more superdroplets or gridboxes than the context holds */
  CLEO_ERR_ARGUMENT = 12,        /* invalid argument (null pointer, bad enum, size mismatch) */
  CLEO_ERR_CUDA = 13,            /* a CUDA runtime call failed */
  CLEO_ERR_TIMEOUT = 14,         /* a bounded device-side wait gave up */
  CLEO_ERR_MLP = 15,             /* surrogate not loaded / bad shape */
  CLEO_ERR_XI_OUTPUT = 16,       /* superdrops_observer.hpp:229-234  xi too large to write */
  CLEO_ERR_IO = 17               /* a file of an output dataset could not be written */
} cleo_status;

/* ---- enumerations of the reference's plug-in choices ---- */
enum cleo_terminalv {        /* libs/superdrops/terminalvelocity.hpp:44-122 */
  CLEO_TV_NULL = 0,
  CLEO_TV_SIMMEL = 1,
  CLEO_TV_ROGERSYAU = 2,
  CLEO_TV_ROGERSGK = 3
};
enum cleo_collprob {         /* PairProbability models */
  CLEO_PROB_GOLOVIN = 0,     /* golovinprob.cpp:31-43 */
  CLEO_PROB_LONG = 1,        /* longhydroprob.hpp:38-66 (Simmel terminal velocity) */
  CLEO_PROB_CONST = 2        /* constprob.hpp:34-49 */
};
enum cleo_collenact {        /* PairEnactX models */
  CLEO_ENACT_COALESCENCE = 0, /* coalescence.cpp:39-54 */
  CLEO_ENACT_BREAKUP = 1,     /* breakup.hpp:141-151 */
  CLEO_ENACT_COALBURE = 2     /* coalbure.hpp:207-256 */
};
enum cleo_nfrags {           /* breakup_nfrags.hpp:40-92 */
  CLEO_NFRAGS_CONST = 0,
  CLEO_NFRAGS_CKE = 1
};
enum cleo_coalbureflag {     /* coalbure_flag.hpp:42-198 */
  CLEO_FLAG_STRAUB = 0,
  CLEO_FLAG_TESTIKSTRAUB = 1,
  CLEO_FLAG_SZAKALLURBICH = 2,
  CLEO_FLAG_CONST = 3
};
enum cleo_nrseed {           /* initial guess of the condensation Newton solve */
  CLEO_NRSEED_REFERENCE = 0, /* ImplicitIterations::initialguess, impliciteuler.cpp:156-170 */
  CLEO_NRSEED_MLP = 1        /* surrogate-predicted post-step r^2 */
};
enum cleo_exec {             /* how the microphysics of one SDM step is scheduled on the GPU */
  CLEO_EXEC_PLAIN = 0,       /* one CTA per gridbox does condensation and collisions */
  CLEO_EXEC_BATCHED = 1      /* flat two-pass condensation + size-bucketed persistent collisions */
};

enum cleo_monitor {          /* SDMMonitor members (libs/observers/sdmmonitor/) */
  CLEO_MONITOR_MASSMOMENTS = 1,     /* MonitorMassMomentsChange<MonitorMassMomentsChangeViews> */
  CLEO_MONITOR_RAINMASSMOMENTS = 2, /* MonitorMassMomentsChange<MonitorRainMassMomentsChangeViews> */
  CLEO_MONITOR_PRECIPITATION = 4    /* MonitorPrecipitation */
};

#define CLEO_STEP_OFF 0xFFFFFFFFu /* interval value that switches a process off (on_step false) */

/*
 * Parameters: one field per argument of the reference factories. Intervals are integer model
 * steps (model_step = 0.01 s, libs/initialise/timesteps.hpp:34); the *_delt fields are the
 * doubles those factories derive from them, passed in so host and device share one value.
 */
typedef struct cleo_b200_params {
  uint32_t condstep;        /* Condensation interval (condensation.hpp:242) */
  uint32_t collstep;        /* CollCoal / CoalBuRe / CollBu interval */
  uint32_t motionstep;      /* CartesianMotion interval (cartesian_motion.hpp:61) */
  uint32_t pad0;
  double cond_delt;         /* step2dimlesstime(condstep)  (condensation.hpp:246) */
  double cond_minsubdelt;   /* realtime2dimless(MINSUBTSTEP) (condensation.hpp:247) */
  double coll_delt;         /* step2realtime(collstep), seconds (coalescence.hpp:137) */
  double motion_delt;       /* step2dimlesstime(motionstep) (predcorr.hpp:150) */
  /* condensation (DoCondensation / ImplicitEuler ctor arguments) */
  int32_t do_alter_thermo;
  uint32_t maxniters;
  double rtol;
  double atol;
  /* collisions */
  int32_t coll_prob;        /* enum cleo_collprob */
  int32_t coll_enact;       /* enum cleo_collenact */
  double coaleff;           /* LongHydroProb(coaleff) */
  double const_kernel;      /* ConstProb(k) */
  int32_t nfrags_kind;      /* enum cleo_nfrags */
  int32_t nfrags_tv;        /* terminal velocity used by CollisionKineticEnergyNFrags */
  double nfrags;            /* ConstNFrags(nfrags) */
  int32_t flag_kind;        /* enum cleo_coalbureflag */
  int32_t flag_tv;          /* terminal velocity used by the Straub/TS/SU flags */
  double flag_coaleff;      /* ConstCoalBuReFlag(coaleff) */
  uint64_t seed;            /* seed of the injected counter-based random stream */
  /* motion */
  int32_t motion_tv;        /* terminal velocity subtracted from w (predcorr.hpp:83-105) */
  int32_t nr_seed;          /* enum cleo_nrseed */
  /* execution (no reference counterpart: results do not depend on it) */
  int32_t exec_mode;        /* enum cleo_exec */
  /* SDMMonitor members to run (libs/observers/sdmmonitor/): a bitmask of enum cleo_monitor */
  int32_t monitors;
} cleo_b200_params;

/*
 * Cartesian gridbox maps (the content of CartesianMaps, cartesianmaps.hpp:49-303, for an
 * undecomposed domain): per gridbox {lower, upper} bounds in each direction and the index of the
 * backwards/forwards neighbour. Index = iz + nz*(ix + nx*iy) (doubly_periodic_domain.hpp:41-70).
 * A neighbour equal to 0xFFFFFFFF is out of the domain. Directions that a model does not resolve
 * carry bounds {-DBL_MAX, DBL_MAX} and the gridbox itself as neighbour (createcartesianmaps.cpp:38-45).
 */
typedef struct cleo_b200_grid {
  uint32_t ngbxs;
  uint32_t ndims[3]; /* number of gridboxes along [coord3, coord1, coord2] */
  const double *coord3lo, *coord3hi, *coord1lo, *coord1hi, *coord2lo, *coord2hi;
  const uint32_t *back3, *fwd3, *back1, *fwd1, *back2, *fwd2;
  /* horizontal area of each gridbox (GbxBoundsFromBinary::gbxarea,
   * gbx_bounds_from_binary.cpp:206-215), used by the precipitation monitor; may be NULL */
  const double* gbxarea;
} cleo_b200_grid;

/* Per-gridbox thermodynamic State (state.hpp:33-120) as SoA arrays of length ngbxs. */
typedef struct cleo_b200_gbx_state {
  double *volume, *press, *temp, *qvap, *qcond;
  double *wvel_lo, *wvel_hi, *uvel_lo, *uvel_hi, *vvel_lo, *vvel_hi;
} cleo_b200_gbx_state;

/* Superdroplets (Superdrop, superdrop.hpp:36-48) as SoA arrays of length n. */
typedef struct cleo_b200_supers {
  uint32_t *sdgbxindex;
  double *coord3, *coord1, *coord2;
  uint64_t *xi;
  double *radius, *msol;
  uint64_t *sdid;
} cleo_b200_supers;

/* Where the first device-side failure happened. */
typedef struct cleo_b200_error {
  int32_t code;      /* cleo_status */
  uint32_t gbxindex; /* gridbox of the failing superdroplet (0xFFFFFFFF if unknown) */
  uint64_t index;    /* position of the failing superdroplet in the SoA arrays */
} cleo_b200_error;

typedef struct cleo_b200_ctx cleo_b200_ctx;

/*
 * Create a context on the current CUDA device for up to `capacity` superdroplets on the given
 * grid. Allocates all device memory the context will use. Validates the parameters the way the
 * reference constructors do (e.g. ImplicitEuler: cond_delt >= cond_minsubdelt).
 */
int cleo_b200_create(const cleo_b200_params* params, const cleo_b200_grid* grid, size_t capacity,
                     cleo_b200_ctx** out);
void cleo_b200_destroy(cleo_b200_ctx* ctx);

/*
 * Copy n superdroplets (host SoA) into the context and sort them by gridbox, like the
 * SupersInDomain constructor (supersindomain.hpp:55-62). n <= capacity.
 */
int cleo_b200_upload_supers(cleo_b200_ctx* ctx, const cleo_b200_supers* host, size_t n);
/* Copy ngbxs gridbox states (host SoA) into the context. */
int cleo_b200_upload_state(cleo_b200_ctx* ctx, const cleo_b200_gbx_state* host);
/*
 * Asynchronous state exchange, for a host whose coupling-step states are known ahead of the
 * step (prescribed or file-driven dynamics): cleo_b200_upload_state_async copies the states
 * (host arrays; pinned memory lets the copy overlap) into a device staging area on a copy stream
 * of the context, behind the previous step's use of that area, and returns at once; the next
 * cleo_b200_step waits for the copy, makes the staged states the live ones at its start, and
 * returns once the host arrays have been read (they may be refilled after it returns). An
 * upload_state (synchronous) in between replaces the staged states.
 * cleo_b200_download_budgets_async takes a device snapshot of the budgets behind the work so far
 * and copies it to the host arrays on a stream of its own while the following steps run; the arrays
 * hold the values once cleo_b200_synchronize has returned. Results are those of the synchronous
 * calls.
 */
int cleo_b200_upload_state_async(cleo_b200_ctx* ctx, const cleo_b200_gbx_state* h);
int cleo_b200_download_budgets_async(cleo_b200_ctx* ctx, double* cond_mass, uint64_t* nr_iters);
int cleo_b200_synchronize(cleo_b200_ctx* ctx);

/*
 * Advance the domain from model step t_mdl to t_next: motion + sort, then microphysics
 * sub-stepping in every gridbox, then removal of null superdroplets (SDMMethods::run_step).
 * Asynchronous: enqueues work on the context's stream. Device failures are reported by
 * cleo_b200_status().
 */
int cleo_b200_step(cleo_b200_ctx* ctx, uint32_t t_mdl, uint32_t t_next);

/* Synchronise the context's stream and return the first recorded failure (CLEO_OK if none). */
int cleo_b200_status(cleo_b200_ctx* ctx, cleo_b200_error* err);

/* Forget the recorded failure (after a host that handled it, e.g. by leaving out the droplets a
 * batch solve marked with CLEO_NITERS_FAILED, carries on; the reference would have aborted).
 * No reference counterpart. Synchronises the context's stream. */
int cleo_b200_clear_status(cleo_b200_ctx* ctx);

/* Number of superdroplets inside the domain (SupersInDomain::domain_nsupers). Synchronises. */
int cleo_b200_domain_nsupers(cleo_b200_ctx* ctx, size_t* n);

/*
 * Copy superdroplets back to host SoA arrays of length >= capacity. The first *n_domain entries
 * are the in-domain superdroplets, sorted by gridbox with the reference's order inside each
 * gridbox; the remaining *n_total - *n_domain are out of the domain (order unspecified, as in
 * sortsupers.hpp:89-92).
 */
int cleo_b200_download_supers(cleo_b200_ctx* ctx, cleo_b200_supers* host, size_t* n_domain,
                              size_t* n_total);
/* Copy the gridbox states back. */
int cleo_b200_download_state(cleo_b200_ctx* ctx, cleo_b200_gbx_state* host);
/*
 * Cumulative FP64 budgets per gridbox (length ngbxs each, may be NULL): condensed mass (the sum of
 * the per-step totmass_condensed that DoCondensation reports to its monitor, condensation.hpp:149)
 * and the number of Newton iterations spent by the condensation solves in the gridbox.
 */
int cleo_b200_download_budgets(cleo_b200_ctx* ctx, double* cond_mass, uint64_t* nr_iters);

/*
 * Solve one implicit-Euler condensation step for n independent droplets already resident in
 * device memory (ImplicitEuler::solve_condensation, impliciteuler.cpp:35-54, with the
 * per-droplet Kohler factors of thermodynamic_equations.hpp:95-107 and the diffusion factor of
 * thermodynamic_equations.cpp:93-114). Inputs are device pointers of length n: radius, msol,
 * temp, press, s_ratio and delt (dimensionless). Writes the new radius (after change_radius, i.e.
 * not below the dry radius) to radius_out and, if niters_out is non-NULL, the Newton iterations
 * spent per droplet, with CLEO_NITERS_FAILED or-ed in for each droplet whose solve hit one of the
 * reference's aborts (no convergence within maxniters, impliciteuler.cpp:213-217; the status
 * reports the first such droplet). Uses the context's maxniters/rtol/atol/minsubdelt and nr_seed.
 */
#define CLEO_NITERS_FAILED 0x80000000u
int cleo_b200_condensation_solve(cleo_b200_ctx* ctx, size_t n, const double* d_radius,
                                 const double* d_msol, const double* d_temp, const double* d_press,
                                 const double* d_s_ratio, const double* d_delt,
                                 double* d_radius_out, uint32_t* d_niters_out);

/* The CUDA stream the context enqueues on (cudaStream_t, as void*). */
void* cleo_b200_stream(cleo_b200_ctx* ctx);

/* Number of kernels the context has launched since it was created (for launch accounting). */
int cleo_b200_kernel_launches(cleo_b200_ctx* ctx, uint64_t* n);

/* What the last re-sort after motion did (synchronises the context's stream): out[0] superdroplets
 * that moved (changed gridbox, left the domain, or were made null by collisions; for a full sort,
 * the valid ones that changed gridbox), out[1] pages rewritten, out[2] how: 0 the touched
 * gridboxes in place, 1 every page repacked, 2 the full sort, out[3] pages in the store (a page
 * holds 64 gridboxes). No reference counterpart: a measurement of the paged store. */
int cleo_b200_resort_stats(cleo_b200_ctx* ctx, uint64_t out[4]);

/* Which re-sort follows motion (same results either way): CLEO_RESORT_AUTO (default) the page
 * re-sort unless more than a fifth of the superdroplets moved in the previous motion step or the
 * store has fewer pages than the GPU has SMs, CLEO_RESORT_PAGES the page re-sort always,
 * CLEO_RESORT_FULL the full sort always. */
#define CLEO_RESORT_AUTO 0
#define CLEO_RESORT_PAGES 1
#define CLEO_RESORT_FULL 2
int cleo_b200_set_resort_policy(cleo_b200_ctx* ctx, int policy);

/*
 * Per-stage device timing with CUDA events on the context's stream, the counterpart of the
 * reference's Kokkos profiling regions (sdm_movement_*, timestep_sdm_microphysics;
 * libs/gridboxes/movesupersindomain.hpp:190-261, libs/runcleo/sdmmethods.hpp:159-216).
 * cleo_b200_set_profiling(ctx, 1) starts recording; cleo_b200_stage_times synchronises, returns
 * the summed milliseconds and counts of the stages {motion, sort, microphysics, condensation,
 * collisions} since the last call, and resets them (condensation and collisions are the parts of
 * microphysics that the batched schedule runs as separate kernels; zero on the plain schedule).
 */
int cleo_b200_set_profiling(cleo_b200_ctx* ctx, int enable);
int cleo_b200_stage_times(cleo_b200_ctx* ctx, double ms[5], uint64_t count[5]);

/*
 * Stable sort of superdroplets by gridbox index that allocates no device memory. No counterpart in
 * the reference: it is for callers that cannot call cudaMalloc while they run (a host model that
 * reserves all device memory at start-up and forbids allocation in its time loop, where an
 * allocation would also synchronise the device, or a caller whose memory belongs to another
 * framework's pool). It computes what the context's sort computes (sortsupers.hpp:93-226
 * semantics: keys above ngbxs share the last bucket) with scratch held in a file-scope device
 * array of about 16.3 MiB, which every GPU that loads the library keeps until the process exits.
 *   d_sdgbxindex  n gridbox indices (device memory)
 *   d_order       out: n positions, d_order[j] = position of the j-th superdroplet in sorted order
 *   d_gstart      out, may be NULL: ngbxs + 2 entries, the first sorted position of each gridbox
 *                 (entry ngbxs = number of in-domain superdroplets, entry ngbxs + 1 = n)
 *   stream        cudaStream_t to enqueue on (as void*; NULL = default stream)
 * n must not exceed 1,048,576 (else CLEO_ERR_CAPACITY). The first call on a device looks up the
 * scratch array's device address (cudaGetSymbolAddress) with that device current. With CUDA's
 * lazy module loading (the default) that lookup is what loads this code onto the device, so the
 * ~16.3 MiB array is allocated by the driver then, and the device may synchronise. Make that
 * first call once per device at start-up, before reserving the rest of device memory, entering
 * the time loop or capturing a stream: a call with n = 0 (pointers may then be NULL) does only
 * the set-up. All calls share the one scratch array, so calls whose work overlaps on the GPU
 * (e.g. on two streams at once) race; each call writes every scratch word it reads, so nothing
 * needs clearing between calls. Asynchronous on `stream`.
 */
int cleo_b200_sort_by_gridbox_static(const uint32_t* d_sdgbxindex, uint32_t n, uint32_t ngbxs,
                                     uint32_t* d_order, uint32_t* d_gstart, void* stream);

/*
 * SDMMonitor members selected by params.monitors, per gridbox (host arrays of ngbxs, any may be
 * NULL). Mass moments (calculate_massmoments / calculate_rainmassmoments,
 * massmoments_observer.cpp:38-113): mom0 = sum xi (u64), mom1 = sum (float)(xi m), mom2 = sum
 * (float)(xi m m) over the gridbox's superdroplets (rain: radius >= 40 um), summed in the
 * superdroplets' order; the changes accumulated after each SDM step's microphysics and after each
 * motion step (MonitorMassMomentsChange::monitor_microphysics / monitor_motion,
 * monitor_massmoments_change.hpp:99-121, 287-305). Precipitation: condensate mass x xi / rho_l /
 * gridbox area of superdroplets that cross their gridbox's lower coord3 bound during motion
 * (MonitorPrecipitation::monitor_precipitation, monitor_precipitation_observer.hpp:97-107).
 */
typedef struct cleo_b200_monitors {
  uint64_t *mom0_micro, *mom0_motion, *rain_mom0_micro, *rain_mom0_motion;
  float *mom1_micro, *mom2_micro, *mom1_motion, *mom2_motion;
  float *rain_mom1_micro, *rain_mom2_micro, *rain_mom1_motion, *rain_mom2_motion;
  double* precip;
} cleo_b200_monitors;
/* before_timestepping of the monitors: the current moments become the baseline of the
 * accumulated changes, and all accumulations restart from zero. */
int cleo_b200_monitors_begin(cleo_b200_ctx* ctx);
/* Copy the accumulated changes and precipitation to the host; reset != 0 then zeroes them
 * (reset_monitor; the baselines stay). */
int cleo_b200_download_monitors(cleo_b200_ctx* ctx, cleo_b200_monitors* out, int reset);

/*
 * Condensation surrogate (no counterpart in the reference, whose Newton-Raphson iteration always
 * starts from ImplicitIterations::initialguess, impliciteuler.cpp:156-170). A 7 -> 64 -> 64 -> 1
 * GELU multilayer perceptron predicts log(z_new / r^2) of one implicit-Euler condensation step
 * (z = r^2) from the features log r, log msol, s_ratio - 1, T, p, delt, log(3 b / a)
 * (dimensionless units). With nr_seed = CLEO_NRSEED_MLP and a surrogate attached to a context,
 * its prediction replaces the initial guess of the branches whose root is unique (the branch
 * decision itself is the reference's); a seeded solve that does not converge within maxniters
 * restarts from the reference's guess. Weights: FP32 master copy for training, BF16 copies with
 * FP32 accumulation for inference (layer 2 on tcgen05 tensor cores). All calls are on the stream
 * given at creation and return once their results are ready.
 */
typedef struct cleo_b200_mlp cleo_b200_mlp;
#define CLEO_MLP_NFEATURES 7
#define CLEO_MLP_NHIDDEN 64
#define CLEO_MLP_NPARAMS 4737 /* W1[64][7], b1[64], W2[64][64], b2[64], W3[64], b3 */
#define CLEO_MLP_NNORM 16     /* feature means[7], feature inverse scales[7], target mean, scale */
enum cleo_mlp_path {
  CLEO_MLP_TCGEN05 = 0,  /* layer 2 by tcgen05.mma, accumulator in tensor memory */
  CLEO_MLP_MMA_SYNC = 1, /* layer 2 by warp-level mma.sync m16n8k16 (check path) */
  CLEO_MLP_FP32 = 2      /* scalar FP32 on the same BF16 operands (check path) */
};
/* New model on the current device, Glorot-uniform weights from `seed`, identity standardisation. */
int cleo_b200_mlp_create(void* stream, uint64_t seed, cleo_b200_mlp** out);
int cleo_b200_mlp_destroy(cleo_b200_mlp* mlp);
/* Host arrays of CLEO_MLP_NPARAMS and CLEO_MLP_NNORM floats; set also resets the Adam state. */
int cleo_b200_mlp_set_params(cleo_b200_mlp* mlp, const float* params, const float* norm);
int cleo_b200_mlp_get_params(cleo_b200_mlp* mlp, float* params, float* norm);
/*
 * Raw features of n droplets (device arrays as cleo_b200_condensation_solve takes them) into
 * d_features[n][7]. Optional: d_target[n] = log(r_new^2 / r^2) from d_radius_new, and d_direct[n]
 * = 1 where solve_condensation takes its direct (non-sub-stepping) branch, the branch a seed
 * applies to.
 */
int cleo_b200_mlp_features(cleo_b200_mlp* mlp, size_t n, const double* d_radius,
                           const double* d_msol, const double* d_temp, const double* d_press,
                           const double* d_s_ratio, const double* d_delt,
                           const double* d_radius_new, float* d_features, float* d_target,
                           uint8_t* d_direct);
/* Feature and target means and scales from n training pairs (device arrays). */
int cleo_b200_mlp_fit_normalisation(cleo_b200_mlp* mlp, size_t n, const float* d_features,
                                    const float* d_target);
/*
 * Mean squared error of the standardised target over n samples (n <= 2^24) and its gradient with
 * respect to the FP32 master parameters: d_grad[CLEO_MLP_NPARAMS], d_loss[1] (device, FP32).
 */
int cleo_b200_mlp_loss_grad(cleo_b200_mlp* mlp, size_t n, const float* d_features,
                            const float* d_target, float* d_grad, float* d_loss);
/*
 * `steps` Adam steps (beta 0.9 / 0.999, linear warm-up then cosine decay of `lr`) on minibatches
 * of `batch` samples (a multiple of 128) drawn uniformly from the n pairs by a counter generator
 * keyed by `seed`. d_loss_per_step (device, optional) receives each step's minibatch loss.
 */
int cleo_b200_mlp_train(cleo_b200_mlp* mlp, size_t n, const float* d_features,
                        const float* d_target, uint32_t steps, uint32_t batch, float lr,
                        uint64_t seed, float* d_loss_per_step);
/* Predicted log(z_new / r^2) of n feature rows into d_out[n] by one of cleo_mlp_path. */
int cleo_b200_mlp_infer(cleo_b200_mlp* mlp, size_t n, const float* d_features, float* d_out,
                        int path);
/* Attach (or detach, with NULL) the surrogate that nr_seed = CLEO_NRSEED_MLP uses. */
int cleo_b200_set_surrogate(cleo_b200_ctx* ctx, cleo_b200_mlp* mlp);

/*
 * CUDA graphs for the batched schedule (on by default; no counterpart in the reference). Each
 * batched SDM step's launch sequence is captured once per distinct pattern (current buffer,
 * motion, step length, sub-step pattern) and replayed as one graph launch afterwards; results
 * are the same with graphs on or off. Steps run eagerly while stage profiling is on.
 */
int cleo_b200_set_graphs(cleo_b200_ctx* ctx, int on);

/*
 * Autotuner of the batched schedule (no counterpart in the reference). The next 4 * reps batched
 * SDM steps run as ordinary steps (same results) while each times one of four candidate launch
 * configurations per stage: for condensation pass A, the block size (128 or 256) and the
 * compiled variant's resident-CTA target (4 or 5 per SM, i.e. its register budget); for
 * collisions, the largest gridbox of the warp-per-gridbox kernel (64 or 128) and the resident-CTA
 * target (2 or 3) of its 64-slot variant (the 128-slot variant, for gridboxes of 65..128
 * superdroplets, runs at 2). The fastest option of each stage is kept, and cached per process
 * by GPU name and domain size so that later contexts of that size start from it. Steps run
 * eagerly (with a stream synchronisation each) while tuning.
 */
int cleo_b200_autotune(cleo_b200_ctx* ctx, int reps);
/* Current configuration {pass-A block, pass-A CTA target, warp-kernel gridbox limit, CTA target of
 * the warp kernel's 64-slot variant}; returns 1 while tuning is still in progress, else CLEO_OK. */
int cleo_b200_tuned_config(cleo_b200_ctx* ctx, int32_t cfg[4]);
/* Set that configuration directly (ending a tuning run in progress): pass-A block 128 or 256,
 * pass-A CTA target 3, 4 or 5, warp-kernel gridbox limit 1..128 (gridboxes above it go to the
 * CTA-per-gridbox kernels), CTA target 2 or 3 of the warp kernel's 64-slot variant. Results do
 * not depend on it. */
int cleo_b200_set_launch_config(cleo_b200_ctx* ctx, const int32_t cfg[4]);

/*
 * Superdroplet output (SuperdropsObserver, observers/superdrops_observer.hpp:485-490, with the
 * Collect* variables of superdrops_observer.hpp:139-470, and TimeObserver, time_observer.hpp:
 * 46-144, writing into a SimpleDataset<FSStore>, zarr/simple_dataset.hpp:44-292). An
 * observation writes the domain superdroplets (each gridbox's superdroplets in gridbox order,
 * as SDMMethods::at_start_step passes them, sdmmethods.hpp:300-305) to ragged 1-D Zarr v2
 * arrays, converted the way the Collect* functors convert them: sdgbxindex and sdId to uint32,
 * xi to uint64, radius, msol and the coordinates to float (dimensionless values, with the
 * reference's units and scale factors in each array's .zattrs), then appends their count to
 * "raggedcount" and the observation time float(t_mdl / 1e5) (step2dimlesstime,
 * initialise/timesteps.hpp:56-59) to "time". The files are the ones the reference writes for
 * the same observations, byte for byte.
 */
enum cleo_obs_var {
  CLEO_OBS_SDID = 1,
  CLEO_OBS_SDGBXINDEX = 2,
  CLEO_OBS_XI = 4,
  CLEO_OBS_RADIUS = 8,
  CLEO_OBS_MSOL = 16,
  CLEO_OBS_COORD3 = 32,
  CLEO_OBS_COORD1 = 64,
  CLEO_OBS_COORD2 = 128,
  CLEO_OBS_ALL = 255
};
/* Host arrays of the output types; a NULL member is skipped. */
typedef struct cleo_b200_obs_supers {
  uint32_t* sdid;
  uint32_t* sdgbxindex;
  uint64_t* xi;
  float* radius;
  float* msol;
  float* coord3;
  float* coord1;
  float* coord2;
} cleo_b200_obs_supers;
/*
 * The domain superdroplets of a context, gathered and converted on the GPU (the Collect*
 * functors' copy loop, parallel_write_data.hpp:240-246) and copied into out's host arrays of at
 * least `cap` elements (pinned memory copies fastest). *n receives their number; more than cap
 * gives CLEO_ERR_CAPACITY with nothing copied.
 */
int cleo_b200_gather_supers(cleo_b200_ctx* ctx, uint32_t vars, const cleo_b200_obs_supers* out,
                            size_t cap, size_t* n);

typedef struct cleo_b200_zarr cleo_b200_zarr;
/* New dataset in directory `dir` (created if needed): TimeObserver >> SuperdropsObserver of the
 * variables in `vars`, observing at model steps that are multiples of `interval`, all arrays in
 * chunks of `maxchunk` elements. */
int cleo_b200_zarr_open(const char* dir, size_t maxchunk, uint32_t interval, uint32_t vars,
                        cleo_b200_zarr** out);
/* ConstTstepObserver::at_start_step at model step t_mdl with a context's domain superdroplets
 * (nothing unless t_mdl is a multiple of the interval). */
int cleo_b200_zarr_observe(cleo_b200_zarr* z, cleo_b200_ctx* ctx, uint32_t t_mdl);
/* The same observation of n superdroplets given as host arrays of the output types (members of
 * the dataset's variables must be non-NULL). */
int cleo_b200_zarr_observe_host(cleo_b200_zarr* z, uint32_t t_mdl, const cleo_b200_obs_supers* s,
                                size_t n);
/* Write the last partly filled chunks and the final array shapes, then free the writer. */
int cleo_b200_zarr_close(cleo_b200_zarr* z);

/*
 * Self-check of the bounded device waits (no counterpart in the reference). Every wait of the
 * library's kernels on an mbarrier (bulk-copy staging, tensor-core completion) gives up after a
 * bounded number of tries, records CLEO_ERR_TIMEOUT and lets the kernel return, so that a stuck
 * wait surfaces as a status instead of a hung device. This runs that wait on the current device
 * on a barrier that nothing completes, with max_tries (1 .. 2^24) tries per thread, and returns
 * the status the wait produced: CLEO_ERR_TIMEOUT when the bound works.
 */
int cleo_b200_check_bounded_wait(uint32_t max_tries);

/*
 * Self-check of the device math (no counterpart in the reference), for n elements of device
 * arrays on the current device's default stream (synchronised before return):
 *   fn = CLEO_MATH_POW:  out[i] = the correctly rounded pow(x[i], y[i])
 *   fn = CLEO_MATH_EXP:  out[i] = the correctly rounded exp(x[i])  (y unused)
 *   fn = CLEO_MATH_VENT: out[i] = the ventilation factor of radius x[i] (impliciteuler.cpp:
 *                        131-145, as the condensation kernels evaluate it; y unused)
 * The same functions built for the host give the values to compare with, bit for bit.
 */
#define CLEO_MATH_POW 0
#define CLEO_MATH_EXP 1
#define CLEO_MATH_VENT 2
int cleo_b200_check_math(int fn, const double* d_x, const double* d_y, double* d_out, size_t n);

/* Library version string. */
const char* cleo_b200_version(void);

#ifdef __cplusplus
}
#endif

#endif /* CLEO_B200_H_ */
