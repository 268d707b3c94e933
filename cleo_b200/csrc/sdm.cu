// sdm.cu — the B200 SDM step behind the C ABI of include/cleo_b200.h.
//
// Device layout: structure-of-arrays superdroplets (sdgbxindex u32, coord3/1/2 f64, xi u64,
// radius f64, msol f64, sdid u64) in the paged store of pages.cuh: pages of 64 gridboxes, each
// page's gridboxes in index order with free slots between and after them; per gridbox g the
// superdroplets [gstart[g], gstart[g] + gcount[g]) are the ones SupersInGbx refs would select.
// Superdroplets that leave the domain or become null are appended to a separate out-of-domain
// store (the reference keeps them at the tail of its array in unspecified order). Null
// superdroplets made by collisions stay after the gcount valid ones of their gridbox until the
// next re-sort (the reference re-sorts at once, sdmmethods.hpp:221-229; both give the same
// in-domain superdroplets in the same order).
//
// One SDM step (SDMMethods::run_step, sdmmethods.hpp:319-332):
//   motion  -> k_motion: predictor-corrector coords + new gridbox index per droplet, and either
//              the movers of every 32 slots as a mask (the page re-sort) or the sort keys
//   sort    -> chosen per step from the previous motion step's mover count: the page re-sort
//              (the movers listed and radix-sorted alone, the gridboxes they leave or enter
//              rewritten in place, pages.cuh) while at most a fifth of the droplets moved, else
//              the full sort (radix passes over (key, position), every page written packed); then
//              the append of out-of-domain droplets to the store
//   microphysics -> plain schedule: k_micro, one CTA per gridbox: qcond from the moved droplets,
//              condensation (FP64 Newton) and collisions (shared-memory shuffle, parallel pairs,
//              null removal) for every sub-step of the SDM step; batched schedule: the kernels of
//              batched.cuh, captured as one CUDA graph per step pattern.
// Around the step: superdroplet output (gather into CLEO's output types), SDMMonitor members,
// the asynchronous state and budget exchange, the autotuner and the condensation surrogate's
// seeding.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "mlp.cuh"
#include "physics.cuh"
#include "sort.cuh"

using namespace cleo;

namespace {

constexpr int MICRO_THREADS = 256;
constexpr uint32_t NSMEM = 1024;  // gridboxes up to this size are staged in shared memory
constexpr size_t MICRO_SMEM = (size_t)NSMEM * (8 + 8 + 8 + 4 + 4);

struct Fields {  // one SoA buffer
  uint32_t* gbx;
  double *c3, *c1, *c2;
  unsigned long long* xi;
  double *r, *msol;
  unsigned long long* id;
};

struct DevCtx {
  cleo_b200_params p;
  uint32_t ngbxs;
  uint32_t ndims[3];
  uint32_t capacity;
  // maps
  const double *b3lo, *b3hi, *b1lo, *b1hi, *b2lo, *b2hi;
  const uint32_t *back3, *fwd3, *back1, *fwd1, *back2, *fwd2;
  // states
  double *volume, *press, *temp, *qvap, *qcond, *wlo, *whi, *ulo, *uhi, *vlo, *vhi;
  double* cond_mass;
  unsigned long long* nr_iters;
  // superdroplets (current buffer) and the out-of-domain store
  Fields sd;
  Fields grave;
  uint32_t* gstart;  // ngbxs + 2
  uint32_t* gcount;  // ngbxs
  uint32_t* counters;  // [0] nrange, [1] ndomain, [2] ngrave
  // SDMMonitor members (allocated when params.monitors != 0): mass-moment changes
  // [all, rain][after microphysics, after motion], the previous moments, precipitation
  unsigned long long* mm0[2][2];
  float *mm1[2][2], *mm2[2][2];
  unsigned long long* prev0[2];
  float *prev1[2], *prev2[2];
  double *precip, *precip_c, *gbxarea;  // per gridbox, per superdroplet, per gridbox
  // re-sort after motion (pages.cuh): mover flags then their exclusive scan (slots + 1); a full
  // sort's per-key first sorted positions (ngbxs + 2)
  uint32_t *mv_scan, *gstart_new;  // mv_scan: movers per 32 slots, scanned (exclusive)
  uint32_t* mv_mask;   // the movers among each 32 slots, a bit each (k_motion)
  uint32_t* mv_tsums;  // the count scan's tile offsets (the scan's readers add them: mv_before)
  uint32_t* mv_total;  // valid superdroplets that changed gridbox in the last motion step
  // paged layout (pages.cuh): pages of PAGE_GBXS gridboxes, their slot starts (npages + 1), the
  // touched-page flags and list, the re-sort's counters, the movers' records; slots = the SoA
  // buffers' length (capacity plus the pages' slack)
  uint32_t npages, slots;
  uint32_t *pstart, *pg_flag, *pg_list, *pg_ctr;
  uint32_t *mv_lo, *mv_hi, *mv_stamp;  // per gridbox: its run of sorted movers, the re-sort's stamp
  Fields mvrec;
  // scratch
  double *scr_r, *scr_m, *scr_c3, *scr_c1, *scr_c2;
  unsigned long long *scr_x, *scr_id;
  uint32_t *scr_p, *scr_j;
  DevError* err;
};

// droplet inputs of cleo_b200_condensation_solve -> Newton seed r^2 (the surrogate's IO)
struct CondSeedIO {
  const double *radius, *msol, *temp, *press, *s_ratio, *delt;
  double* seed;
  __device__ __forceinline__ void features(uint32_t i, float x[mlp::NIN]) const {
    mlp::raw_features(radius[i], msol[i], temp[i], press[i], s_ratio[i], delt[i], x);
  }
  __device__ __forceinline__ void store(uint32_t i, float t) const {
    seed[i] = mlp::seed_from(radius[i], t);
  }
  __device__ __forceinline__ uint32_t rows(uint32_t n) const { return n; }
};
}  // namespace

#include "batched_types.cuh"

struct cleo_b200_ctx {
  DevCtx d;
  Fields buf[2];
  int cur = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  int device = 0;
  // sort scratch
  uint32_t *keys[2], *vals[2], *hist, *tile_sums;
  uint32_t *gs_tsums = nullptr, *mv_count = nullptr;  // scan tile totals, the mover count
  uint32_t *pstart_new = nullptr, *ps_tsums = nullptr;  // page re-sort: repacked page starts
  double* qm_buf = nullptr;  // BatchScratch::qm's storage
  bool one_box = false;      // a one-gridbox domain: collisions by the kernels of onebox.cuh
  OneBox ob{};
  // re-sort choice: {movers, superdroplets} of the previous motion step, written by the device
  // into mapped pinned memory right after that step's motion kernel; an event recorded behind
  // the write (an external event node inside a captured step) lets the host wait for exactly
  // that step's values before it chooses the next step's sort, so the choice is deterministic
  uint32_t* h_motion = nullptr;
  uint32_t* d_motion = nullptr;
  cudaEvent_t ev_report = nullptr;
  bool report_recorded = false;
  bool sort_full = false;
  bool last_sort_full = false;  // what the last re-sort after motion was (cleo_b200_resort_stats)
  int resort_policy = CLEO_RESORT_AUTO;
  int sms = 148;                // the device's SMs
  // asynchronous state upload (cleo_b200_upload_state_async): staging area for the 11 state
  // fields, a copy stream, and events for "copied" and "taken by a step"
  double* stage_state = nullptr;
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t ev_uploaded = nullptr, ev_consumed = nullptr;
  bool upload_pending = false, consumed_recorded = false;
  // asynchronous budget download: a device snapshot copied to the host on the copy stream
  double* snap_budgets = nullptr;  // [2][ngbxs]: condensed mass, Newton iterations
  cudaStream_t d2h_stream = nullptr;  // its own stream: the next upload must not queue behind it
  cudaEvent_t ev_snap = nullptr, ev_snap_free = nullptr;
  bool snap_in_flight = false;
  int ensure_copy_stream() {
    if (copy_stream) return CLEO_OK;
    bool ok = cudaStreamCreateWithFlags(&copy_stream, cudaStreamNonBlocking) == cudaSuccess &&
              cudaStreamCreateWithFlags(&d2h_stream, cudaStreamNonBlocking) == cudaSuccess;
    for (cudaEvent_t* e : {&ev_uploaded, &ev_consumed, &ev_snap, &ev_snap_free})
      ok = ok && cudaEventCreateWithFlags(e, cudaEventDisableTiming) == cudaSuccess;
    return ok ? CLEO_OK : CLEO_ERR_CUDA;
  }
  // superdroplet output staging (allocated at the first gather): converted fields, offsets
  uint8_t* obs_stage = nullptr;
  uint32_t *obs_start = nullptr, *obs_tsums = nullptr;
  uint32_t ntiles_max, key_bits;
  BatchScratch bs{};              // batched-schedule scratch
  int grid_small[2] = {0, 0};  // the 64-slot warp kernel at [2 / 3 CTAs per SM]
  int grid_wide = 0;            // the 128-slot warp kernel (2 CTAs per SM)
  int grid_medium = 0, grid_large = 0, grid_flat = 0;
  int grid_condb[3] = {0, 0, 0};  // pass B at 3, 4, 5 resident CTAs per SM
  unsigned long long launches = 0;  // kernels launched by this context
  std::vector<void*> allocs;
  // stage timing: (stage, start, end) event triples recorded while profiling is on
  bool profiling = false;
  struct Mark {
    int stage;
    cudaEvent_t a, b;
  };
  std::vector<Mark> marks;
  std::vector<cudaEvent_t> event_pool;
  // launch configuration of the batched schedule (results do not depend on it) and the online
  // autotuner that chooses it by timing candidates on live steps
  struct TuneCfg {
    int cond_block;       // threads per block of pass A
    int cond_minb;        // pass-A variant (3, 4 or 5): resident 256-thread CTAs per SM it is
                          // compiled for
    uint32_t small_max;   // gridboxes up to this size go to the warp kernel
    int small_minb;       // 64-slot warp kernel: resident CTAs per SM it is compiled for
    int condb_minb;       // pass-B variant (3, 4 or 5), tuned apart from pass A's
  };
  TuneCfg cfg{256, 3, SMALL_MAX, 2, 3};
  std::vector<TuneCfg> cand;
  std::vector<double> t_cond, t_condb, t_coll;
  size_t tune_step = 0, tune_total = 0;
  std::string tune_key;
  // CUDA graphs of batched SDM steps, keyed by what decides a step's launch sequence (the
  // current SoA buffer, motion on/off, the step length and the sub-step pattern)
  struct StepGraph {
    std::vector<uint32_t> sig;
    cudaGraphExec_t exec;
    int cur_after;
    unsigned long long nodes;
  };
  std::vector<StepGraph> graphs;
  bool use_graphs = true;
  uint32_t t_dev = 0xFFFFFFFFu;  // the step time the device word holds (host mirror)
  void drop_graphs() {
    for (auto& g : graphs) cudaGraphExecDestroy(g.exec);
    graphs.clear();
  }
  // condensation surrogate (nr_seed = CLEO_NRSEED_MLP) and its seed buffer for condensation_solve
  const cleo_b200_mlp* mlp = nullptr;
  double* seed_buf = nullptr;
  size_t seed_cap = 0;
  // two-pass condensation_solve scratch (deferred-solve list and its radix sort)
  struct CsScratch {
    size_t cap = 0;
    uint32_t *k0 = nullptr, *v0 = nullptr, *k1 = nullptr, *v1 = nullptr;
    uint32_t *hist = nullptr, *tsums = nullptr, *ctr = nullptr;  // ctr: deferred solves
    double* zres = nullptr;  // pass A's iterates of the restarts
    uint32_t nt = 0;
  } cs;
  void free_cs() {
    for (uint32_t* q : {cs.k0, cs.v0, cs.k1, cs.v1, cs.hist, cs.tsums, cs.ctr}) cudaFree(q);
    cudaFree(cs.zres);
    cs = CsScratch();
  }
  cudaEvent_t take_event() {
    if (!event_pool.empty()) {
      cudaEvent_t e = event_pool.back();
      event_pool.pop_back();
      return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
  }
};

namespace {
// RAII stage marker: records an event pair around a stage when profiling is on
// stage indexes of cleo_b200_stage_times are 0..4; marks past them are the tuner's own
constexpr int STAGE_COND_B = 5;
struct StageMark {
  cleo_b200_ctx* x;
  int stage;
  cudaEvent_t a = nullptr;
  StageMark(cleo_b200_ctx* x_, int st) : x(x_), stage(st) {
    if (x->profiling) {
      a = x->take_event();
      cudaEventRecord(a, x->stream);
    }
  }
  ~StageMark() {
    if (x->profiling && a) {
      cudaEvent_t b = x->take_event();
      cudaEventRecord(b, x->stream);
      x->marks.push_back({stage, a, b});
    }
  }
};
}  // namespace

#define CUDA_TRY(expr)                                          \
  do {                                                          \
    cudaError_t e_ = (expr);                                    \
    if (e_ != cudaSuccess) {                                    \
      fprintf(stderr, "cleo_b200: %s failed: %s\n", #expr, cudaGetErrorString(e_)); \
      return CLEO_ERR_CUDA;                                     \
    }                                                           \
  } while (0)

// ------------------------------------------------------------------------------------------
// kernels
// ------------------------------------------------------------------------------------------
namespace {

__device__ __forceinline__ void bounds_of(const double* lo, const double* hi, uint32_t ngbxs,
                                          uint32_t i, double& l, double& h) {
  if (i < ngbxs) {
    l = lo[i];
    h = hi[i];
  } else {  // oob key: nullbounds (createcartesianmaps.cpp:40)
    l = -DBLMAX;
    h = DBLMAX;
  }
}

}  // namespace

#include "pages.cuh"

namespace {

// interpolation: predcorr.cpp:30-42
__device__ __forceinline__ double interpolation(double blo, double bhi, double vlo, double vhi,
                                                double sdcoord) {
  // zero wind on both faces: with a finite positive extent the clamped coordinate gives alpha in
  // [0, 1], so alpha * vhi + (1 - alpha) * vlo is exactly vhi + vlo (signed zeros included),
  // without the division
  const double extent = bhi - blo;
  if (vlo == 0.0 && vhi == 0.0 && extent > 0.0 && extent <= DBLMAX) return vhi + vlo;
  const double coord = fmin(bhi, fmax(blo, sdcoord));
  const double alpha = (coord - blo) / (bhi - blo);
  return alpha * vhi + (1 - alpha) * vlo;
}

__device__ __forceinline__ int flag_sdgbxindex(uint32_t idx, uint32_t ngbxs, double blo,
                                               double bhi, double coord) {
  if (idx == OOB || idx >= ngbxs) return 0;  // cartesianmaps.cpp:93-107
  if (coord < blo) return 1;
  if (coord >= bhi) return 2;
  return 0;
}

__device__ __forceinline__ bool beyond_domainboundary(uint32_t gbxindex, uint32_t increment,
                                                      uint32_t ndim) {
  return (gbxindex / increment) % ndim == 0;  // domainboundaries.hpp:34-37
}

// k_motion: MoveSupersInGridboxesFunctor (movesupersindomain.hpp:47-93) for every droplet:
// PredCorr::operator() (predcorr.hpp:156-171), cfl_criteria, PredCorrMotion::superdrop_gbx
// (predcorrmotion.hpp:85-106) with get_no_decomposition_bounding_gridbox (cartesianmaps.cpp:278)
// and CartesianCheckBounds. For the full re-sort it writes each slot's sort key (its new
// gridbox, ngbxs out of the domain, ngbxs + 1 for a free slot) and position; for the page re-sort
// it flags the movers (pages.cuh).
// One superdroplet's motion (movesupersindomain.hpp:255-261: the predictor-corrector step, the
// neighbour search, the bounds check); returns whether it moves in the re-sort (changes gridbox,
// leaves the domain, or is a null one collisions left). For the full sort it writes the sort key
// (gridbox, ngbxs out of the domain, ngbxs + 1 for a free slot) and position.
__device__ __forceinline__ bool move_superdroplet(const DevCtx& c, uint32_t i,
                                                  uint32_t* __restrict__ keys,
                                                  uint32_t* __restrict__ vals, int incremental) {
  const uint32_t ng = c.ngbxs;
  const double delt = c.p.motion_delt;
  const uint32_t g = c.sd.gbx[i];
  if (!incremental) vals[i] = i;
  if (g >= ng) {  // a null superdroplet left by collisions (out of the domain), or a free slot
    const bool hole = is_hole(c.sd, i);
    if (!incremental) keys[i] = hole ? ng + 1 : ng;
    return !hole;  // a null one moves to the out-of-domain store
  }
    const Where w{c.err, g, i};
    double bzl, bzh, bxl, bxh, byl, byh;
    bounds_of(c.b3lo, c.b3hi, ng, g, bzl, bzh);
    bounds_of(c.b1lo, c.b1hi, ng, g, bxl, bxh);
    bounds_of(c.b2lo, c.b2hi, ng, g, byl, byh);
    const double wl = c.wlo[g], wh = c.whi[g], ul = c.ulo[g], uh = c.uhi[g], vl = c.vlo[g],
                 vh = c.vhi[g];
    const double c3 = c.sd.c3[i], c1 = c.sd.c1[i], c2 = c.sd.c2[i];
    // delta_coord3: predcorr.hpp:83-105
    double coord3 = c3;
    const double terminal = terminalv(c.p.motion_tv, c.sd.r[i]);
    double vel3 = interpolation(bzl, bzh, wl, wh, coord3);
    vel3 -= terminal;
    coord3 += vel3 * delt;
    double corrvel3 = interpolation(bzl, bzh, wl, wh, coord3);
    corrvel3 -= terminal;
    const double delta3 = (vel3 + corrvel3) * (delt / 2);
    // delta_coord1: predcorr.hpp:107-125
    double coord1 = c1;
    const double vel1 = interpolation(bxl, bxh, ul, uh, coord1);
    coord1 += vel1 * delt;
    const double corrvel1 = interpolation(bxl, bxh, ul, uh, coord1);
    const double delta1 = (vel1 + corrvel1) * (delt / 2);
    // delta_coord2: predcorr.hpp:127-145
    double coord2 = c2;
    const double vel2 = interpolation(byl, byh, vl, vh, coord2);
    coord2 += vel2 * delt;
    const double corrvel2 = interpolation(byl, byh, vl, vh, coord2);
    const double delta2 = (vel2 + corrvel2) * (delt / 2);
    // cfl_criteria: cfl_criteria.hpp:30-57
    bool cfl = (fabs(delta3) <= fabs(bzh - bzl));
    cfl = (fabs(delta1) <= fabs(bxh - bxl)) && cfl;
    cfl = (fabs(delta2) <= fabs(byh - byl)) && cfl;
    if (!cfl) w.fail(CLEO_ERR_CFL);
    double n3 = c3 + delta3, n1 = c1 + delta1, n2 = c2 + delta2;
    // monitor_precipitation (monitor_precipitation_observer.hpp:97-107): the contribution of a
    // superdroplet below its gridbox's lower bound, added per gridbox in order by k_mon_precip
    if (c.precip_c)
      c.precip_c[i] = (n3 < bzl) ? condensate_mass(c.sd.r[i], c.sd.msol[i], w) *
                                       (double)c.sd.xi[i] / Rho_l / c.gbxarea[g]
                                 : 0.0;
    // change_if_coord3nghbr: finite z, coordinate unchanged at the edge (cartesianmaps.cpp:184-213)
    uint32_t idx = g;
    int flag = flag_sdgbxindex(idx, ng, bzl, bzh, n3);
    bool crossed = flag != 0;  // whether any face was crossed (then idx may differ from g)
    if (flag == 1) idx = c.back3[idx];
    else if (flag == 2) idx = c.fwd3[idx];
    // change_if_coord1nghbr: periodic x (cartesianmaps.cpp:148-179)
    {
      double l = bxl, h = bxh;  // g's own bounds unless z moved the superdroplet
      if (crossed) bounds_of(c.b1lo, c.b1hi, ng, idx, l, h);
      flag = flag_sdgbxindex(idx, ng, l, h, n1);
      crossed |= flag != 0;
      const uint32_t incre = c.ndims[0];
      if (flag == 1) {
        const uint32_t nghbr = c.back1[idx];
        if (beyond_domainboundary(idx, incre, c.ndims[1])) {
          double nl, nh;
          bounds_of(c.b1lo, c.b1hi, ng, nghbr, nl, nh);
          n1 = n1 + nh - l;
        }
        idx = nghbr;
      } else if (flag == 2) {
        const uint32_t nghbr = c.fwd1[idx];
        if (beyond_domainboundary(idx + incre, incre, c.ndims[1])) {
          double nl, nh;
          bounds_of(c.b1lo, c.b1hi, ng, nghbr, nl, nh);
          n1 = n1 + nl - h;
        }
        idx = nghbr;
      }
    }
    // change_if_coord2nghbr: periodic y (cartesianmaps.cpp:112-143)
    {
      double l = byl, h = byh;
      if (crossed) bounds_of(c.b2lo, c.b2hi, ng, idx, l, h);
      flag = flag_sdgbxindex(idx, ng, l, h, n2);
      crossed |= flag != 0;
      const uint32_t incre = c.ndims[0] * c.ndims[1];
      if (flag == 1) {
        const uint32_t nghbr = c.back2[idx];
        if (beyond_domainboundary(idx, incre, c.ndims[2])) {
          double nl, nh;
          bounds_of(c.b2lo, c.b2hi, ng, nghbr, nl, nh);
          n2 = n2 + nh - l;
        }
        idx = nghbr;
      } else if (flag == 2) {
        const uint32_t nghbr = c.fwd2[idx];
        if (beyond_domainboundary(idx + incre, incre, c.ndims[2])) {
          double nl, nh;
          bounds_of(c.b2lo, c.b2hi, ng, nghbr, nl, nh);
          n2 = n2 + nl - h;
        }
        idx = nghbr;
      }
    }
    // a field whose bits did not change is not stored (sedimentation alone changes coord3 only,
    // and few superdroplets change gridbox): the same values, less DRAM written
    const auto bits = [](double v) { return __double_as_longlong(v); };
    if (bits(n3) != bits(c3)) c.sd.c3[i] = n3;
    if (bits(n1) != bits(c1)) c.sd.c1[i] = n1;
    if (bits(n2) != bits(c2)) c.sd.c2[i] = n2;
    if (idx != g) c.sd.gbx[i] = idx;
    // CartesianCheckBounds (cartesian_motion.hpp:38-54); a superdroplet that crossed no face
    // stays in g with every coordinate inside g's bounds (the three flags were 0), so passes it
    if (crossed && idx < ng) {
      double l, h;
      bool bad = false;
      bounds_of(c.b3lo, c.b3hi, ng, idx, l, h);
      bad |= (n3 < l) | (n3 >= h);
      bounds_of(c.b1lo, c.b1hi, ng, idx, l, h);
      bad |= (n1 < l) | (n1 >= h);
      bounds_of(c.b2lo, c.b2hi, ng, idx, l, h);
      bad |= (n2 < l) | (n2 >= h);
      if (bad) w.fail(CLEO_ERR_OUT_OF_BOX);
    }
    const uint32_t key = idx < ng ? idx : ng;
    if (!incremental) keys[i] = key;  // the incremental re-sort takes min(gbx, ngbxs) instead
    // a superdroplet that changes gridbox (or leaves the domain) moves in the re-sort
    const bool mover = key != g;
    {  // count them (warp-aggregated) for the choice of the next re-sort
      const unsigned am = __activemask();
      const unsigned bm = __ballot_sync(am, mover);
      if (bm && (int)(threadIdx.x & 31) == __ffs(am) - 1) atomicAdd(c.mv_total, __popc(bm));
    }
    return mover;
}
__global__ void __launch_bounds__(256, 4)  // 64 registers: measured 15% faster than 80
k_motion(const __grid_constant__ DevCtx c, uint32_t* __restrict__ keys, uint32_t* __restrict__ vals, int incremental) {
  const uint32_t n = c.counters[0];
  const uint32_t nchunks = (n + 31) / 32;
  if (incremental && blockIdx.x == 0 && threadIdx.x == 0) c.mv_scan[nchunks] = 0;  // scan total
  // i0 is the same for the whole block, so every warp's lanes cover 32 consecutive slots together
  for (uint32_t i0 = blockIdx.x * blockDim.x; i0 < n; i0 += gridDim.x * blockDim.x) {
    const uint32_t i = i0 + threadIdx.x;
    bool mover = false;
    if (i < n) mover = move_superdroplet(c, i, keys, vals, incremental);
    if (incremental) {  // the movers of the warp's 32 slots: a mask and its count
      const unsigned bm = __ballot_sync(0xFFFFFFFFu, mover);
      if ((threadIdx.x & 31) == 0 && i < n) {
        c.mv_mask[i >> 5] = bm;
        c.mv_scan[i >> 5] = __popc(bm);
      }
    }
  }
}
__global__ void k_mv_report(const __grid_constant__ DevCtx c, uint32_t* __restrict__ out) {  // mapped host memory
  out[0] = *c.mv_total;
  out[1] = c.counters[0];
}

// ---- the movers of a page re-sort (pages.cuh), listed in position order ----
// the exclusive scan of the per-32-slot mover counts at chunk w: the scan within its tile plus
// the tile's offset (the scan's own pass adding the offsets in place is left out; its readers add
// them)
__device__ __forceinline__ uint32_t mv_before(const DevCtx& c, uint32_t w) {
  return c.mv_scan[w] + c.mv_tsums[w / SCAN_TILE];
}
// the movers, from the masks of the chunks that hold any: positions and keys (min(gbx, ngbxs) of
// the gridbox indices k_motion wrote)
__global__ void k_mv_list(const __grid_constant__ DevCtx c, uint32_t* __restrict__ mk, uint32_t* __restrict__ mvp) {
  const uint32_t nchunks = (c.counters[0] + 31) / 32;
  for (uint32_t w = blockIdx.x * blockDim.x + threadIdx.x; w < nchunks;
       w += gridDim.x * blockDim.x) {
    uint32_t m = c.mv_mask[w];
    if (m == 0u) continue;
    uint32_t p = mv_before(c, w);
    while (m) {
      const uint32_t i = w * 32 + (uint32_t)(__ffs(m) - 1);
      m &= m - 1u;
      const uint32_t gbx = c.sd.gbx[i];
      mk[p] = gbx < c.ngbxs ? gbx : c.ngbxs;
      mvp[p] = i;
      ++p;
    }
  }
}
__global__ void k_mv_count(const __grid_constant__ DevCtx c, uint32_t* __restrict__ count) {
  *count = mv_before(c, (c.counters[0] + 31) / 32);  // number of movers
}
// ---- superdroplet output: the domain superdroplets, gathered in gridbox order and converted
// the way the reference's Collect* functors convert them (superdrops_observer.hpp:139-464) ----
struct ObsOut {
  uint32_t* sdid;
  uint32_t* gbx;
  uint64_t* xi;
  float *r, *msol, *c3, *c1, *c2;
};
__global__ void k_obs_counts(const __grid_constant__ DevCtx c, uint32_t* __restrict__ start) {  // scanned to out offsets
  for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < c.ngbxs; g += gridDim.x * blockDim.x)
    start[g] = c.gcount[g];
}
__global__ void __launch_bounds__(256)
k_obs_gather(const __grid_constant__ DevCtx c, ObsOut o, const uint32_t* __restrict__ start) {
  const uint32_t n = c.counters[0];
  const uint32_t ng = c.ngbxs;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint32_t g = c.sd.gbx[i];
    if (g >= ng) continue;  // a null superdroplet: not in the domain
    // valid superdroplets lead their gridbox's range [gstart[g], gstart[g] + gcount[g])
    const uint32_t k = start[g] + (i - c.gstart[g]);
    if (o.sdid) o.sdid[k] = (uint32_t)c.sd.id[i];
    if (o.gbx) o.gbx[k] = g;
    if (o.xi) {
      const uint64_t xi = c.sd.xi[i];
      if (xi == ~0ull) Where{c.err, g, i}.fail(CLEO_ERR_XI_OUTPUT);
      o.xi[k] = xi;
    }
    if (o.r) o.r[k] = (float)c.sd.r[i];
    if (o.msol) o.msol[k] = (float)c.sd.msol[i];
    if (o.c3) o.c3[k] = (float)c.sd.c3[i];
    if (o.c1) o.c1[k] = (float)c.sd.c1[i];
    if (o.c2) o.c2[k] = (float)c.sd.c2[i];
  }
}

// self-check of the bounded waits: an mbarrier that nothing arrives on, waited for with the
// same bounded wait as the bulk-copy and tensor-core waits; the bound must run out
__global__ void k_math_check(int fn, const double* __restrict__ x, const double* __restrict__ y,
                             double* __restrict__ out, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    out[i] = fn == CLEO_MATH_POW   ? cleo::dpow(x[i], y[i])
             : fn == CLEO_MATH_EXP ? cleo::dexp(x[i])
                                   : ventilation_factor(x[i]);
}
__global__ void k_wait_check(uint32_t max_tries, int* __restrict__ out) {
  __shared__ uint64_t bar;
  if (threadIdx.x == 0) mlp::mbar_init(&bar, 1);
  __syncthreads();
  const bool completed = mlp::mbar_wait_bounded(&bar, 0, max_tries);
  const int all = __syncthreads_or(completed ? 1 : 0);
  if (threadIdx.x == 0) *out = all ? CLEO_OK : CLEO_ERR_TIMEOUT;
}

// The sum of a gridbox's n terms in the superdroplets' order, the way the reference's
// reductions add them (condensation.cpp:29-35 and movesupersindomain.hpp:125-131 state the
// sequential loop as their meaning): one thread adds term(0), term(1), ... one after another.
// Four terms are loaded before they are added, so the loads overlap the chain of additions; the
// additions keep their order, so the result is the sequential loop's double.
template <class Term>
__device__ __forceinline__ double seq_sum(uint32_t n, Term term) {
  double acc = 0.0;
  uint32_t k = 0;
  for (; k + 4 <= n; k += 4) {
    const double t0 = term(k), t1 = term(k + 1), t2 = term(k + 2), t3 = term(k + 3);
    acc += t0;
    acc += t1;
    acc += t2;
    acc += t3;
  }
  for (; k < n; ++k) acc += term(k);
  return acc;
}

// ---- block reductions (fixed order: warp shuffles then warps in order; integers) ----
template <class T>
__device__ __forceinline__ T block_sum(T v, T* sh) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xFFFFFFFFu, v, o);
  __syncthreads();
  if (lane == 0) sh[warp] = v;
  __syncthreads();
  T s = 0;
  if (threadIdx.x == 0) {
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) s += sh[k];
    sh[0] = s;
  }
  __syncthreads();
  s = sh[0];
  __syncthreads();
  return s;
}

// exclusive scan over a block (any blockDim multiple of 32, <= 1024)
__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t* wsum, uint32_t& total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nw = blockDim.x >> 5;
  uint32_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) wsum[warp] = x;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t s = 0;
    for (int k = 0; k < nw; ++k) {
      const uint32_t t = wsum[k];
      wsum[k] = s;
      s += t;
    }
    wsum[nw] = s;
  }
  __syncthreads();
  const uint32_t r = wsum[warp] + x - v;
  total = wsum[nw];
  __syncthreads();
  return r;
}

// ------------------------------------------------------------------------------------------
// k_micro: SDMMicrophysicsFunctor (sdmmethods.hpp:54-93) for one gridbox per CTA
// ------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(MICRO_THREADS)
k_micro(const __grid_constant__ DevCtx c, uint32_t t_sdm, uint32_t t_sdm_next, int did_motion) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ unsigned long long shu[32];
  __shared__ uint32_t shw[40];
  const cleo_b200_params& p = c.p;
  const int tid = threadIdx.x;
  for (uint32_t g = blockIdx.x; g < c.ngbxs; g += gridDim.x) {
    const uint32_t base = c.gstart[g];
    uint32_t n = c.gcount[g];
    // per-superdroplet terms of the gridbox's sums (shared memory, or the gridbox's range of the
    // global scratch beyond NSMEM), added in order by thread 0 (seq_sum)
    double* terms = n <= NSMEM ? reinterpret_cast<double*>(smem) : c.scr_r + base;
    // effect_on_hydrometeor_states after motion (movesupersindomain.hpp:95-136)
    if (did_motion) {
      for (uint32_t k = tid; k < n; k += blockDim.x) {
        const Where w{c.err, g, base + k};
        terms[k] = condensate_mass(c.sd.r[base + k], c.sd.msol[base + k], w) *
                   (double)c.sd.xi[base + k];
      }
      __syncthreads();
      if (tid == 0) {
        const double totmass_cond = seq_sum(n, [&](uint32_t k) { return terms[k]; });
        const double R0cubed_VOL0 = R0 * R0 * R0 / VOL0;
        const double rho_cond = totmass_cond / c.volume[g] * R0cubed_VOL0;
        const double rho_dry = dry_air_density(c.press[g], c.temp[g], c.qvap[g]);
        c.qcond[g] = rho_cond / rho_dry;
      }
      __syncthreads();
    }
    const uint64_t key = cleo_rng_key(p.seed, t_sdm, g);
    uint64_t slot = 0;
    uint32_t subt = t_sdm;
    while (subt < t_sdm_next) {
      // ---- DoCondensation (condensation.cpp:43-138) ----
      if (on_step(p.condstep, subt)) {
        const Where wg{c.err, g, base};
        const double temp = c.temp[g];
        const double psat = saturation_pressure(temp, wg);
        const double s_ratio = supersaturation_ratio(c.press[g], c.qvap[g], psat);
        const double ffactor = diffusion_factor(c.press[g], temp, psat);
        const NewtonCfg cfg{p.maxniters, p.rtol, p.atol};
        double* dm = terms;  // (n only shrinks within the step: the choice of storage holds)
        unsigned long long its = 0;
        for (uint32_t k = tid; k < n; k += blockDim.x) {
          const uint32_t i = base + k;
          const Where w{c.err, g, i};
          const double r = c.sd.r[i], msol = c.sd.msol[i];
          const double old_m_cond = condensate_mass(r, msol, w);
          double akoh, bkoh;
          kohler_factors(msol, temp, akoh, bkoh);
          uint32_t ni = 0;
          const double newr = solve_condensation(cfg, p.cond_delt, p.cond_minsubdelt, s_ratio,
                                                 akoh, bkoh, ffactor, r, 0.0, ni, w);
          const double rnew = max_dryradius(newr, msol);  // change_radius
          c.sd.r[i] = rnew;
          dm[k] = (condensate_mass(rnew, msol, w) - old_m_cond) * (double)c.sd.xi[i];
          its += ni;
        }
        const unsigned long long totits = block_sum(its, shu);  // (its barriers publish dm)
        if (tid == 0) {
          const double totmass = seq_sum(n, [&](uint32_t k) { return dm[k]; });
          if (p.do_alter_thermo) {  // state_change: condensation.cpp:126-138
            const double R0cubed_VOL0 = R0 * R0 * R0 / VOL0;
            const double totrho = totmass / c.volume[g] * R0cubed_VOL0;
            const double rho_dry = dry_air_density(c.press[g], c.temp[g], c.qvap[g]);
            const double dq = totrho / rho_dry;
            c.qvap[g] -= dq;
            c.qcond[g] += dq;
            const double dtemp = (Latent_v / moist_specifc_heat(c.qvap[g], c.qcond[g])) * dq;
            c.temp[g] += dtemp;
          }
          c.cond_mass[g] += totmass;
          c.nr_iters[g] += totits;
        }
        __syncthreads();
      }
      // ---- DoCollisions (collisions.hpp:263-278) ----
      if (on_step(p.collstep, subt)) {
        const bool in_smem = n <= NSMEM;
        double* Sr = in_smem ? reinterpret_cast<double*>(smem) : c.scr_r + base;
        double* Sm = in_smem ? reinterpret_cast<double*>(smem) + NSMEM : c.scr_m + base;
        unsigned long long* Sx = in_smem ? reinterpret_cast<unsigned long long*>(smem) + 2 * NSMEM
                                         : c.scr_x + base;
        uint32_t* P = in_smem ? reinterpret_cast<uint32_t*>(smem + 24 * NSMEM) : c.scr_p + base;
        uint32_t* J = in_smem ? reinterpret_cast<uint32_t*>(smem + 28 * NSMEM) : c.scr_j + base;
        for (uint32_t k = tid; k < n; k += blockDim.x) {
          Sr[k] = c.sd.r[base + k];
          Sm[k] = c.sd.msol[base + k];
          Sx[k] = c.sd.xi[base + k];
          P[k] = k;
          // Fisher-Yates draw for position k (k >= 1): slot n-1-k (shuffle.hpp:80-87)
          if (k >= 1) J[k] = (uint32_t)cleo_rng_range(cleo_rng_u64(key, slot + (n - 1 - k)), 0, (uint64_t)k + 1);
        }
        __syncthreads();
        if (tid == 0) {
          for (uint32_t it = n > 0 ? n - 1 : 0; it > 0; --it) {
            const uint32_t j = J[it];
            const uint32_t t = P[it];
            P[it] = P[j];
            P[j] = t;
          }
        }
        __syncthreads();
        const uint64_t slot_pairs = slot + (n >= 1 ? n - 1 : 0);
        const uint32_t npairs = n / 2;
        const double scale_p = (double)n * ((double)n - 1.0) / (2.0 * (double)npairs);
        const double VOLUME = c.volume[g] * VOL0;
        uint32_t nnull = 0;
        for (uint32_t jj = tid; jj < npairs; jj += blockDim.x) {
          const uint32_t a = P[2 * jj], b = P[2 * jj + 1];
          const Where w{c.err, g, (uint64_t)base + 2 * jj};
          Drop dA{Sx[a], Sr[a], Sm[a]};
          Drop dB{Sx[b], Sr[b], Sm[b]};
          const bool swap = dA.xi < dB.xi;  // assign_drops: collisions.hpp:94-101
          Drop& d1 = swap ? dB : dA;
          Drop& d2 = swap ? dA : dB;
          const double prob_jk = pair_prob(p, d1.r, d2.r, VOLUME);
          const double large_xi = (double)d1.xi;
          const double prob = scale_p * large_xi * prob_jk;
          const double phi_coll = cleo_rng_to_unit(cleo_rng_u64(key, slot_pairs + 2ull * jj));
          const double phi_out = cleo_rng_to_unit(cleo_rng_u64(key, slot_pairs + 2ull * jj + 1));
          nnull += enact_collision(p, d1, d2, prob, phi_coll, phi_out, w);
          Sx[a] = dA.xi; Sr[a] = dA.r; Sm[a] = dA.msol;
          Sx[b] = dB.xi; Sr[b] = dB.r; Sm[b] = dB.msol;
        }
        slot = slot_pairs + 2ull * npairs;
        const uint32_t totnull = block_sum(nnull, shw);
        // write back in shuffled order; nulls moved behind the valid ones, stably
        // (remove_null_supers: collisions.hpp:240-248)
        uint32_t nvalid = n - totnull;
        uint32_t cval = 0, cnull = 0;
        for (uint32_t k0 = 0; k0 < n; k0 += blockDim.x) {
          const uint32_t k = k0 + tid;
          const bool act = k < n;
          const uint32_t src = act ? P[k] : 0;
          const bool valid = act && Sx[src] != 0;
          uint32_t tv, tn;
          const uint32_t ev = block_excl_scan(valid ? 1u : 0u, shw, tv);
          const uint32_t en = block_excl_scan((act && !valid) ? 1u : 0u, shw, tn);
          if (act) {
            const uint32_t q = valid ? (cval + ev) : (nvalid + cnull + en);
            const uint32_t o = base + q;
            const uint32_t s = base + src;
            c.scr_c3[o] = c.sd.c3[s];
            c.scr_c1[o] = c.sd.c1[s];
            c.scr_c2[o] = c.sd.c2[s];
            c.scr_id[o] = c.sd.id[s];
            J[q] = src;  // inverse map, J no longer needed
          }
          cval += tv;
          cnull += tn;
        }
        __syncthreads();
        for (uint32_t q = tid; q < n; q += blockDim.x) {
          const uint32_t src = J[q];
          const uint32_t o = base + q;
          c.sd.r[o] = Sr[src];
          c.sd.msol[o] = Sm[src];
          c.sd.xi[o] = Sx[src];
          c.sd.gbx[o] = q < nvalid ? g : OOB;
          c.sd.c3[o] = c.scr_c3[o];
          c.sd.c1[o] = c.scr_c1[o];
          c.sd.c2[o] = c.scr_c2[o];
          c.sd.id[o] = c.scr_id[o];
        }
        __syncthreads();
        n = nvalid;
      }
      subt = min(next_step(p.condstep, subt), next_step(p.collstep, subt));
    }
    if (tid == 0) c.gcount[g] = n;
    __syncthreads();
  }
}

// batched implicit-Euler solves of independent droplets
__global__ void k_condsolve(const __grid_constant__ DevCtx c, uint32_t n, const double* __restrict__ radius,
                            const double* __restrict__ msol, const double* __restrict__ temp,
                            const double* __restrict__ press, const double* __restrict__ s_ratio,
                            const double* __restrict__ delt, const double* __restrict__ seeds,
                            double* __restrict__ out, uint32_t* __restrict__ niters_out) {
  const NewtonCfg cfg{c.p.maxniters, c.p.rtol, c.p.atol};
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    uint32_t failed = 0;
    const Where w{c.err, OOB, i, &failed};
    const double T = temp[i];
    const double psat = saturation_pressure(T, w);
    const double ffactor = diffusion_factor(press[i], T, psat);
    double akoh, bkoh;
    kohler_factors(msol[i], T, akoh, bkoh);
    uint32_t ni = 0;
    const double newr = solve_condensation(cfg, delt[i], c.p.cond_minsubdelt, s_ratio[i], akoh,
                                           bkoh, ffactor, radius[i], seeds ? seeds[i] : 0.0, ni,
                                           w);
    out[i] = max_dryradius(newr, msol[i]);
    if (niters_out) niters_out[i] = ni | (failed ? CLEO_NITERS_FAILED : 0u);
  }
}

// ---- SDMMonitor members: one thread per gridbox, sums in the superdroplets' order ----
// calculate_massmoments / calculate_rainmassmoments (massmoments_observer.cpp:38-113)
__device__ __forceinline__ void mon_moments(const DevCtx& c, uint32_t g, int rain,
                                            unsigned long long& m0, float& m1, float& m2) {
  const double rlim = 40e-6 / R0;
  const uint32_t base = c.gstart[g], n = c.gcount[g];
  unsigned long long a0 = 0;
  float a1 = 0.0f, a2 = 0.0f;
  for (uint32_t k = base; k < base + n; ++k) {
    const double r = c.sd.r[k];
    const unsigned long long x = c.sd.xi[k];
    const bool binary = rain ? (r >= rlim) : true;
    a0 += x * (unsigned long long)binary;
    const double mass = sd_mass(r, c.sd.msol[k]);
    const double xi = (double)x;
    a1 += (float)(xi * mass * (double)binary);
    a2 += (float)(xi * mass * mass * (double)binary);
  }
  m0 = a0;
  m1 = a1;
  m2 = a2;
}
// fetch_delta_massmoments (monitor_massmoments_change.hpp:99-121); which = 0 after
// microphysics, 1 after motion; begin != 0: before_timestepping (moments become the baseline)
__global__ void k_mon_mm(const __grid_constant__ DevCtx c, int which, int begin) {
  const int mask = c.p.monitors;
  for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < c.ngbxs;
       g += gridDim.x * blockDim.x) {
    for (int rain = 0; rain < 2; ++rain) {
      if (!begin && !(mask & (rain ? CLEO_MONITOR_RAINMASSMOMENTS : CLEO_MONITOR_MASSMOMENTS)))
        continue;
      unsigned long long m0;
      float m1, m2;
      mon_moments(c, g, rain, m0, m1, m2);
      if (!begin) {
        c.mm0[rain][which][g] += m0 - c.prev0[rain][g];
        c.mm1[rain][which][g] += m1 - c.prev1[rain][g];
        c.mm2[rain][which][g] += m2 - c.prev2[rain][g];
      }
      c.prev0[rain][g] = m0;
      c.prev1[rain][g] = m1;
      c.prev2[rain][g] = m2;
    }
  }
}
// the precipitation contributions of each gridbox's superdroplets, in their order (the
// reference adds them one by one as it moves the gridbox's superdroplets)
__global__ void k_mon_precip(const __grid_constant__ DevCtx c) {
  for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < c.ngbxs;
       g += gridDim.x * blockDim.x) {
    const uint32_t base = c.gstart[g], n = c.gcount[g];
    double acc = c.precip[g];
    for (uint32_t k = base; k < base + n; ++k) {
      const double v = c.precip_c[k];
      if (v > 0.0) acc += v;
    }
    c.precip[g] = acc;
  }
}

}  // namespace

#include "batched.cuh"
#include "onebox.cuh"

namespace {

// Two-pass form of the batch solve (the batched schedule), as k_cond_a / k_cond_b do for the
// SDM step: pass A finishes every direct solve that converges within its first two iterations
// (or within the seeded attempt) and lists the rest, keyed by sub-step count; pass B solves the
// listed ones after the list has been sorted by that key, so that neighbouring lanes carry
// similar work. Iterations spent in pass A on an abandoned seed are carried in niters_out.
__device__ __forceinline__ uint32_t cs_warp_append(uint32_t* ctr, bool flag) {
  const unsigned m = __ballot_sync(0xFFFFFFFFu, flag);
  uint32_t base = 0;
  const int lane = threadIdx.x & 31;
  if (lane == 0 && m) base = atomicAdd(ctr, (uint32_t)__popc(m));
  base = __shfl_sync(0xFFFFFFFFu, base, 0);
  return base + __popc(m & ((1u << lane) - 1u));
}
__global__ void __launch_bounds__(256)
k_cs_a(const __grid_constant__ DevCtx c, uint32_t n, const double* __restrict__ radius, const double* __restrict__ msol,
       const double* __restrict__ temp, const double* __restrict__ press,
       const double* __restrict__ s_ratio, const double* __restrict__ delt,
       double* __restrict__ seeds, double* __restrict__ out, uint32_t* __restrict__ niters_out,
       double* __restrict__ zres, uint32_t* __restrict__ lkeys, uint32_t* __restrict__ lvals,
       uint32_t* __restrict__ ctr) {
  const NewtonCfg cfg{c.p.maxniters, c.p.rtol, c.p.atol};
  for (uint32_t i0 = blockIdx.x * blockDim.x; i0 < n; i0 += gridDim.x * blockDim.x) {
    const uint32_t i = i0 + threadIdx.x;
    bool defer = false;
    uint32_t key = 0;
    if (i < n) {
      uint32_t failed = 0;
      const Where w{c.err, OOB, i, &failed};
      const double T = temp[i], r = radius[i], dt = delt[i];
      const double psat = saturation_pressure(T, w);
      const double ffactor = diffusion_factor(press[i], T, psat);
      double akoh, bkoh;
      kohler_factors(msol[i], T, akoh, bkoh);
      const OdeConsts o{s_ratio[i], akoh, bkoh, ffactor / ventilation_factor(r)};
      const double z0 = initialguess(o, r);
      const bool ucrit1 = first_unique_criteria(o, r, z0);
      double crit = 0.0;
      uint32_t ni = 0, carried = 0;
      if (ucrit1 || below_critical_timestep(o, dt, crit)) {
        bool conv = false, seeded = false, conv1 = false;
        double z1 = 0.0;
        GEval e = eval_g(o, dt, r, z0);
        if (seeds && seed_ok(seeds[i])) {  // the surrogate's seed, when its residual is smaller
          const GEval es = eval_g(o, dt, r, seeds[i]);
          if (fabs(es.g) < fabs(e.g)) {
            double zs;
            conv = integrate_seeded(cfg, o, dt, r, es, ni, zs) && seeded_root_ok(o, ucrit1, zs);
            e.z = zs;
            seeded = true;
            if (!conv) {
              seeds[i] = -1.0;  // pass B starts from the reference guess
              carried = ni;
            }
          }
        }
        if (!seeded) {
          e = nr_iterate(cfg, o, dt, r, e, conv, ni);
          conv1 = conv;
          z1 = e.z;
          e = nr_iterate(cfg, o, dt, r, e, conv, ni);
        }
        if (conv) {
          out[i] = max_dryradius(sqrt(e.z), msol[i]);
          if (niters_out) niters_out[i] = ni | (failed ? CLEO_NITERS_FAILED : 0u);
        } else {
          defer = true;  // restart until converged (impliciteuler.cpp:136-140), key 0
          // where pass B's restart continues; NaN after an abandoned seed (a full solve)
          zres[i] = seeded ? __longlong_as_double(0x7FF8000000000000ll) : (conv1 ? -z1 : e.z);
        }
      } else {
        defer = true;
        key = deferred_key(dt, fmax(crit, c.p.cond_minsubdelt), true);
      }
      if (defer && niters_out) niters_out[i] = carried | (failed ? CLEO_NITERS_FAILED : 0u);
    }
    const uint32_t pos = cs_warp_append(ctr, defer);
    if (defer) {
      lkeys[pos] = key;
      lvals[pos] = i;
    }
  }
}
__global__ void __launch_bounds__(256)
k_cs_b(const __grid_constant__ DevCtx c, const double* __restrict__ radius, const double* __restrict__ msol,
       const double* __restrict__ temp, const double* __restrict__ press,
       const double* __restrict__ s_ratio, const double* __restrict__ delt,
       const double* __restrict__ seeds, double* __restrict__ out,
       uint32_t* __restrict__ niters_out, const double* __restrict__ zres,
       const uint32_t* __restrict__ lkeys, const uint32_t* __restrict__ lvals,
       const uint32_t* __restrict__ ctr) {
  const NewtonCfg cfg{c.p.maxniters, c.p.rtol, c.p.atol};
  const uint32_t nl = *ctr;
  for (uint32_t jr = blockIdx.x * blockDim.x + threadIdx.x; jr < nl;
       jr += gridDim.x * blockDim.x) {
    const uint32_t j = nl - 1 - jr;  // most expensive solves first (the list is sorted by cost)
    const uint32_t i = lvals[j];
    uint32_t failed = 0;
    const Where w{c.err, OOB, i, &failed};
    const double T = temp[i], r = radius[i], dt = delt[i];
    const double psat = saturation_pressure(T, w);
    const double ffactor = diffusion_factor(press[i], T, psat);
    double akoh, bkoh;
    kohler_factors(msol[i], T, akoh, bkoh);
    uint32_t ni = 0;
    double newr;
    const double zr = lkeys[j] == 0u ? zres[i] : 0.0;
    if (lkeys[j] == 0u && cfg.maxniters >= 2 && zr == zr) {
      // a direct solve whose two reference iterations in pass A did not converge: the restart
      // continues from them (resume_restart)
      const OdeConsts o{s_ratio[i], akoh, bkoh, ffactor / ventilation_factor(r)};
      ni = 2;
      double rsqrd = 0.0;
      const int code = resume_restart(cfg, o, dt, r, zr, ni, rsqrd);
      if (code) w.fail(code);
      newr = sqrt(rsqrd);
    } else {
      const double seed = seeds ? seeds[i] : 0.0;
      newr = solve_condensation(cfg, dt, c.p.cond_minsubdelt, s_ratio[i], akoh, bkoh, ffactor, r,
                                seed, ni, w);
    }
    out[i] = max_dryradius(newr, msol[i]);
    if (niters_out) niters_out[i] = (niters_out[i] + ni) | (failed ? CLEO_NITERS_FAILED : 0u);
  }
}

}  // namespace

// ------------------------------------------------------------------------------------------
// host side
// ------------------------------------------------------------------------------------------
namespace {

template <class T>
int dalloc(cleo_b200_ctx* x, T** p, size_t n) {
  void* q = nullptr;
  CUDA_TRY(cudaMalloc(&q, (n ? n : 1) * sizeof(T)));
  x->allocs.push_back(q);
  *p = static_cast<T*>(q);
  return CLEO_OK;
}

// two elements of padding: the warp collision kernel's bulk copies may read one element past
// the last superdroplet
int alloc_fields(cleo_b200_ctx* x, Fields& f, size_t n) {
  int rc = 0;
  n += 2;
  rc |= dalloc(x, &f.gbx, n);
  rc |= dalloc(x, &f.c3, n);
  rc |= dalloc(x, &f.c1, n);
  rc |= dalloc(x, &f.c2, n);
  rc |= dalloc(x, &f.xi, n);
  rc |= dalloc(x, &f.r, n);
  rc |= dalloc(x, &f.msol, n);
  rc |= dalloc(x, &f.id, n);
  return rc ? CLEO_ERR_CUDA : CLEO_OK;
}

int grid_for(size_t n, int threads) {
  size_t b = (n + threads - 1) / threads;
  if (b < 1) b = 1;
  if (b > 148 * 64) b = 148 * 64;
  return (int)b;
}

// exclusive scan of a[0, n) on the context's stream, in place, the total into a[n] (tsums: the
// scan's tile totals, (n + SCAN_TILE) / SCAN_TILE + 1 words)
void scan_u32(cleo_b200_ctx* x, uint32_t* a, uint32_t n, uint32_t* tsums) {
  cudaStream_t s = x->stream;
  const uint32_t nt = (uint32_t)(((uint64_t)n + SCAN_TILE - 1) / SCAN_TILE);
  k_scan_tiles<<<nt ? nt : 1, SCAN_THREADS, 0, s>>>(a, a, n, tsums);
  k_scan_sums<<<1, SCAN_THREADS, 0, s>>>(tsums, nt ? nt : 1, a + n);
  k_scan_add<<<(unsigned)((n + 255) / 256 + 1), 256, 0, s>>>(a, n, tsums);
  x->launches += 3;
}

// Full re-sort (pages.cuh): stable radix sort of the current buffer's slots [0, nrange) by the
// keys in keys[0] (gridbox, out of domain, free slot), then the in-domain superdroplets written
// into the other buffer page by page with PAGE_SLACK free slots after each page, the gridboxes'
// ranges, and the out-of-domain ones appended to their store.
int sort_current(cleo_b200_ctx* x) {
  DevCtx& d = x->d;
  cudaStream_t s = x->stream;
  const uint32_t nt = x->ntiles_max;
  uint32_t* kin = x->keys[0];
  uint32_t* vin = x->vals[0];
  uint32_t* kout = x->keys[1];
  uint32_t* vout = x->vals[1];
  const uint64_t nh = (uint64_t)256 * nt;
  const uint32_t nscan_tiles = (uint32_t)((nh + SCAN_TILE - 1) / SCAN_TILE);
  for (uint32_t shift = 0; shift < x->key_bits; shift += 8) {
    k_rs_upsweep<<<nt, RS_THREADS, 0, s>>>(kin, d.counters, (int)shift, x->hist, nt);
    k_scan_tiles<<<nscan_tiles, SCAN_THREADS, 0, s>>>(x->hist, x->hist, nh, x->tile_sums);
    k_scan_sums<<<1, SCAN_THREADS, 0, s>>>(x->tile_sums, nscan_tiles, nullptr);
    k_scan_add<<<(unsigned)((nh + 255) / 256), 256, 0, s>>>(x->hist, nh, x->tile_sums);
    k_rs_downsweep<<<nt, RS_THREADS, 0, s>>>(kin, vin, d.counters, (int)shift, x->hist, nt, kout,
                                             vout);
    x->launches += 5;
    std::swap(kin, kout);
    std::swap(vin, vout);
  }
  // sorted (key, position) now in kin/vin
  Fields& src = x->buf[x->cur];
  Fields& dst = x->buf[1 - x->cur];
  uint32_t* gp = d.gstart_new;
  const int gs = grid_for(d.slots, 256), gp2 = grid_for((size_t)d.ngbxs + 2, 256);
  k_lower_bounds<<<gp2, 256, 0, s>>>(d, kin, gp);
  k_pg_sizes_full<<<grid_for(d.npages, 256), 256, 0, s>>>(d, gp, d.pstart);
  x->launches += 2;
  scan_u32(x, d.pstart, d.npages, x->ps_tsums);
  k_gather_paged<<<gs, 256, 0, s>>>(d, src, dst, kin, vin, gp);
  k_pg_fill_full<<<grid_for(std::max(d.npages, d.ngbxs), 256), 256, 0, s>>>(d, dst, gp);
  k_grave_sorted<<<gs, 256, 0, s>>>(d, src, vin, gp);
  k_full_commit<<<1, 1, 0, s>>>(d, gp);
  x->launches += 4;
  x->cur = 1 - x->cur;
  d.sd = x->buf[x->cur];
  CUDA_TRY(cudaGetLastError());
  return CLEO_OK;
}

int radix_pairs_on(cleo_b200_ctx* x, uint32_t* k0, uint32_t* v0, uint32_t* k1, uint32_t* v1,
                   const uint32_t* n_ptr, uint32_t bits, uint32_t* hist, uint32_t* tile_sums,
                   uint32_t nt, uint32_t unsorted_max = 0);

// The page re-sort after motion (pages.cuh; k_motion left a mover mask per 32 slots): scan of the
// masks' counts, the movers listed in position order and stably radix-sorted by key, copied out
// to the mover
// buffer; the touched pages rewritten in place, or, when one would outgrow its slots, every page
// rewritten into the other buffer and copied back (the device decides; both paths are launched);
// movers out of the domain appended to their store. The current buffer stays current.
int sort_incremental(cleo_b200_ctx* x) {
  DevCtx& d = x->d;
  cudaStream_t s = x->stream;
  // exclusive scan of the per-32-slot mover counts, chunks + 1 of them for the slots' capacity
  // (entries past the slots in use are stale but only move the values after them, which nothing
  // reads) (readers add the tile offsets: mv_before)
  const uint64_t n1 = ((uint64_t)d.slots + 31) / 32 + 1;
  const uint32_t nscan = (uint32_t)((n1 + SCAN_TILE - 1) / SCAN_TILE);
  k_pg_reset<<<1, 1, 0, s>>>(d);
  k_scan_tiles<<<nscan, SCAN_THREADS, 0, s>>>(d.mv_scan, d.mv_scan, n1, d.mv_tsums);
  k_scan_sums<<<1, SCAN_THREADS, 0, s>>>(d.mv_tsums, nscan, nullptr);
  x->launches += 3;
  k_mv_list<<<grid_for(n1, 256), 256, 0, s>>>(d, x->keys[1], x->vals[1]);
  k_mv_count<<<1, 1, 0, s>>>(d, x->mv_count);
  x->launches += 2;
  // the movers stably by key (the mover count is read by the radix kernels on the device)
  const int where = radix_pairs_on(x, x->keys[1], x->vals[1], d.scr_p, d.scr_j, x->mv_count,
                                   x->key_bits, x->hist, x->tile_sums, x->ntiles_max);
  const uint32_t* mk = where == 0 ? x->keys[1] : d.scr_p;
  const uint32_t* mvp = where == 0 ? x->vals[1] : d.scr_j;
  const int pgrid = 148 * 8;  // CTAs over the touched pages (persistent loop)
  Fields& cur = x->buf[x->cur];
  Fields& other = x->buf[1 - x->cur];
  // grid-stride kernels over the movers, whose count only the device knows: one wave of CTAs
  const int mgrid = 148 * 8;
  k_mv_gather<<<mgrid, 256, 0, s>>>(d, cur, mvp, x->mv_count);
  k_pg_touch<<<mgrid, 256, 0, s>>>(d, mk, mvp, x->mv_count);
  k_mv_runs<<<mgrid, 256, 0, s>>>(d, mk, x->mv_count);
  k_pg_plan<<<pgrid, 256, 0, s>>>(d, mk, mvp, x->mv_count);
  k_grave_movers<<<mgrid, 256, 0, s>>>(d, x->mv_count);
  k_grave_movers_commit<<<1, 1, 0, s>>>(d, x->mv_count);
  k_pg_write<false><<<pgrid, 256, 0, s>>>(d, cur, mk, mvp, x->mv_count, d.pstart);
  x->launches += 7;
  // the repack path: its kernels return at once unless k_pg_plan chose it
  k_pg_sizes_repack<<<pgrid, 256, 0, s>>>(d, mk, mvp, x->mv_count, x->pstart_new);
  x->launches += 1;
  scan_u32(x, x->pstart_new, d.npages, x->ps_tsums);
  k_pg_write<true><<<pgrid, 256, 0, s>>>(d, other, mk, mvp, x->mv_count, x->pstart_new);
  k_pg_copy_back<<<mgrid, 256, 0, s>>>(d, other, x->pstart_new);
  k_pg_commit<<<grid_for((size_t)d.npages + 1, 256), 256, 0, s>>>(d, x->pstart_new);
  x->launches += 3;
  CUDA_TRY(cudaGetLastError());
  return CLEO_OK;
}

// stable radix sort of (key, value) pairs whose count is *n_ptr (device), over `bits` key bits,
// from (k0, v0) using (k1, v1) as the other buffer; returns 0 if the result is in (k0, v0)
// with explicit digit-table scratch for nt tiles (hist: 256 nt words, tile_sums: enough for the
// scan of the table)
int radix_pairs_on(cleo_b200_ctx* x, uint32_t* k0, uint32_t* v0, uint32_t* k1, uint32_t* v1,
                   const uint32_t* n_ptr, uint32_t bits, uint32_t* hist, uint32_t* tile_sums,
                   uint32_t nt, uint32_t unsorted_max) {
  cudaStream_t s = x->stream;
  const uint64_t nh = (uint64_t)256 * nt;
  const uint32_t nscan_tiles = (uint32_t)((nh + SCAN_TILE - 1) / SCAN_TILE);
  int cur = 0;
  uint32_t* K[2] = {k0, k1};
  uint32_t* V[2] = {v0, v1};
  // counts up to RS_SMALL_MAX (the usual mover list) are sorted by one block; the multi-tile passes
  // below then return at once, and the other way round
  // (with unsorted_max, counts up to it stay as they are: a caller for whom the order is only a
  // schedule, and an even number of passes, so that the sorted result would be in place too)
  k_rs_small<<<1, RS_SMALL_THREADS, 0, s>>>(k0, v0, k1, v1, n_ptr, bits, unsorted_max);
  x->launches += 1;
  constexpr uint32_t SMALL = RS_SMALL_MAX;
  for (uint32_t shift = 0; shift < bits; shift += 8) {
    k_rs_upsweep<<<nt, RS_THREADS, 0, s>>>(K[cur], n_ptr, (int)shift, hist, nt, SMALL);
    k_scan_tiles<<<nscan_tiles, SCAN_THREADS, 0, s>>>(hist, hist, nh, tile_sums, n_ptr, SMALL);
    k_scan_sums<<<1, SCAN_THREADS, 0, s>>>(tile_sums, nscan_tiles, nullptr, n_ptr, SMALL);
    k_scan_add<<<(unsigned)((nh + 255) / 256), 256, 0, s>>>(hist, nh, tile_sums, n_ptr, SMALL);
    k_rs_downsweep<<<nt, RS_THREADS, 0, s>>>(K[cur], V[cur], n_ptr, (int)shift, hist, nt,
                                             K[1 - cur], V[1 - cur], SMALL);
    x->launches += 5;
    cur = 1 - cur;
  }
  return cur;
}
int radix_pairs(cleo_b200_ctx* x, uint32_t* k0, uint32_t* v0, uint32_t* k1, uint32_t* v1,
                const uint32_t* n_ptr, uint32_t bits, uint32_t unsorted_max = 0) {
  return radix_pairs_on(x, k0, v0, k1, v1, n_ptr, bits, x->hist, x->tile_sums, x->ntiles_max,
                        unsorted_max);
}

// the microphysics of one SDM step on the batched schedule (batched.cuh)
int run_batched_micro(cleo_b200_ctx* x, uint32_t t_sdm, uint32_t t_sdm_next, bool did_motion) {
  DevCtx& d = x->d;
  BatchScratch& b = x->bs;
  b.small_max = x->cfg.small_max;
  b.medium_max = MEDIUM_MAX;
  cudaStream_t s = x->stream;
  StageMark m(x, 2);
  const int gg = grid_for(d.ngbxs, 256);
  // warps of 32 gridboxes each
  const int gw = grid_for(((size_t)d.ngbxs + 31) / 32 * 32, SEQ_THREADS);
  // qcond from the moved superdroplets: summed by the first condensation sub-step's commit when
  // it starts the step (pass A stores each droplet's condensate mass before its solve), else here
  const bool fuse_qcond = did_motion && on_step(d.p.condstep, t_sdm);
  if (did_motion && !fuse_qcond) {
    k_b_qcond<<<gw, SEQ_THREADS, 0, s>>>(d);
    x->launches += 1;
  }
  b.qm = nullptr;
  BatchScratch bq = b;  // the first sub-step's scratch
  bq.qm = fuse_qcond ? x->qm_buf : nullptr;
  // every gridbox's RNG slot from 0 at the step's start (a one-gridbox domain's was reset by the
  // previous step's k_b_advance_t, or at creation)
  if (!x->one_box) {
    k_b_reset<<<gg, 256, 0, s>>>(d, b, 1);
    x->launches += 1;
  }
  uint32_t subt = t_sdm;
  while (subt < t_sdm_next) {
    const bool cond = on_step(d.p.condstep, subt);
    const bool coll = on_step(d.p.collstep, subt);
    if (cond) {
      StageMark mc(x, 3);
      const BatchScratch& bc = subt == t_sdm ? bq : b;  // qcond with the first sub-step's commit
      k_b_thermo<<<gg, 256, 0, s>>>(d, b);
      x->launches += 1;
      if (x->cfg.cond_minb == 5)
        k_cond_a<5><<<grid_for(d.slots, x->cfg.cond_block), x->cfg.cond_block, 0, s>>>(d, bc);
      else if (x->cfg.cond_minb == 4)
        k_cond_a<4><<<grid_for(d.slots, x->cfg.cond_block), x->cfg.cond_block, 0, s>>>(d, bc);
      else
        k_cond_a<3><<<grid_for(d.slots, x->cfg.cond_block), x->cfg.cond_block, 0, s>>>(d, bc);
      x->launches += 1;
      // 16 key bits: two passes, result back in place. The order (most expensive solves first)
      // balances pass B's load; a list of up to RS_SMALL_MAX solves runs at once on pass B's
      // resident threads whatever its order, so it stays unsorted, unless the surrogate needs
      // its restarts at the front
      const uint32_t unsorted_max = d.p.nr_seed == CLEO_NRSEED_MLP ? 0u : RS_SMALL_MAX;
      const int where =
          radix_pairs(x, b.lkeys, b.lvals, x->keys[1], x->vals[1], b.ctr, 16, unsorted_max);
      if (where != 0) return CLEO_ERR_CUDA;
      if (d.p.nr_seed == CLEO_NRSEED_MLP) {
        // the surrogate seeds only the direct solves pass A left unconverged, in b.dm
        mlp::Infer w;
        if (cleo_mlp_infer_view(x->mlp, &w) != CLEO_OK) return CLEO_ERR_MLP;
        w.err = reinterpret_cast<uint32_t*>(&d.err->code);
        const SdmListSeedIO io{d.sd.gbx, d.sd.r,  d.sd.msol, d.temp, d.press, b.th_s,
                               d.p.cond_delt, b.lvals, b.ctr + 9, b.dm};
        const uint32_t tiles = (d.slots + mlp::TILE_M - 1) / mlp::TILE_M;
        mlp::k_mlp_tc<SdmListSeedIO><<<tiles < mlp::TC_GRID_MAX ? tiles : mlp::TC_GRID_MAX, 128, mlp::TC_SMEM,
                                       s>>>(w, io, d.slots);
        x->launches += 1;
      }
      {  // pass B in its own tuned variant (grid: twice its resident CTAs)
        StageMark mb(x, STAGE_COND_B);
        if (x->cfg.condb_minb >= 5)
          k_cond_b<5><<<x->grid_condb[2], 256, 0, s>>>(d, b);
        else if (x->cfg.condb_minb == 4)
          k_cond_b<4><<<x->grid_condb[1], 256, 0, s>>>(d, b);
        else
          k_cond_b<3><<<x->grid_condb[0], 256, 0, s>>>(d, b);
      }
      // every gridbox's condensed mass summed in order, its state updated (the gridboxes of
      // more than SEQ_BIG superdroplets by a warp each)
      k_b_commit<<<gw, SEQ_THREADS, 0, s>>>(d, bc);
      k_b_commit_big<<<x->sms * 4, SEQ_THREADS, 0, s>>>(d, bc);
      x->launches += 3;
    }
    if (coll && x->one_box) {  // the one gridbox's collision step over the whole GPU
      StageMark mk(x, 4);
      const OneBox& o = x->ob;
      const int go = grid_for((size_t)d.slots + 1, 256);
      if (d.p.coll_prob == CLEO_PROB_LONG) {  // otherwise the pair terminal velocities stay 0
        k_b_tv<<<grid_for(d.slots, 256), 256, 0, s>>>(d, b);
        x->launches += 1;
      }
      // scans of n + 1 entries (entries past n unused): one block while the slots allow
      const bool one_block = (uint64_t)d.slots + 1 <= OB_SCAN_MAX;
      const auto scan = [&](uint32_t* a, const uint32_t* skip) {
        if (one_block) {
          k_ob_scan<<<1, SCAN_THREADS, 0, s>>>(d, a, skip);
          x->launches += 1;
        } else {
          scan_u32(x, a, d.slots + 1, o.tsums);
        }
      };
      const bool front = d.slots <= OB_FRONT_MAX;
      if (front) {  // draws, counting sort, chains and their walks in one block
        k_ob_front<<<1, OB_FRONT_THREADS, ob_front_smem(d.slots), s>>>(d, b, o);
        x->launches += 1;
      } else {
        k_ob_draw<<<go, 256, 0, s>>>(d, b, o);
        x->launches += 1;
        scan(o.cnt, nullptr);  // bucket starts
        k_ob_place<<<go, 256, 0, s>>>(d, o);
        k_ob_chains<<<go, 256, 0, s>>>(d, o);
        x->launches += 2;
      }
      k_ob_pairs<<<go, 256, 0, s>>>(d, b, o, front ? 1 : 0);
      x->launches += 1;
      scan(o.vflag, o.ninv);  // valid ones before each shuffled position (none to count: left out)
      k_ob_gather<<<go, 256, 0, s>>>(d, o);
      k_ob_commit<<<go, 256, 0, s>>>(d, b, o);
      x->launches += 2;
    } else if (coll) {
      StageMark mk(x, 4);
      k_b_reset<<<1, 32, 0, s>>>(d, b, 0);
      k_b_classify<<<gg, 256, 0, s>>>(d, b);
      if (d.p.coll_prob == CLEO_PROB_LONG) {  // otherwise the pair terminal velocities stay 0
        k_b_tv<<<grid_for(d.slots, 256), 256, 0, s>>>(d, b);
        x->launches += 1;
      }
      // the warp kernel's 64-slot variant takes gridboxes up to 64 superdroplets, its 128-slot
      // variant those of 65 .. small_max (when small_max > 64)
      const int wide = x->cfg.small_max > SMALL_MAX ? 1 : 0, m3 = x->cfg.small_minb == 3 ? 1 : 0;
      constexpr uint32_t SW = SmallLayout<WARP_MAX>::BYTES, SS = SmallLayout<SMALL_MAX>::BYTES;
      if (m3)
        k_b_small<3, SMALL_MAX><<<x->grid_small[1], B_THREADS, SS, s>>>(d, b, 0);
      else
        k_b_small<2, SMALL_MAX><<<x->grid_small[0], B_THREADS, SS, s>>>(d, b, 0);
      // the 128-slot variant at 2 CTAs per SM whatever the 64-slot one's budget: at 3 it spills
      // (measured: collisions 3.87 ms with both at 2, 3.67 ms with the 64-slot one at 3)
      if (wide) k_b_small<2, WARP_MAX><<<x->grid_wide, B_THREADS, SW, s>>>(d, b, 1);
      x->launches += wide;
      k_b_cta<false><<<x->grid_medium, B_THREADS, (size_t)MEDIUM_SMEM, s>>>(d, b);
      k_b_cta<true><<<x->grid_large, LARGE_THREADS, LARGE_SMEM, s>>>(d, b);
      x->launches += 5;
    }
    subt = min(next_step(d.p.condstep, subt), next_step(d.p.collstep, subt));
  }
  k_b_advance_t<<<1, 1, 0, s>>>(b, t_sdm_next - t_sdm, x->one_box ? 1 : 0);
  x->launches += 1;
  CUDA_TRY(cudaGetLastError());
  return CLEO_OK;
}

int run_sdm_step(cleo_b200_ctx* x, uint32_t t_sdm, uint32_t t_sdm_next) {
  DevCtx& d = x->d;
  cudaStream_t s = x->stream;
  const bool did_motion = on_step(d.p.motionstep, t_sdm);
  const int gg = grid_for(d.ngbxs, 256);
  const bool mon_mm =
      (d.p.monitors & (CLEO_MONITOR_MASSMOMENTS | CLEO_MONITOR_RAINMASSMOMENTS)) != 0;
  if (did_motion) {
    {
      StageMark m(x, 0);
      const bool inc = !x->sort_full;
      CUDA_TRY(cudaMemsetAsync(d.mv_total, 0, 4, s));
      k_motion<<<grid_for(d.slots, 256), 256, 0, s>>>(d, x->keys[0], x->vals[0], inc ? 1 : 0);
      k_mv_report<<<1, 1, 0, s>>>(d, x->d_motion);
      x->launches += 2;
      {  // inside a captured step the record becomes an external event node of the graph
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        CUDA_TRY(cudaStreamIsCapturing(s, &cs));
        if (cs == cudaStreamCaptureStatusActive)
          CUDA_TRY(cudaEventRecordWithFlags(x->ev_report, s, cudaEventRecordExternal));
        else
          CUDA_TRY(cudaEventRecord(x->ev_report, s));
      }
      x->report_recorded = true;
      if (d.p.monitors & CLEO_MONITOR_PRECIPITATION) {  // before the sort moves the droplets
        k_mon_precip<<<gg, 256, 0, s>>>(d);
        x->launches += 1;
      }
    }
    StageMark m(x, 1);
    const int rc = x->sort_full ? sort_current(x) : sort_incremental(x);
    if (rc) return rc;
    if (mon_mm) {  // monitor_motion (movesupersindomain.hpp:297)
      k_mon_mm<<<gg, 256, 0, s>>>(d, 1, 0);
      x->launches += 1;
    }
  }
  const bool micro = (d.p.condstep != CLEO_STEP_OFF || d.p.collstep != CLEO_STEP_OFF);
  if (d.p.exec_mode == CLEO_EXEC_BATCHED) {
    const int rc = run_batched_micro(x, t_sdm, t_sdm_next, did_motion);
    if (rc == CLEO_OK && mon_mm) {  // monitor_microphysics (sdmmethods.hpp:76)
      k_mon_mm<<<gg, 256, 0, s>>>(d, 0, 0);
      x->launches += 1;
    }
    return rc;
  }
  if (micro || did_motion) {
    const uint32_t blocks = d.ngbxs < (1u << 30) ? d.ngbxs : (1u << 30);
    if (blocks > 0) {
      StageMark m(x, 2);
      k_micro<<<blocks, MICRO_THREADS, MICRO_SMEM, s>>>(d, t_sdm, t_sdm_next, did_motion ? 1 : 0);
      x->launches += 1;
    }
  }
  if (mon_mm) {
    k_mon_mm<<<gg, 256, 0, s>>>(d, 0, 0);
    x->launches += 1;
  }
  CUDA_TRY(cudaGetLastError());
  return CLEO_OK;
}

// ---- autotuner ----
// Candidate launch configurations are timed on live batched steps (per-stage CUDA events): the
// condensation options (pass-A block, pass-B grid) and the collision options (bucket
// thresholds) are scored independently and the fastest of each kept. Chosen configurations are
// cached per process by GPU name and domain size, so later contexts start from them.
std::mutex g_tune_mutex;
std::map<std::string, cleo_b200_ctx::TuneCfg> g_tune_cache;

const cleo_b200_ctx::TuneCfg COND_OPTS[4] = {
    {128, 4, 0, 0, 3}, {256, 4, 0, 0, 4}, {128, 5, 0, 0, 5}, {256, 5, 0, 0, 3}};
const cleo_b200_ctx::TuneCfg COLL_OPTS[4] = {
    {0, 0, SMALL_MAX, 2, 0}, {0, 0, WARP_MAX, 2, 0}, {0, 0, SMALL_MAX, 3, 0},
    {0, 0, WARP_MAX, 3, 0}};

std::string tune_key(const cleo_b200_ctx* x) {
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, x->device) != cudaSuccess) return std::string();
  uint32_t lg = 0;
  while ((1ull << lg) < (unsigned long long)x->d.capacity) ++lg;
  return std::string(prop.name) + "|" + std::to_string(x->d.ngbxs) + "|" + std::to_string(lg);
}

// one tuning step: run the step eagerly with stage events, score the candidate, and when all
// candidates have been timed choose the fastest
int run_tuning_step(cleo_b200_ctx* x, uint32_t t_sdm, uint32_t t_sdm_next) {
  const size_t k = x->tune_step % 4;
  x->cfg.cond_block = COND_OPTS[k].cond_block;
  x->cfg.cond_minb = COND_OPTS[k].cond_minb;
  x->cfg.condb_minb = COND_OPTS[k].condb_minb;
  x->cfg.small_max = COLL_OPTS[k].small_max;
  x->cfg.small_minb = COLL_OPTS[k].small_minb;
  const bool prof = x->profiling;
  const size_t m0 = x->marks.size();
  x->profiling = true;
  const int rc = run_sdm_step(x, t_sdm, t_sdm_next);
  x->profiling = prof;
  CUDA_TRY(cudaStreamSynchronize(x->stream));
  double tc = 0.0, tb = 0.0, tl = 0.0;
  for (size_t i = m0; i < x->marks.size(); ++i) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, x->marks[i].a, x->marks[i].b);
    if (x->marks[i].stage == 3) tc += ms;
    if (x->marks[i].stage == STAGE_COND_B) tb += ms;
    if (x->marks[i].stage == 4) tl += ms;
    if (!prof) {
      x->event_pool.push_back(x->marks[i].a);
      x->event_pool.push_back(x->marks[i].b);
    }
  }
  if (!prof) x->marks.resize(m0);
  if (rc != CLEO_OK) return rc;
  x->t_cond[k] += tc - tb;  // pass A and the rest of the stage
  x->t_condb[k] += tb;
  x->t_coll[k] += tl;
  if (++x->tune_step == x->tune_total) {
    size_t bc = 0, bb = 0, bl = 0;
    for (size_t i = 1; i < 4; ++i) {
      if (x->t_cond[i] < x->t_cond[bc]) bc = i;
      if (x->t_condb[i] < x->t_condb[bb]) bb = i;
      if (x->t_coll[i] < x->t_coll[bl]) bl = i;
    }
    x->cfg = {COND_OPTS[bc].cond_block, COND_OPTS[bc].cond_minb, COLL_OPTS[bl].small_max,
              COLL_OPTS[bl].small_minb, COND_OPTS[bb].condb_minb};
    x->tune_total = 0;
    x->drop_graphs();
    std::lock_guard<std::mutex> lock(g_tune_mutex);
    g_tune_cache[x->tune_key] = x->cfg;
  }
  return CLEO_OK;
}

// The launch sequence of one batched SDM step as a CUDA graph: captured the first time a
// signature is seen, replayed afterwards. The injected random numbers are keyed by the device
// word bs.tsdm, so a replay needs no parameter update.
int run_step_graphed(cleo_b200_ctx* x, uint32_t t_sdm, uint32_t t_sdm_next) {
  const cleo_b200_params& p = x->d.p;
  std::vector<uint32_t> sig;
  sig.push_back((uint32_t)x->cur);
  sig.push_back((on_step(p.motionstep, t_sdm) ? 1u : 0u) | (x->sort_full ? 2u : 0u));
  sig.push_back(t_sdm_next - t_sdm);
  for (uint32_t subt = t_sdm; subt < t_sdm_next;
       subt = min(next_step(p.condstep, subt), next_step(p.collstep, subt))) {
    sig.push_back(subt - t_sdm);
    sig.push_back((on_step(p.condstep, subt) ? 1u : 0u) | (on_step(p.collstep, subt) ? 2u : 0u));
  }
  for (auto& g : x->graphs) {
    if (g.sig == sig) {
      CUDA_TRY(cudaGraphLaunch(g.exec, x->stream));
      x->cur = g.cur_after;
      x->d.sd = x->buf[x->cur];
      x->launches += g.nodes;
      return CLEO_OK;
    }
  }
  if (x->graphs.size() >= 8) x->drop_graphs();
  const int cur0 = x->cur;
  const unsigned long long l0 = x->launches;
  CUDA_TRY(cudaStreamBeginCapture(x->stream, cudaStreamCaptureModeThreadLocal));
  const int rc = run_sdm_step(x, t_sdm, t_sdm_next);
  cudaGraph_t graph = nullptr;
  const cudaError_t ce = cudaStreamEndCapture(x->stream, &graph);
  const unsigned long long nodes = x->launches - l0;
  x->launches = l0;
  const int cur_after = x->cur;
  x->cur = cur0;  // nothing has run yet
  x->d.sd = x->buf[x->cur];
  cudaGraphExec_t exec = nullptr;
  if (rc != CLEO_OK || ce != cudaSuccess || !graph ||
      cudaGraphInstantiate(&exec, graph, 0) != cudaSuccess) {
    if (graph) cudaGraphDestroy(graph);
    cudaGetLastError();
    return rc != CLEO_OK ? rc : CLEO_ERR_CUDA;
  }
  cudaGraphDestroy(graph);
  x->graphs.push_back({sig, exec, cur_after, nodes});
  CUDA_TRY(cudaGraphLaunch(exec, x->stream));
  x->cur = cur_after;
  x->d.sd = x->buf[x->cur];
  x->launches += nodes;
  return CLEO_OK;
}

}  // namespace

extern "C" {

const char* cleo_b200_version(void) { return "cleo_b200 0.1 (sm_100a)"; }

int cleo_b200_create(const cleo_b200_params* params, const cleo_b200_grid* grid, size_t capacity,
                     cleo_b200_ctx** out) {
  if (!params || !grid || !out) return CLEO_ERR_ARGUMENT;
  if (capacity >= 0xFFFFFFFFull || grid->ngbxs >= 0xFFFFFFF0u) return CLEO_ERR_CAPACITY;
  // the SoA buffers hold the pages' free slots too (pages.cuh)
  const uint64_t npages = ((uint64_t)grid->ngbxs + PAGE_GBXS - 1) / PAGE_GBXS;
  if ((uint64_t)capacity + (npages ? npages : 1) * PAGE_SLACK >= 0xFFFFFFF0ull)
    return CLEO_ERR_CAPACITY;
  if (params->condstep != CLEO_STEP_OFF && params->cond_delt < params->cond_minsubdelt)
    return CLEO_ERR_SUBDELT;  // ImplicitEuler ctor, impliciteuler.hpp:320-326
  if (params->condstep == 0 || params->collstep == 0 || params->motionstep == 0)
    return CLEO_ERR_ARGUMENT;
  // the surrogate seeds the batched schedule; the plain schedule is the unseeded form
  if (params->nr_seed == CLEO_NRSEED_MLP && params->exec_mode != CLEO_EXEC_BATCHED)
    return CLEO_ERR_ARGUMENT;
  if (params->nr_seed != CLEO_NRSEED_REFERENCE && params->nr_seed != CLEO_NRSEED_MLP)
    return CLEO_ERR_ARGUMENT;
  // a sub-stepping loop needs a positive minimum sub-step, and Newton solves a finite budget
  if (params->condstep != CLEO_STEP_OFF &&
      (!(params->cond_minsubdelt > 0.0) || params->maxniters > 1000000u))
    return CLEO_ERR_ARGUMENT;
  if ((uint64_t)grid->ndims[0] * grid->ndims[1] * grid->ndims[2] != grid->ngbxs ||
      grid->ndims[0] == 0 || grid->ndims[1] == 0 || grid->ndims[2] == 0)
    return CLEO_ERR_ARGUMENT;
  auto* x = new (std::nothrow) cleo_b200_ctx();
  if (!x) return CLEO_ERR_CAPACITY;
  CUDA_TRY(cudaGetDevice(&x->device));
  DevCtx& d = x->d;
  d.p = *params;
  d.ngbxs = grid->ngbxs;
  for (int i = 0; i < 3; ++i) d.ndims[i] = grid->ndims[i];
  d.capacity = (uint32_t)capacity;
  d.npages = (uint32_t)(npages ? npages : 1);
  d.slots = (uint32_t)(capacity + (size_t)d.npages * PAGE_SLACK);
  const size_t ng = grid->ngbxs, cap = d.slots;  // position-indexed arrays cover every slot
  int rc = 0;
  double* maps[6];
  for (int k = 0; k < 6; ++k) rc |= dalloc(x, &maps[k], ng);
  uint32_t* nb[6];
  for (int k = 0; k < 6; ++k) rc |= dalloc(x, &nb[k], ng);
  double* st[11];
  for (int k = 0; k < 11; ++k) rc |= dalloc(x, &st[k], ng);
  rc |= dalloc(x, &d.cond_mass, ng);
  rc |= dalloc(x, &d.nr_iters, ng);
  rc |= alloc_fields(x, x->buf[0], cap);
  rc |= alloc_fields(x, x->buf[1], cap);
  rc |= alloc_fields(x, d.grave, capacity);
  rc |= alloc_fields(x, d.mvrec, capacity);
  rc |= dalloc(x, &d.pstart, (size_t)d.npages + 1);
  rc |= dalloc(x, &d.pg_flag, d.npages);
  rc |= dalloc(x, &d.pg_list, d.npages);
  rc |= dalloc(x, &d.pg_ctr, 4);
  rc |= dalloc(x, &d.mv_lo, d.ngbxs);
  rc |= dalloc(x, &d.mv_hi, d.ngbxs);
  rc |= dalloc(x, &d.mv_stamp, d.ngbxs);
  rc |= dalloc(x, &x->pstart_new, (size_t)d.npages + 1);
  rc |= dalloc(x, &x->ps_tsums, ((size_t)d.npages + SCAN_TILE) / SCAN_TILE + 1);
  rc |= dalloc(x, &d.gstart, ng + 2);
  rc |= dalloc(x, &d.gcount, ng);
  rc |= dalloc(x, &d.counters, 4);
  rc |= dalloc(x, &d.scr_r, cap);
  rc |= dalloc(x, &d.scr_m, cap);
  rc |= dalloc(x, &d.scr_c3, cap);
  rc |= dalloc(x, &d.scr_c1, cap);
  rc |= dalloc(x, &d.scr_c2, cap);
  rc |= dalloc(x, &d.scr_x, cap);
  rc |= dalloc(x, &d.scr_id, cap);
  rc |= dalloc(x, &d.scr_p, cap);
  rc |= dalloc(x, &d.scr_j, cap);
  rc |= dalloc(x, &d.err, 1);
  x->ntiles_max = (uint32_t)((cap + RS_TILE - 1) / RS_TILE);
  if (x->ntiles_max == 0) x->ntiles_max = 1;
  for (int k = 0; k < 2; ++k) {
    rc |= dalloc(x, &x->keys[k], cap);
    rc |= dalloc(x, &x->vals[k], cap);
  }
  rc |= dalloc(x, &x->hist, (size_t)256 * x->ntiles_max);
  rc |= dalloc(x, &x->bs.th_s, ng);
  rc |= dalloc(x, &x->bs.th_ff, ng);
  rc |= dalloc(x, &x->bs.th_ak, ng);
  rc |= dalloc(x, &x->bs.th_a3, ng);
  rc |= dalloc(x, &x->bs.th_u3, ng);
  rc |= dalloc(x, &x->bs.dm, cap);
  rc |= dalloc(x, &x->bs.its, cap);
  rc |= dalloc(x, &x->bs.tv, cap + 2);
  rc |= dalloc(x, &x->qm_buf, cap);
  if (ng == 1) {  // one gridbox: its collisions by the whole GPU (onebox.cuh)
    OneBox& o = x->ob;
    for (uint32_t** q : {&o.J, &o.cnt, &o.fill, &o.bkt, &o.first, &o.next, &o.P, &o.vflag})
      rc |= dalloc(x, q, cap + 2);
    rc |= dalloc(x, &o.tsums, (cap + 2 + SCAN_TILE - 1) / SCAN_TILE + 1);
    rc |= dalloc(x, &o.nnull, 1);
    rc |= dalloc(x, &o.ninv, 1);
    rc |= dalloc(x, &o.nstep, 1);
    x->one_box = true;
  }
  rc |= dalloc(x, &x->bs.zres, cap);
  rc |= dalloc(x, &x->bs.ffv, cap);
  rc |= dalloc(x, &x->bs.lkeys, cap);
  rc |= dalloc(x, &x->bs.lvals, cap);
  rc |= dalloc(x, &x->bs.bucket, 4 * ng);
  rc |= dalloc(x, &x->bs.big, ng);
  rc |= dalloc(x, &x->bs.brec, 2 * ng);
  rc |= dalloc(x, &x->bs.slot, ng);
  rc |= dalloc(x, &x->bs.ctr, 12);
  rc |= dalloc(x, &x->bs.tsdm, 1);
  rc |= dalloc(x, &x->tile_sums, ((size_t)256 * x->ntiles_max + SCAN_TILE - 1) / SCAN_TILE + 1);
  rc |= dalloc(x, &d.mv_scan, ((size_t)cap + 31) / 32 + 1);
  rc |= dalloc(x, &d.mv_mask, ((size_t)cap + 31) / 32);
  rc |= dalloc(x, &d.mv_total, 1);
  if (cudaHostAlloc(&x->h_motion, 2 * sizeof(uint32_t), cudaHostAllocMapped) != cudaSuccess ||
      cudaHostGetDevicePointer(&x->d_motion, x->h_motion, 0) != cudaSuccess ||
      cudaEventCreateWithFlags(&x->ev_report, cudaEventDisableTiming) != cudaSuccess)
    rc |= CLEO_ERR_CUDA;
  else
    x->h_motion[0] = x->h_motion[1] = 0;
  rc |= dalloc(x, &d.gstart_new, (size_t)ng + 2);
  rc |= dalloc(x, &x->mv_count, 1);
  {
    const size_t a = ((size_t)cap + 1 + SCAN_TILE - 1) / SCAN_TILE, b = ((size_t)ng + SCAN_TILE) / SCAN_TILE;
    rc |= dalloc(x, &d.mv_tsums, a + 1);
    rc |= dalloc(x, &x->gs_tsums, b + 1);
  }
  if (params->monitors) {
    for (int r = 0; r < 2; ++r) {
      for (int w = 0; w < 2; ++w) {
        rc |= dalloc(x, &d.mm0[r][w], ng);
        rc |= dalloc(x, &d.mm1[r][w], ng);
        rc |= dalloc(x, &d.mm2[r][w], ng);
      }
      rc |= dalloc(x, &d.prev0[r], ng);
      rc |= dalloc(x, &d.prev1[r], ng);
      rc |= dalloc(x, &d.prev2[r], ng);
    }
    rc |= dalloc(x, &d.precip, ng);
    rc |= dalloc(x, &d.gbxarea, ng);
    if (params->monitors & CLEO_MONITOR_PRECIPITATION) rc |= dalloc(x, &d.precip_c, cap);
  }
  if (rc) {
    cleo_b200_destroy(x);
    return CLEO_ERR_CUDA;
  }
  // key bits: keys run over [0, ngbxs]
  uint32_t bits = 0;
  while (bits < 32 && (((uint64_t)1 << bits) <= (uint64_t)ng)) ++bits;
  x->key_bits = bits == 0 ? 8 : ((bits + 7) / 8) * 8;
  d.b3lo = maps[0]; d.b3hi = maps[1]; d.b1lo = maps[2]; d.b1hi = maps[3]; d.b2lo = maps[4]; d.b2hi = maps[5];
  d.back3 = nb[0]; d.fwd3 = nb[1]; d.back1 = nb[2]; d.fwd1 = nb[3]; d.back2 = nb[4]; d.fwd2 = nb[5];
  d.volume = st[0]; d.press = st[1]; d.temp = st[2]; d.qvap = st[3]; d.qcond = st[4];
  d.wlo = st[5]; d.whi = st[6]; d.ulo = st[7]; d.uhi = st[8]; d.vlo = st[9]; d.vhi = st[10];
  d.sd = x->buf[0];
  CUDA_TRY(cudaStreamCreateWithFlags(&x->stream, cudaStreamNonBlocking));
  x->own_stream = true;
  const double* src_maps[6] = {grid->coord3lo, grid->coord3hi, grid->coord1lo,
                               grid->coord1hi, grid->coord2lo, grid->coord2hi};
  const uint32_t* src_nb[6] = {grid->back3, grid->fwd3, grid->back1, grid->fwd1, grid->back2, grid->fwd2};
  for (int k = 0; k < 6; ++k) {
    if (!src_maps[k] || !src_nb[k]) {
      cleo_b200_destroy(x);
      return CLEO_ERR_ARGUMENT;
    }
    CUDA_TRY(cudaMemcpyAsync(maps[k], src_maps[k], ng * 8, cudaMemcpyHostToDevice, x->stream));
    CUDA_TRY(cudaMemcpyAsync(nb[k], src_nb[k], ng * 4, cudaMemcpyHostToDevice, x->stream));
  }
  CUDA_TRY(cudaMemsetAsync(d.cond_mass, 0, ng * 8, x->stream));
  CUDA_TRY(cudaMemsetAsync(d.nr_iters, 0, ng * 8, x->stream));
  CUDA_TRY(cudaMemsetAsync(d.counters, 0, 16, x->stream));
  CUDA_TRY(cudaMemsetAsync(d.gstart, 0, (ng + 2) * 4, x->stream));
  CUDA_TRY(cudaMemsetAsync(d.gcount, 0, (ng ? ng : 1) * 4, x->stream));
  CUDA_TRY(cudaMemsetAsync(d.pstart, 0, ((size_t)d.npages + 1) * 4, x->stream));
  CUDA_TRY(cudaMemsetAsync(d.pg_flag, 0, (size_t)d.npages * 4, x->stream));
  CUDA_TRY(cudaMemsetAsync(d.pg_ctr, 0, 16, x->stream));
  CUDA_TRY(cudaMemsetAsync(d.mv_stamp, 0, (size_t)d.ngbxs * 4, x->stream));
  // pair terminal velocities: 0 unless the Long kernel's k_b_tv writes them
  CUDA_TRY(cudaMemsetAsync(x->bs.tv, 0, ((size_t)d.slots + 2) * 8, x->stream));
  if (x->one_box) {  // the one-box counts start at zero (k_ob_gather clears what a step used)
    CUDA_TRY(cudaMemsetAsync(x->ob.cnt, 0, ((size_t)d.slots + 2) * 4, x->stream));
    CUDA_TRY(cudaMemsetAsync(x->ob.fill, 0, ((size_t)d.slots + 2) * 4, x->stream));
  }
  CUDA_TRY(cudaMemsetAsync(d.err, 0, sizeof(DevError), x->stream));
  CUDA_TRY(cudaFuncSetAttribute(k_micro, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)MICRO_SMEM));
  CUDA_TRY(cudaMemsetAsync(x->bs.ctr, 0, 48, x->stream));
  CUDA_TRY(cudaMemsetAsync(x->bs.tsdm, 0, 4, x->stream));
  CUDA_TRY(cudaMemsetAsync(x->bs.slot, 0, (ng ? ng : 1) * 4, x->stream));
  if (params->monitors) {  // gridbox areas (GbxBoundsFromBinary::gbxarea) and zeroed monitors
    std::vector<double> area(ng ? ng : 1, 0.0);
    for (uint32_t i = 0; i < ng; ++i)
      area[i] = grid->gbxarea ? grid->gbxarea[i]
                              : (grid->coord1hi[i] - grid->coord1lo[i]) *
                                    (grid->coord2hi[i] - grid->coord2lo[i]);
    CUDA_TRY(cudaMemcpyAsync(d.gbxarea, area.data(), ng * 8, cudaMemcpyHostToDevice, x->stream));
    CUDA_TRY(cudaStreamSynchronize(x->stream));  // area is a host temporary
    const int rc2 = cleo_b200_monitors_begin(x);
    if (rc2 != CLEO_OK) {
      cleo_b200_destroy(x);
      return rc2;
    }
  }
  {  // persistent grids of the batched kernels: full occupancy on every SM
    int dev = 0, sms = 148, occ = 1;
    CUDA_TRY(cudaGetDevice(&dev));
    CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    x->sms = sms;
    constexpr int SW = (int)SmallLayout<WARP_MAX>::BYTES, SS = (int)SmallLayout<SMALL_MAX>::BYTES;
    CUDA_TRY(cudaFuncSetAttribute(k_b_small<2, SMALL_MAX>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, SS));
    CUDA_TRY(cudaFuncSetAttribute(k_b_small<3, SMALL_MAX>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, SS));
    CUDA_TRY(cudaFuncSetAttribute(k_b_small<2, WARP_MAX>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, SW));
    CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_b_small<2, SMALL_MAX>,
                                                           B_THREADS, SS));
    x->grid_small[0] = sms * (occ > 0 ? occ : 1);
    CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_b_small<3, SMALL_MAX>,
                                                           B_THREADS, SS));
    x->grid_small[1] = sms * (occ > 0 ? occ : 1);
    CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_b_small<2, WARP_MAX>,
                                                           B_THREADS, SW));
    x->grid_wide = sms * (occ > 0 ? occ : 1);
    CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_b_cta<false>, B_THREADS,
                                                           (size_t)MEDIUM_SMEM));
    x->grid_medium = sms * (occ > 0 ? occ : 1);
    CUDA_TRY(cudaFuncSetAttribute(k_b_cta<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)LARGE_SMEM));
    if (x->one_box && x->d.slots <= OB_FRONT_MAX)  // at most 219 KB of tables
      CUDA_TRY(cudaFuncSetAttribute(k_ob_front, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)ob_front_smem(x->d.slots)));
    CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_b_cta<true>, LARGE_THREADS,
                                                           LARGE_SMEM));
    x->grid_large = sms * (occ > 0 ? occ : 1);
    CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_cond_b<3>, 256, 0));
    x->grid_condb[0] = 2 * sms * (occ > 0 ? occ : 1);
    CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_cond_b<4>, 256, 0));
    x->grid_condb[1] = 2 * sms * (occ > 0 ? occ : 1);
    CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_cond_b<5>, 256, 0));
    x->grid_condb[2] = 2 * sms * (occ > 0 ? occ : 1);
    CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_cs_b, 256, 0));
    x->grid_flat = sms * (occ > 0 ? occ : 1);
  }
  x->tune_key = tune_key(x);
  {
    std::lock_guard<std::mutex> lock(g_tune_mutex);
    const auto it = g_tune_cache.find(x->tune_key);
    if (it != g_tune_cache.end()) x->cfg = it->second;
  }
  CUDA_TRY(cudaStreamSynchronize(x->stream));
  *out = x;
  return CLEO_OK;
}

void cleo_b200_destroy(cleo_b200_ctx* x) {
  if (!x) return;
  if (x->stream) cudaStreamSynchronize(x->stream);
  for (auto& m : x->marks) {
    cudaEventDestroy(m.a);
    cudaEventDestroy(m.b);
  }
  for (auto e : x->event_pool) cudaEventDestroy(e);
  x->drop_graphs();
  cudaFree(x->seed_buf);
  x->free_cs();
  for (cudaStream_t cs : {x->copy_stream, x->d2h_stream}) {
    if (!cs) continue;
    cudaStreamSynchronize(cs);
    cudaStreamDestroy(cs);
  }
  for (cudaEvent_t e : {x->ev_uploaded, x->ev_consumed, x->ev_snap, x->ev_snap_free, x->ev_report})
    if (e) cudaEventDestroy(e);
  for (void* p : x->allocs) cudaFree(p);
  if (x->h_motion) cudaFreeHost(x->h_motion);
  if (x->own_stream && x->stream) cudaStreamDestroy(x->stream);
  delete x;
}

void* cleo_b200_stream(cleo_b200_ctx* x) { return x ? (void*)x->stream : nullptr; }

int cleo_b200_set_profiling(cleo_b200_ctx* x, int enable) {
  if (!x) return CLEO_ERR_ARGUMENT;
  x->profiling = enable != 0;
  return CLEO_OK;
}

int cleo_b200_stage_times(cleo_b200_ctx* x, double ms[5], uint64_t count[5]) {
  if (!x || !ms || !count) return CLEO_ERR_ARGUMENT;
  CUDA_TRY(cudaStreamSynchronize(x->stream));
  for (int k = 0; k < 5; ++k) {
    ms[k] = 0.0;
    count[k] = 0;
  }
  for (auto& m : x->marks) {
    float t = 0.f;
    CUDA_TRY(cudaEventElapsedTime(&t, m.a, m.b));
    if (m.stage < 5) {  // the tuner's inner marks are not stages of their own
      ms[m.stage] += t;
      count[m.stage] += 1;
    }
    x->event_pool.push_back(m.a);
    x->event_pool.push_back(m.b);
  }
  x->marks.clear();
  return CLEO_OK;
}

int cleo_b200_set_resort_policy(cleo_b200_ctx* x, int policy) {
  if (!x || policy < CLEO_RESORT_AUTO || policy > CLEO_RESORT_FULL) return CLEO_ERR_ARGUMENT;
  x->resort_policy = policy;
  return CLEO_OK;
}

int cleo_b200_resort_stats(cleo_b200_ctx* x, uint64_t out[4]) {
  if (!x || !out) return CLEO_ERR_ARGUMENT;
  CUDA_TRY(cudaStreamSynchronize(x->stream));
  uint32_t pg[4] = {0, 0, 0, 0}, m = 0;
  CUDA_TRY(cudaMemcpy(pg, x->d.pg_ctr, sizeof pg, cudaMemcpyDeviceToHost));
  CUDA_TRY(cudaMemcpy(&m, x->mv_count, sizeof m, cudaMemcpyDeviceToHost));
  if (x->last_sort_full) {  // every slot sorted, every page written
    out[0] = x->h_motion[0];
    out[1] = x->d.npages;
    out[2] = 2;
  } else {
    out[0] = m;
    out[1] = pg[1] ? x->d.npages : pg[0];
    out[2] = pg[1] ? 1u : 0u;
  }
  out[3] = x->d.npages;
  return CLEO_OK;
}

int cleo_b200_kernel_launches(cleo_b200_ctx* x, uint64_t* n) {
  if (!x || !n) return CLEO_ERR_ARGUMENT;
  *n = x->launches;
  return CLEO_OK;
}

int cleo_b200_upload_supers(cleo_b200_ctx* x, const cleo_b200_supers* h, size_t n) {
  if (!x || !h) return CLEO_ERR_ARGUMENT;
  if (n > x->d.capacity) return CLEO_ERR_CAPACITY;
  if (!h->sdgbxindex || !h->coord3 || !h->coord1 || !h->coord2 || !h->xi || !h->radius || !h->msol)
    return CLEO_ERR_ARGUMENT;
  cudaStream_t s = x->stream;
  Fields& f = x->buf[x->cur];
  CUDA_TRY(cudaMemcpyAsync(f.gbx, h->sdgbxindex, n * 4, cudaMemcpyHostToDevice, s));
  CUDA_TRY(cudaMemcpyAsync(f.c3, h->coord3, n * 8, cudaMemcpyHostToDevice, s));
  CUDA_TRY(cudaMemcpyAsync(f.c1, h->coord1, n * 8, cudaMemcpyHostToDevice, s));
  CUDA_TRY(cudaMemcpyAsync(f.c2, h->coord2, n * 8, cudaMemcpyHostToDevice, s));
  CUDA_TRY(cudaMemcpyAsync(f.xi, h->xi, n * 8, cudaMemcpyHostToDevice, s));
  CUDA_TRY(cudaMemcpyAsync(f.r, h->radius, n * 8, cudaMemcpyHostToDevice, s));
  CUDA_TRY(cudaMemcpyAsync(f.msol, h->msol, n * 8, cudaMemcpyHostToDevice, s));
  if (h->sdid) {
    CUDA_TRY(cudaMemcpyAsync(f.id, h->sdid, n * 8, cudaMemcpyHostToDevice, s));
  } else {
    std::vector<unsigned long long> ids(n);
    for (size_t k = 0; k < n; ++k) ids[k] = k;
    CUDA_TRY(cudaMemcpyAsync(f.id, ids.data(), n * 8, cudaMemcpyHostToDevice, s));
    CUDA_TRY(cudaStreamSynchronize(s));
  }
  const uint32_t cnt[4] = {(uint32_t)n, 0, 0, 0};
  CUDA_TRY(cudaMemcpyAsync(x->d.counters, cnt, 16, cudaMemcpyHostToDevice, s));
  k_keys_paged<<<grid_for(x->d.slots, 256), 256, 0, s>>>(x->d, x->keys[0], x->vals[0]);
  x->launches += 1;
  const int rc = sort_current(x);  // SupersInDomain ctor: supersindomain.hpp:55-62
  if (rc) return rc;
  CUDA_TRY(cudaStreamSynchronize(s));
  return CLEO_OK;
}

int cleo_b200_upload_state(cleo_b200_ctx* x, const cleo_b200_gbx_state* h) {
  if (!x || !h) return CLEO_ERR_ARGUMENT;
  if (x->upload_pending) {  // these states replace the staged ones
    CUDA_TRY(cudaStreamSynchronize(x->copy_stream));
    x->upload_pending = false;
  }
  const size_t ng = x->d.ngbxs;
  const double* src[11] = {h->volume, h->press, h->temp, h->qvap, h->qcond, h->wvel_lo,
                           h->wvel_hi, h->uvel_lo, h->uvel_hi, h->vvel_lo, h->vvel_hi};
  double* dst[11] = {x->d.volume, x->d.press, x->d.temp, x->d.qvap, x->d.qcond, x->d.wlo,
                     x->d.whi, x->d.ulo, x->d.uhi, x->d.vlo, x->d.vhi};
  for (int k = 0; k < 11; ++k) {
    if (!src[k]) return CLEO_ERR_ARGUMENT;
    CUDA_TRY(cudaMemcpyAsync(dst[k], src[k], ng * 8, cudaMemcpyHostToDevice, x->stream));
  }
  CUDA_TRY(cudaStreamSynchronize(x->stream));
  return CLEO_OK;
}

int cleo_b200_upload_state_async(cleo_b200_ctx* x, const cleo_b200_gbx_state* h) {
  if (!x || !h) return CLEO_ERR_ARGUMENT;
  const size_t ng = x->d.ngbxs;
  const double* src[11] = {h->volume, h->press, h->temp, h->qvap, h->qcond, h->wvel_lo,
                           h->wvel_hi, h->uvel_lo, h->uvel_hi, h->vvel_lo, h->vvel_hi};
  for (int k = 0; k < 11; ++k)
    if (!src[k]) return CLEO_ERR_ARGUMENT;
  if (!x->stage_state) {  // first use: staging area, copy stream, events
    if (dalloc(x, &x->stage_state, 11 * (ng ? ng : 1))) return CLEO_ERR_CUDA;
    const int rc = x->ensure_copy_stream();
    if (rc) return rc;
  }
  // the staging area is free once the previous step has taken its states
  if (x->consumed_recorded) CUDA_TRY(cudaStreamWaitEvent(x->copy_stream, x->ev_consumed, 0));
  for (int k = 0; k < 11; ++k)
    CUDA_TRY(cudaMemcpyAsync(x->stage_state + (size_t)k * ng, src[k], ng * 8,
                             cudaMemcpyHostToDevice, x->copy_stream));
  CUDA_TRY(cudaEventRecord(x->ev_uploaded, x->copy_stream));
  x->upload_pending = true;
  return CLEO_OK;
}

int cleo_b200_download_budgets_async(cleo_b200_ctx* x, double* cond_mass, uint64_t* nr_iters) {
  if (!x) return CLEO_ERR_ARGUMENT;
  const size_t ng = x->d.ngbxs;
  if (!x->snap_budgets) {
    if (dalloc(x, &x->snap_budgets, 2 * (ng ? ng : 1))) return CLEO_ERR_CUDA;
    const int rc = x->ensure_copy_stream();
    if (rc) return rc;
  }
  // snapshot behind the work so far (device to device), once the previous snapshot has left
  if (x->snap_in_flight) CUDA_TRY(cudaStreamWaitEvent(x->stream, x->ev_snap_free, 0));
  double* sc = x->snap_budgets;
  uint64_t* si = reinterpret_cast<uint64_t*>(x->snap_budgets + ng);
  CUDA_TRY(cudaMemcpyAsync(sc, x->d.cond_mass, ng * 8, cudaMemcpyDeviceToDevice, x->stream));
  CUDA_TRY(cudaMemcpyAsync(si, x->d.nr_iters, ng * 8, cudaMemcpyDeviceToDevice, x->stream));
  CUDA_TRY(cudaEventRecord(x->ev_snap, x->stream));
  // to the host on a stream of its own, overlapping the next step
  CUDA_TRY(cudaStreamWaitEvent(x->d2h_stream, x->ev_snap, 0));
  if (cond_mass)
    CUDA_TRY(cudaMemcpyAsync(cond_mass, sc, ng * 8, cudaMemcpyDeviceToHost, x->d2h_stream));
  if (nr_iters)
    CUDA_TRY(cudaMemcpyAsync(nr_iters, si, ng * 8, cudaMemcpyDeviceToHost, x->d2h_stream));
  CUDA_TRY(cudaEventRecord(x->ev_snap_free, x->d2h_stream));
  x->snap_in_flight = true;
  return CLEO_OK;
}

int cleo_b200_synchronize(cleo_b200_ctx* x) {
  if (!x) return CLEO_ERR_ARGUMENT;
  if (x->copy_stream) CUDA_TRY(cudaStreamSynchronize(x->copy_stream));
  CUDA_TRY(cudaStreamSynchronize(x->stream));
  if (x->d2h_stream) CUDA_TRY(cudaStreamSynchronize(x->d2h_stream));
  return CLEO_OK;
}

// the states staged by cleo_b200_upload_state_async become the live ones (on the context's
// stream, after the copy); returns once the host arrays have been read
static int take_staged_state(cleo_b200_ctx* x) {
  const size_t ng = x->d.ngbxs;
  double* dst[11] = {x->d.volume, x->d.press, x->d.temp, x->d.qvap, x->d.qcond, x->d.wlo,
                     x->d.whi, x->d.ulo, x->d.uhi, x->d.vlo, x->d.vhi};
  CUDA_TRY(cudaStreamWaitEvent(x->stream, x->ev_uploaded, 0));
  for (int k = 0; k < 11; ++k)
    CUDA_TRY(cudaMemcpyAsync(dst[k], x->stage_state + (size_t)k * ng, ng * 8,
                             cudaMemcpyDeviceToDevice, x->stream));
  CUDA_TRY(cudaEventRecord(x->ev_consumed, x->stream));
  x->consumed_recorded = true;
  x->upload_pending = false;
  CUDA_TRY(cudaEventSynchronize(x->ev_uploaded));
  return CLEO_OK;
}

int cleo_b200_step(cleo_b200_ctx* x, uint32_t t_mdl, uint32_t t_next) {
  if (!x) return CLEO_ERR_ARGUMENT;
  if (x->d.p.nr_seed == CLEO_NRSEED_MLP && x->d.p.condstep != CLEO_STEP_OFF && !x->mlp)
    return CLEO_ERR_MLP;
  if (x->upload_pending) {
    const int rc = take_staged_state(x);
    if (rc) return rc;
  }
  const bool batched = x->d.p.exec_mode == CLEO_EXEC_BATCHED;
  uint32_t t_sdm = t_mdl;
  while (t_sdm < t_next) {
    const uint32_t next_move = next_step(x->d.p.motionstep, t_sdm);
    const uint32_t t_sdm_next = t_next < next_move ? t_next : next_move;
    {  // full re-sort when more than a fifth of the superdroplets changed gridbox in the
       // previous motion step (whose report the event marks; it completes early in that step,
       // while the rest of the step is still queued, so the device does not idle), or when the
       // store has fewer pages than SMs (the page re-sort works a page per CTA: on a small
       // domain of large gridboxes the few pages would run on a few SMs)
      if (x->report_recorded) CUDA_TRY(cudaEventSynchronize(x->ev_report));
      const volatile uint32_t* hm = x->h_motion;
      const uint32_t movers = hm[0], nsd = hm[1];
      x->sort_full = x->resort_policy == CLEO_RESORT_FULL ||
                     (x->resort_policy == CLEO_RESORT_AUTO &&
                      ((uint64_t)movers * 5 > (uint64_t)nsd || x->d.npages < (uint32_t)x->sms));
      if (on_step(x->d.p.motionstep, t_sdm)) x->last_sort_full = x->sort_full;
    }
    int rc;
    if (batched) {
      if (x->t_dev != t_sdm) {
        k_b_set_t<<<1, 1, 0, x->stream>>>(x->bs, t_sdm);
        x->launches += 1;
      }
      x->t_dev = 0xFFFFFFFFu;
      if (x->tune_step < x->tune_total)
        rc = run_tuning_step(x, t_sdm, t_sdm_next);
      else
        rc = (x->use_graphs && !x->profiling) ? run_step_graphed(x, t_sdm, t_sdm_next)
                                              : run_sdm_step(x, t_sdm, t_sdm_next);
      if (rc == CLEO_OK) x->t_dev = t_sdm_next;
    } else {
      rc = run_sdm_step(x, t_sdm, t_sdm_next);
    }
    if (rc) return rc;
    t_sdm = t_sdm_next;
  }
  return CLEO_OK;
}

int cleo_b200_autotune(cleo_b200_ctx* x, int reps) {
  if (!x || reps < 1 || reps > 1000 || x->d.p.exec_mode != CLEO_EXEC_BATCHED)
    return CLEO_ERR_ARGUMENT;
  x->tune_step = 0;
  x->tune_total = (size_t)4 * (size_t)reps;
  x->t_cond.assign(4, 0.0);
  x->t_condb.assign(4, 0.0);
  x->t_coll.assign(4, 0.0);
  return CLEO_OK;
}

int cleo_b200_tuned_config(cleo_b200_ctx* x, int32_t cfg[4]) {
  if (!x || !cfg) return CLEO_ERR_ARGUMENT;
  cfg[0] = x->cfg.cond_block;
  cfg[1] = x->cfg.cond_minb;
  cfg[2] = (int32_t)x->cfg.small_max;
  cfg[3] = x->cfg.small_minb;
  return x->tune_step < x->tune_total ? 1 : CLEO_OK;
}

int cleo_b200_set_launch_config(cleo_b200_ctx* x, const int32_t cfg[4]) {
  if (!x || !cfg) return CLEO_ERR_ARGUMENT;
  if ((cfg[0] != 128 && cfg[0] != 256) || cfg[1] < 3 || cfg[1] > 5 || cfg[2] < 1 ||
      cfg[2] > (int32_t)WARP_MAX || (cfg[3] != 2 && cfg[3] != 3))
    return CLEO_ERR_ARGUMENT;
  CUDA_TRY(cudaStreamSynchronize(x->stream));
  x->cfg = {cfg[0], cfg[1], (uint32_t)cfg[2], cfg[3], 3};  // pass B at its unspilled budget
  x->tune_total = 0;  // ends a tuning run in progress
  x->tune_step = 0;
  x->drop_graphs();
  return CLEO_OK;
}

int cleo_b200_check_math(int fn, const double* d_x, const double* d_y, double* d_out,
                         size_t n) {
  if (fn != CLEO_MATH_POW && fn != CLEO_MATH_EXP && fn != CLEO_MATH_VENT) return CLEO_ERR_ARGUMENT;
  if (n == 0) return CLEO_OK;
  if (!d_x || !d_out || (fn == CLEO_MATH_POW && !d_y)) return CLEO_ERR_ARGUMENT;
  k_math_check<<<grid_for(n, 256), 256>>>(fn, d_x, d_y, d_out, n);
  CUDA_TRY(cudaGetLastError());
  CUDA_TRY(cudaDeviceSynchronize());
  return CLEO_OK;
}

int cleo_b200_check_bounded_wait(uint32_t max_tries) {
  if (max_tries == 0 || max_tries > (1u << 24)) return CLEO_ERR_ARGUMENT;
  int* d_out = nullptr;
  CUDA_TRY(cudaMalloc(&d_out, sizeof(int)));
  int h = -1;
  k_wait_check<<<1, 128>>>(max_tries, d_out);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpy(&h, d_out, sizeof(int), cudaMemcpyDeviceToHost);
  cudaFree(d_out);
  if (e != cudaSuccess) return CLEO_ERR_CUDA;
  return h;
}

int cleo_b200_set_graphs(cleo_b200_ctx* x, int on) {
  if (!x) return CLEO_ERR_ARGUMENT;
  CUDA_TRY(cudaStreamSynchronize(x->stream));
  x->use_graphs = on != 0;
  if (!x->use_graphs) x->drop_graphs();
  return CLEO_OK;
}

int cleo_b200_status(cleo_b200_ctx* x, cleo_b200_error* err) {
  if (!x) return CLEO_ERR_ARGUMENT;
  CUDA_TRY(cudaStreamSynchronize(x->stream));
  DevError e;
  CUDA_TRY(cudaMemcpy(&e, x->d.err, sizeof(e), cudaMemcpyDeviceToHost));
  if (err) {
    err->code = e.code;
    err->gbxindex = e.gbx;
    err->index = e.index;
  }
  return e.code;
}

int cleo_b200_clear_status(cleo_b200_ctx* x) {
  if (!x) return CLEO_ERR_ARGUMENT;
  CUDA_TRY(cudaStreamSynchronize(x->stream));
  CUDA_TRY(cudaMemsetAsync(x->d.err, 0, sizeof(DevError), x->stream));
  CUDA_TRY(cudaStreamSynchronize(x->stream));
  return CLEO_OK;
}

int cleo_b200_domain_nsupers(cleo_b200_ctx* x, size_t* n) {
  if (!x || !n) return CLEO_ERR_ARGUMENT;
  CUDA_TRY(cudaStreamSynchronize(x->stream));
  std::vector<uint32_t> cnt(x->d.ngbxs ? x->d.ngbxs : 1);
  CUDA_TRY(cudaMemcpy(cnt.data(), x->d.gcount, (size_t)x->d.ngbxs * 4, cudaMemcpyDeviceToHost));
  size_t s = 0;
  for (uint32_t g = 0; g < x->d.ngbxs; ++g) s += cnt[g];
  *n = s;
  return CLEO_OK;
}

int cleo_b200_gather_supers(cleo_b200_ctx* x, uint32_t vars, const cleo_b200_obs_supers* out,
                            size_t cap, size_t* n) {
  if (!x || !out || !n || (vars & ~(uint32_t)CLEO_OBS_ALL)) return CLEO_ERR_ARGUMENT;
  DevCtx& d = x->d;
  cudaStream_t s = x->stream;
  const size_t C = d.capacity ? d.capacity : 1;
  const uint32_t ng = d.ngbxs;
  if (!x->obs_stage) {  // 36 bytes per superdroplet of the capacity + field alignment, once
    if (dalloc(x, &x->obs_stage, C * 36 + 8 * 16) || dalloc(x, &x->obs_start, (size_t)ng + 1) ||
        dalloc(x, &x->obs_tsums, ((size_t)ng + SCAN_TILE) / SCAN_TILE + 1))
      return CLEO_ERR_CUDA;
  }
  // field offsets in the staging area: 8-byte fields first, all 16-byte aligned
  uint8_t* st = x->obs_stage;
  ObsOut o{};
  const auto want = [&](uint32_t bit) { return (vars & bit) != 0; };
  const size_t a4 = (C * 4 + 15) / 16 * 16, a8 = (C * 8 + 15) / 16 * 16;
  size_t off = 0;
  if (want(CLEO_OBS_XI)) o.xi = reinterpret_cast<uint64_t*>(st + off), off += a8;
  if (want(CLEO_OBS_SDID)) o.sdid = reinterpret_cast<uint32_t*>(st + off), off += a4;
  if (want(CLEO_OBS_SDGBXINDEX)) o.gbx = reinterpret_cast<uint32_t*>(st + off), off += a4;
  if (want(CLEO_OBS_RADIUS)) o.r = reinterpret_cast<float*>(st + off), off += a4;
  if (want(CLEO_OBS_MSOL)) o.msol = reinterpret_cast<float*>(st + off), off += a4;
  if (want(CLEO_OBS_COORD3)) o.c3 = reinterpret_cast<float*>(st + off), off += a4;
  if (want(CLEO_OBS_COORD1)) o.c1 = reinterpret_cast<float*>(st + off), off += a4;
  if (want(CLEO_OBS_COORD2)) o.c2 = reinterpret_cast<float*>(st + off), off += a4;
  // output offsets: exclusive scan of the valid counts, the total at start[ngbxs]
  const uint32_t ns = (uint32_t)(((uint64_t)ng + SCAN_TILE - 1) / SCAN_TILE);
  k_obs_counts<<<grid_for(ng, 256), 256, 0, s>>>(d, x->obs_start);
  k_scan_tiles<<<ns ? ns : 1, SCAN_THREADS, 0, s>>>(x->obs_start, x->obs_start, ng, x->obs_tsums);
  k_scan_sums<<<1, SCAN_THREADS, 0, s>>>(x->obs_tsums, ns ? ns : 1, x->obs_start + ng);
  k_scan_add<<<(unsigned)((ng + 255) / 256 + 1), 256, 0, s>>>(x->obs_start, ng, x->obs_tsums);
  k_obs_gather<<<grid_for(d.slots, 256), 256, 0, s>>>(d, o, x->obs_start);
  x->launches += 5;
  CUDA_TRY(cudaGetLastError());
  uint32_t total = 0;
  CUDA_TRY(cudaMemcpyAsync(&total, x->obs_start + ng, 4, cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaStreamSynchronize(s));
  *n = total;
  if (total > cap) return CLEO_ERR_CAPACITY;
  const auto get = [&](void* dst, const void* src, size_t esize) -> int {
    if (dst && src && total) {
      CUDA_TRY(cudaMemcpyAsync(dst, src, total * esize, cudaMemcpyDeviceToHost, s));
    }
    return CLEO_OK;
  };
  int rc = 0;
  rc |= get(out->xi, o.xi, 8);
  rc |= get(out->sdid, o.sdid, 4);
  rc |= get(out->sdgbxindex, o.gbx, 4);
  rc |= get(out->radius, o.r, 4);
  rc |= get(out->msol, o.msol, 4);
  rc |= get(out->coord3, o.c3, 4);
  rc |= get(out->coord1, o.c1, 4);
  rc |= get(out->coord2, o.c2, 4);
  if (rc) return CLEO_ERR_CUDA;
  return cleo_b200_status(x, nullptr);
}

int cleo_b200_download_supers(cleo_b200_ctx* x, cleo_b200_supers* h, size_t* n_domain,
                              size_t* n_total) {
  if (!x || !h) return CLEO_ERR_ARGUMENT;
  cudaStream_t s = x->stream;
  CUDA_TRY(cudaStreamSynchronize(s));
  uint32_t cnt[4];
  CUDA_TRY(cudaMemcpy(cnt, x->d.counters, 16, cudaMemcpyDeviceToHost));
  const uint32_t nrange = cnt[0], ngrave = cnt[2];
  const size_t ng = x->d.ngbxs;
  std::vector<uint32_t> gstart(ng + 2), gcount(ng ? ng : 1);
  CUDA_TRY(cudaMemcpy(gstart.data(), x->d.gstart, (ng + 2) * 4, cudaMemcpyDeviceToHost));
  CUDA_TRY(cudaMemcpy(gcount.data(), x->d.gcount, ng * 4, cudaMemcpyDeviceToHost));
  // pull both regions to host staging
  struct HostF {
    std::vector<uint32_t> gbx;
    std::vector<double> c3, c1, c2, r, m;
    std::vector<unsigned long long> xi, id;
    void resize(size_t n) {
      gbx.resize(n); c3.resize(n); c1.resize(n); c2.resize(n); r.resize(n); m.resize(n);
      xi.resize(n); id.resize(n);
    }
  };
  auto pull = [&](const Fields& f, size_t n, HostF& o) -> int {
    o.resize(n ? n : 1);
    if (!n) return CLEO_OK;
    CUDA_TRY(cudaMemcpy(o.gbx.data(), f.gbx, n * 4, cudaMemcpyDeviceToHost));
    CUDA_TRY(cudaMemcpy(o.c3.data(), f.c3, n * 8, cudaMemcpyDeviceToHost));
    CUDA_TRY(cudaMemcpy(o.c1.data(), f.c1, n * 8, cudaMemcpyDeviceToHost));
    CUDA_TRY(cudaMemcpy(o.c2.data(), f.c2, n * 8, cudaMemcpyDeviceToHost));
    CUDA_TRY(cudaMemcpy(o.xi.data(), f.xi, n * 8, cudaMemcpyDeviceToHost));
    CUDA_TRY(cudaMemcpy(o.r.data(), f.r, n * 8, cudaMemcpyDeviceToHost));
    CUDA_TRY(cudaMemcpy(o.m.data(), f.msol, n * 8, cudaMemcpyDeviceToHost));
    CUDA_TRY(cudaMemcpy(o.id.data(), f.id, n * 8, cudaMemcpyDeviceToHost));
    return CLEO_OK;
  };
  HostF dom, grv;
  if (pull(x->buf[x->cur], nrange, dom) || pull(x->d.grave, ngrave, grv)) return CLEO_ERR_CUDA;
  size_t o = 0;
  auto put = [&](const HostF& f, size_t k) {
    h->sdgbxindex[o] = f.gbx[k];
    h->coord3[o] = f.c3[k]; h->coord1[o] = f.c1[k]; h->coord2[o] = f.c2[k];
    h->xi[o] = f.xi[k]; h->radius[o] = f.r[k]; h->msol[o] = f.m[k];
    if (h->sdid) h->sdid[o] = f.id[k];
    ++o;
  };
  for (size_t g = 0; g < ng; ++g)
    for (uint32_t k = gstart[g]; k < gstart[g] + gcount[g]; ++k) put(dom, k);
  const size_t nd = o;
  // null superdroplets still inside gridbox ranges (a page's free slots are not superdroplets)
  for (size_t g = 0; g < ng; ++g)
    for (uint32_t k = gstart[g] + gcount[g]; k < gstart[g + 1]; ++k)
      if (dom.id[k] != HOLE_ID) put(dom, k);
  for (uint32_t k = gstart[ng]; k < nrange; ++k)
    if (dom.id[k] != HOLE_ID) put(dom, k);
  for (uint32_t k = 0; k < ngrave; ++k) put(grv, k);
  if (n_domain) *n_domain = nd;
  if (n_total) *n_total = o;
  return CLEO_OK;
}

int cleo_b200_download_state(cleo_b200_ctx* x, cleo_b200_gbx_state* h) {
  if (!x || !h) return CLEO_ERR_ARGUMENT;
  CUDA_TRY(cudaStreamSynchronize(x->stream));
  const size_t ng = x->d.ngbxs;
  double* dst[11] = {h->volume, h->press, h->temp, h->qvap, h->qcond, h->wvel_lo,
                     h->wvel_hi, h->uvel_lo, h->uvel_hi, h->vvel_lo, h->vvel_hi};
  const double* src[11] = {x->d.volume, x->d.press, x->d.temp, x->d.qvap, x->d.qcond, x->d.wlo,
                           x->d.whi, x->d.ulo, x->d.uhi, x->d.vlo, x->d.vhi};
  for (int k = 0; k < 11; ++k) {
    if (!dst[k]) return CLEO_ERR_ARGUMENT;
    CUDA_TRY(cudaMemcpy(dst[k], src[k], ng * 8, cudaMemcpyDeviceToHost));
  }
  return CLEO_OK;
}

int cleo_b200_monitors_begin(cleo_b200_ctx* x) {
  if (!x) return CLEO_ERR_ARGUMENT;
  const DevCtx& d = x->d;
  if (!d.precip) return CLEO_OK;  // no monitors selected
  const size_t ng = d.ngbxs ? d.ngbxs : 1;
  k_mon_mm<<<grid_for(d.ngbxs, 256), 256, 0, x->stream>>>(d, 0, 1);
  x->launches += 1;
  for (int r = 0; r < 2; ++r)
    for (int w = 0; w < 2; ++w) {
      CUDA_TRY(cudaMemsetAsync(d.mm0[r][w], 0, ng * 8, x->stream));
      CUDA_TRY(cudaMemsetAsync(d.mm1[r][w], 0, ng * 4, x->stream));
      CUDA_TRY(cudaMemsetAsync(d.mm2[r][w], 0, ng * 4, x->stream));
    }
  CUDA_TRY(cudaMemsetAsync(d.precip, 0, ng * 8, x->stream));
  CUDA_TRY(cudaGetLastError());
  return CLEO_OK;
}

int cleo_b200_download_monitors(cleo_b200_ctx* x, cleo_b200_monitors* o, int reset) {
  if (!x || !o) return CLEO_ERR_ARGUMENT;
  const DevCtx& d = x->d;
  const size_t ng = d.ngbxs;
  CUDA_TRY(cudaStreamSynchronize(x->stream));
  uint64_t* h0[2][2] = {{o->mom0_micro, o->mom0_motion}, {o->rain_mom0_micro, o->rain_mom0_motion}};
  float* h1[2][2] = {{o->mom1_micro, o->mom1_motion}, {o->rain_mom1_micro, o->rain_mom1_motion}};
  float* h2[2][2] = {{o->mom2_micro, o->mom2_motion}, {o->rain_mom2_micro, o->rain_mom2_motion}};
  for (int r = 0; r < 2; ++r)
    for (int w = 0; w < 2; ++w) {
      if (!d.precip) {  // no monitors selected: nothing accumulated
        if (h0[r][w]) memset(h0[r][w], 0, ng * 8);
        if (h1[r][w]) memset(h1[r][w], 0, ng * 4);
        if (h2[r][w]) memset(h2[r][w], 0, ng * 4);
        continue;
      }
      if (h0[r][w]) CUDA_TRY(cudaMemcpy(h0[r][w], d.mm0[r][w], ng * 8, cudaMemcpyDeviceToHost));
      if (h1[r][w]) CUDA_TRY(cudaMemcpy(h1[r][w], d.mm1[r][w], ng * 4, cudaMemcpyDeviceToHost));
      if (h2[r][w]) CUDA_TRY(cudaMemcpy(h2[r][w], d.mm2[r][w], ng * 4, cudaMemcpyDeviceToHost));
      if (reset) {
        CUDA_TRY(cudaMemsetAsync(d.mm0[r][w], 0, ng * 8, x->stream));
        CUDA_TRY(cudaMemsetAsync(d.mm1[r][w], 0, ng * 4, x->stream));
        CUDA_TRY(cudaMemsetAsync(d.mm2[r][w], 0, ng * 4, x->stream));
      }
    }
  if (o->precip) {
    if (d.precip)
      CUDA_TRY(cudaMemcpy(o->precip, d.precip, ng * 8, cudaMemcpyDeviceToHost));
    else
      memset(o->precip, 0, ng * 8);
  }
  if (reset && d.precip) CUDA_TRY(cudaMemsetAsync(d.precip, 0, ng * 8, x->stream));
  CUDA_TRY(cudaStreamSynchronize(x->stream));
  return CLEO_OK;
}

int cleo_b200_download_budgets(cleo_b200_ctx* x, double* cond_mass, uint64_t* nr_iters) {
  if (!x) return CLEO_ERR_ARGUMENT;
  CUDA_TRY(cudaStreamSynchronize(x->stream));
  const size_t ng = x->d.ngbxs;
  if (cond_mass) CUDA_TRY(cudaMemcpy(cond_mass, x->d.cond_mass, ng * 8, cudaMemcpyDeviceToHost));
  if (nr_iters) CUDA_TRY(cudaMemcpy(nr_iters, x->d.nr_iters, ng * 8, cudaMemcpyDeviceToHost));
  return CLEO_OK;
}

int cleo_b200_condensation_solve(cleo_b200_ctx* x, size_t n, const double* d_radius,
                                 const double* d_msol, const double* d_temp, const double* d_press,
                                 const double* d_s_ratio, const double* d_delt,
                                 double* d_radius_out, uint32_t* d_niters_out) {
  if (!x || !d_radius || !d_msol || !d_temp || !d_press || !d_s_ratio || !d_delt || !d_radius_out)
    return CLEO_ERR_ARGUMENT;
  if (n >= 0xFFFFFFFFull) return CLEO_ERR_CAPACITY;
  if (n == 0) return CLEO_OK;
  const bool seeded = x->d.p.nr_seed == CLEO_NRSEED_MLP;
  const bool batched = x->d.p.exec_mode == CLEO_EXEC_BATCHED;
  mlp::Infer w;
  if (seeded) {
    if (cleo_mlp_infer_view(x->mlp, &w) != CLEO_OK) return CLEO_ERR_MLP;
    if (n > x->seed_cap) {
      CUDA_TRY(cudaStreamSynchronize(x->stream));
      cudaFree(x->seed_buf);
      x->seed_buf = nullptr;
      x->seed_cap = 0;
      CUDA_TRY(cudaMalloc(&x->seed_buf, n * sizeof(double)));
      x->seed_cap = n;
    }
    w.err = reinterpret_cast<uint32_t*>(&x->d.err->code);
  }
  const uint32_t tiles = (uint32_t)((n + mlp::TILE_M - 1) / mlp::TILE_M);
  const uint32_t tc_grid = tiles < mlp::TC_GRID_MAX ? tiles : mlp::TC_GRID_MAX;
  const double* seeds = seeded ? x->seed_buf : nullptr;
  // every solve seeded up front: most direct solves of independent droplets need more than the
  // two iterations of pass A, so the seed saves them (the batched SDM step instead seeds only the
  // solves that two iterations did not settle)
  if (seeded) {
    const CondSeedIO io{d_radius, d_msol, d_temp, d_press, d_s_ratio, d_delt, x->seed_buf};
    mlp::k_mlp_tc<CondSeedIO><<<tc_grid, 128, mlp::TC_SMEM, x->stream>>>(w, io, (uint32_t)n);
    x->launches += 1;
  }
  if (!batched) {
    k_condsolve<<<grid_for(n, 128), 128, 0, x->stream>>>(x->d, (uint32_t)n, d_radius, d_msol,
                                                         d_temp, d_press, d_s_ratio, d_delt,
                                                         seeds, d_radius_out, d_niters_out);
    x->launches += 1;
    CUDA_TRY(cudaGetLastError());
    return CLEO_OK;
  }
  // two-pass form: scratch for the deferred list of up to n solves and its 16-bit radix sort
  auto& cs = x->cs;
  if (n > cs.cap) {
    CUDA_TRY(cudaStreamSynchronize(x->stream));
    x->free_cs();
    const uint32_t nt = (uint32_t)((n + RS_TILE - 1) / RS_TILE);
    const uint64_t nh = (uint64_t)256 * nt;
    const size_t nsums = (size_t)((nh + SCAN_TILE - 1) / SCAN_TILE) + 1;
    bool ok = true;
    for (uint32_t** q : {&cs.k0, &cs.v0, &cs.k1, &cs.v1})
      ok = ok && cudaMalloc(q, n * sizeof(uint32_t)) == cudaSuccess;
    ok = ok && cudaMalloc(&cs.hist, nh * sizeof(uint32_t)) == cudaSuccess;
    ok = ok && cudaMalloc(&cs.tsums, nsums * sizeof(uint32_t)) == cudaSuccess;
    ok = ok && cudaMalloc(&cs.ctr, sizeof(uint32_t)) == cudaSuccess;
    ok = ok && cudaMalloc(&cs.zres, n * sizeof(double)) == cudaSuccess;
    if (!ok) {
      x->free_cs();
      cudaGetLastError();
      return CLEO_ERR_CUDA;
    }
    cs.cap = n;
    cs.nt = nt;
  }
  CUDA_TRY(cudaMemsetAsync(cs.ctr, 0, sizeof(uint32_t), x->stream));
  k_cs_a<<<grid_for(n, 256), 256, 0, x->stream>>>(
      x->d, (uint32_t)n, d_radius, d_msol, d_temp, d_press, d_s_ratio, d_delt,
      seeded ? x->seed_buf : nullptr, d_radius_out, d_niters_out, cs.zres, cs.k0, cs.v0, cs.ctr);
  x->launches += 1;
  const int where = radix_pairs_on(x, cs.k0, cs.v0, cs.k1, cs.v1, cs.ctr, 16, cs.hist, cs.tsums,
                                   cs.nt);
  if (where != 0) return CLEO_ERR_CUDA;  // two 8-bit passes leave the result in (k0, v0)
  k_cs_b<<<x->grid_flat * 2, 256, 0, x->stream>>>(x->d, d_radius, d_msol, d_temp, d_press,
                                                  d_s_ratio, d_delt, seeds, d_radius_out,
                                                  d_niters_out, cs.zres, cs.k0, cs.v0, cs.ctr);
  x->launches += 1;
  CUDA_TRY(cudaGetLastError());
  return CLEO_OK;
}

int cleo_b200_set_surrogate(cleo_b200_ctx* x, cleo_b200_mlp* m) {
  if (!x) return CLEO_ERR_ARGUMENT;
  if (m) {
    mlp::Infer w;
    if (cleo_mlp_infer_view(m, &w) != CLEO_OK) return CLEO_ERR_ARGUMENT;
  }
  CUDA_TRY(cudaStreamSynchronize(x->stream));
  x->drop_graphs();  // captured steps hold the previous surrogate's weights
  x->mlp = m;
  return CLEO_OK;
}

}  // extern "C"
