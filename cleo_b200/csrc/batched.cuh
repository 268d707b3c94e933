// batched.cuh — the batched microphysics of one SDM step (exec_mode CLEO_EXEC_BATCHED).
//
// Same results as k_micro (one CTA per gridbox), scheduled for B200 occupancy:
//   k_b_qcond      warp per 32 gridboxes: qcond from the moved superdroplets (after the sort),
//                  their condensate masses added in order (warp_batch_sums)
//   k_b_thermo     thread per gridbox: psat, supersaturation, diffusion factor, the droplets'
//                  Kohler factors that depend on temperature alone
//   k_cond_a       thread per superdroplet: the mandatory two Newton iterations of every
//                  implicit-Euler solve; solves needing more (sub-stepping, or a restart after two
//                  unconverged iterations) are appended to a list keyed by their cost
//   (radix sort of that list by cost, 16-bit keys)
//   k_mlp_tc       with nr_seed = CLEO_NRSEED_MLP only: the surrogate's Newton seeds for the
//                  listed solves (the ones the reference guess did not settle in two iterations)
//   k_cond_b       thread per listed solve, neighbouring lanes of similar cost, from the seed
//                  where its residual beats the reference guess's
//   k_b_commit     warp per 32 gridboxes: the condensed mass of each one's superdroplets added
//                  in their order, their Newton iterations, and the state update
//   k_b_classify   gridboxes into size buckets (warp-aggregated atomics); the warp kernel's
//                  buckets as records {gridbox, start, count, RNG slot}
//   k_b_tv         thread per superdroplet: the pair terminal velocities the warp kernel stages
//   k_b_small      persistent, warp per gridbox (n <= small_max <= 128; 64- and 128-slot
//                  variants): collisions in registers + per-warp shared memory
//   k_b_cta<false> persistent, CTA per gridbox (small_max < n <= medium_max <= 1024): the same
//                  with shared-memory staging
//   k_b_cta<true>  CTA per gridbox (n > medium_max) with global scratch
// small_max, the pass-A block size, the resident-CTA targets (register budgets) of pass A and of
// the warp kernel's 64-slot variant are chosen by the autotuner (results do not depend on them).
// Every per-gridbox sum of doubles adds its terms in the superdroplets' order, as the reference's
// sequential loop does (warp_batch_sums): condensed mass per droplet goes through a scratch array and is
// summed per gridbox after the solves, so budgets and states are the sequential loop's doubles
// whatever the schedule.
#pragma once

namespace {

__device__ __forceinline__ uint32_t warp_sum_u(uint32_t v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xFFFFFFFFu, v, o);
  return __shfl_sync(0xFFFFFFFFu, v, 0);
}

// warp-aggregated append of `want` lanes to a list counter; returns this lane's slot
__device__ __forceinline__ uint32_t warp_append(uint32_t* counter, bool want) {
  const unsigned m = __ballot_sync(0xFFFFFFFFu, want);
  const int lane = threadIdx.x & 31;
  uint32_t base = 0;
  if (m) {
    const int leader = __ffs(m) - 1;
    if (lane == leader) base = atomicAdd(counter, (uint32_t)__popc(m));
    base = __shfl_sync(0xFFFFFFFFu, base, leader);
  }
  return base + __popc(m & ((1u << lane) - 1u));
}

// ---- sums over gridboxes in the superdroplets' order, a warp per 32 consecutive gridboxes ----
// Consecutive gridboxes' ranges follow each other, so a batch of up to 32 gridboxes is one
// contiguous range [gstart[g0], gstart[g0 + nb]). The warp reads it coalesced, SEQ_WIN elements
// at a time, into its shared buffers (term(k) -> dbuf, iters(k) -> ubuf), and lane j adds the
// terms of gridbox g0 + j's valid superdroplets [gstart, gstart + gcount) one after another: the
// reference's sequential loop (seq_sum's order). Each window starts at the first element a lane
// still has to add, so ranges no lane adds are not read, and is loaded into registers while the
// window before it is being added. With skip_big, a gridbox of more than
// SEQ_BIG superdroplets is left out (its lane adds nothing): warp_seq_sums sums it with a warp of
// its own, so that one long sequential sum does not hold up its batch and large gridboxes are
// summed in parallel.
constexpr uint32_t SEQ_WIN = 256;
constexpr int SEQ_THREADS = 256;
constexpr uint32_t SEQ_BIG = 128;
template <class Term, class Iters>
__device__ __forceinline__ void warp_batch_sums(const DevCtx& c, uint32_t g0, uint32_t nb,
                                                double* dbuf, uint32_t* ubuf, Term term,
                                                Iters iters, double& sum,
                                                unsigned long long& its, bool skip_big) {
  constexpr int PER = SEQ_WIN / 32;  // elements of a window per lane
  constexpr uint32_t NONE = 0xFFFFFFFFu;
  const int lane = threadIdx.x & 31;
  const uint32_t hi = c.gstart[g0 + nb];
  const bool own = (uint32_t)lane < nb;
  const uint32_t s = own ? c.gstart[g0 + lane] : hi;
  uint32_t e = own ? s + c.gcount[g0 + lane] : hi;
  if (skip_big && e - s > SEQ_BIG) e = s;
  double acc = 0.0;
  unsigned long long it = 0;
  uint32_t cur = s;  // this lane's next element to add
  // the window [w0, w0 + SEQ_WIN) clipped to hi, loaded into registers a window ahead
  double pv[PER];
  uint32_t pu[PER];
  const auto load = [&](uint32_t w0) {
    const uint32_t w1 = hi - w0 < SEQ_WIN ? hi : w0 + SEQ_WIN;
#pragma unroll
    for (int q = 0; q < PER; ++q) {
      const uint32_t k = w0 + 32 * q + lane;
      pv[q] = k < w1 ? term(k) : 0.0;
      pu[q] = k < w1 ? iters(k) : 0u;
    }
  };
  uint32_t w0 = __reduce_min_sync(0xFFFFFFFFu, cur < e ? cur : NONE);
  if (w0 != NONE) load(w0);
  while (w0 != NONE) {
    const uint32_t w1 = hi - w0 < SEQ_WIN ? hi : w0 + SEQ_WIN;
#pragma unroll
    for (int q = 0; q < PER; ++q) {
      dbuf[32 * q + lane] = pv[q];
      ubuf[32 * q + lane] = pu[q];
    }
    __syncwarp();
    const uint32_t b = e < w1 ? e : w1;
    const uint32_t next = cur < b ? b : cur;  // the cursor after this window
    const uint32_t nw0 = __reduce_min_sync(0xFFFFFFFFu, next < e ? next : NONE);
    if (nw0 != NONE) load(nw0);  // in flight while this window is added
    for (uint32_t k = cur; k < b; ++k) {
      acc += dbuf[k - w0];
      it += ubuf[k - w0];
    }
    cur = next;
    __syncwarp();
    w0 = nw0;
  }
  sum = acc;
  its = it;
}
// the same sequential sums for one gridbox's range [s, e) by a whole warp: up to SEQ_GROUP chunks
// of 32 terms loaded at once, each chunk's terms broadcast one by one and added in order by every
// lane. Two sums (qcond's condensate masses qm, when given, and the condensed masses dm) are
// independent chains and run interleaved; the iterations (integers, any order) are added per lane,
// then across the warp.
constexpr int SEQ_GROUP = 8;
__device__ __forceinline__ void warp_seq_sums(uint32_t s, uint32_t e, const double* qm,
                                              const double* dm, const uint32_t* its_in,
                                              double& qsum, double& dsum,
                                              unsigned long long& its) {
  const uint32_t lane = threadIdx.x & 31;
  double aq = 0.0, ad = 0.0;
  unsigned long long it = 0;
  for (uint32_t k0 = s; k0 < e; k0 += 32 * SEQ_GROUP) {
    double vq[SEQ_GROUP], vd[SEQ_GROUP];
#pragma unroll
    for (int q = 0; q < SEQ_GROUP; ++q) {
      const uint32_t k = k0 + 32 * q + lane;
      const bool in = k < e;
      vq[q] = in && qm ? qm[k] : 0.0;
      vd[q] = in ? dm[k] : 0.0;
      it += in ? its_in[k] : 0u;
    }
#pragma unroll
    for (int q = 0; q < SEQ_GROUP; ++q) {
      const uint32_t c0 = k0 + 32 * q;
      if (c0 >= e) break;  // uniform across the warp
      const uint32_t m = e - c0 < 32 ? e - c0 : 32;
#pragma unroll
      for (uint32_t j = 0; j < 32; ++j) {
        const double tq = __shfl_sync(0xFFFFFFFFu, vq[q], j);
        const double td = __shfl_sync(0xFFFFFFFFu, vd[q], j);
        if (j < m) {
          aq += tq;
          ad += td;
        }
      }
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) it += __shfl_down_sync(0xFFFFFFFFu, it, o);
  qsum = aq;
  dsum = ad;
  its = __shfl_sync(0xFFFFFFFFu, it, 0);
}

// ---- effect_on_hydrometeor_states (movesupersindomain.hpp:95-136) ----
// qcond of gridbox g from the sum m of its superdroplets' condensate masses x xi (summed in their
// order, by k_b_qcond or by the first condensation commit after motion)
__device__ __forceinline__ void set_qcond(const DevCtx& c, uint32_t g, double m) {
  const double R0cubed_VOL0 = R0 * R0 * R0 / VOL0;
  const double rho_cond = m / c.volume[g] * R0cubed_VOL0;
  c.qcond[g] = rho_cond / dry_air_density(c.press[g], c.temp[g], c.qvap[g]);
}
__global__ void __launch_bounds__(SEQ_THREADS) k_b_qcond(const __grid_constant__ DevCtx c) {
  __shared__ double dbuf[SEQ_THREADS / 32][SEQ_WIN];
  __shared__ uint32_t ubuf[SEQ_THREADS / 32][SEQ_WIN];
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  const int wib = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (uint32_t g0 = warp * 32; g0 < c.ngbxs; g0 += nwarps * 32) {
    const uint32_t nb = c.ngbxs - g0 < 32 ? c.ngbxs - g0 : 32;
    double m;
    unsigned long long unused;
    warp_batch_sums(
        c, g0, nb, dbuf[wib], ubuf[wib],
        [&](uint32_t i) {
          const uint32_t g = c.sd.gbx[i];
          return g < c.ngbxs ? condensate_mass(c.sd.r[i], c.sd.msol[i], Where{c.err, g, i}) *
                                   (double)c.sd.xi[i]
                             : 0.0;
        },
        [](uint32_t) { return 0u; }, m, unused, false);
    if ((uint32_t)lane < nb) set_qcond(c, g0 + lane, m);
  }
}

// ---- per-gridbox thermodynamics of superdroplets_change (condensation.cpp:43-59) ----
// (every gridbox, empty ones too: the reference evaluates psat for each, and its check of the
// temperature with it)
__global__ void k_b_thermo(const __grid_constant__ DevCtx c, const __grid_constant__ BatchScratch b) {
  for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < c.ngbxs; g += gridDim.x * blockDim.x) {
    if (g == 0) b.ctr[0] = b.ctr[9] = b.ctr[10] = 0;  // deferred solves, restarts, big gridboxes
    const Where w{c.err, g, c.gstart[g]};
    const double temp = c.temp[g];
    const double psat = saturation_pressure(temp, w);
    b.th_s[g] = supersaturation_ratio(c.press[g], c.qvap[g], psat);
    b.th_ff[g] = diffusion_factor(c.press[g], temp, psat);
    const double akoh = kohler_a(temp);  // the droplets' factors that depend on akoh alone
    b.th_ak[g] = akoh;
    b.th_a3[g] = activation_a3(akoh);
    b.th_u3[g] = unique_a3(akoh);
  }
}

// the surrogate's IO for the batched schedule: row j is the j-th solve of pass A's sorted list,
// whose first b.ctr[9] entries are the direct solves that two iterations did not settle (key 0;
// the sub-stepping solves after them cannot use a seed); the seed r^2 goes to b.dm of that
// droplet, which pass B reads (and then overwrites with the droplet's condensed mass)
struct SdmListSeedIO {
  const uint32_t* gbx;
  const double *r, *msol, *temp, *press, *s_ratio;
  double delt;
  const uint32_t* list;
  const uint32_t* count;
  double* seed;
  __device__ __forceinline__ uint32_t rows(uint32_t n) const {
    const uint32_t c = *count;
    return c < n ? c : n;
  }
  __device__ __forceinline__ void features(uint32_t j, float x[mlp::NIN]) const {
    const uint32_t i = list[j];
    const uint32_t g = gbx[i];
    mlp::raw_features(r[i], msol[i], temp[g], press[g], s_ratio[g], delt, x);
  }
  __device__ __forceinline__ void store(uint32_t j, float t) const {
    const uint32_t i = list[j];
    seed[i] = mlp::seed_from(r[i], t);
  }
};

// cost key of a deferred solve: number of sub-steps (0 for a restart of the unique branch)
__device__ __forceinline__ uint32_t deferred_key(double delt, double mindelt, bool substep) {
  if (!substep) return 0u;
  const double ns = ceil(delt / mindelt);
  return ns >= 65535.0 ? 65535u : (uint32_t)ns;
}

// ---- pass A: superdrop_mass_change (condensation.cpp:98-112) up to two Newton iterations ----
template <int MINB>
__global__ void __launch_bounds__(256, MINB)
k_cond_a(const __grid_constant__ DevCtx c, const __grid_constant__ BatchScratch b) {
  const cleo_b200_params& p = c.p;
  const uint32_t n = c.counters[0];
  const NewtonCfg cfg{p.maxniters, p.rtol, p.atol};
  for (uint32_t i0 = blockIdx.x * blockDim.x; i0 < n; i0 += gridDim.x * blockDim.x) {
    const uint32_t i = i0 + threadIdx.x;
    bool defer = false;
    uint32_t key = 0;
    if (i < n) {
      const uint32_t g = c.sd.gbx[i];
      if (g < c.ngbxs) {
        const Where w{c.err, g, i};
        const double r = c.sd.r[i], msol = c.sd.msol[i];
        // the condensate mass qcond sums (k_b_qcond's term), for the commit to add in order
        if (b.qm) b.qm[i] = condensate_mass(r, msol, w) * (double)c.sd.xi[i];
        const double ffactor_fv = b.th_ff[g] / ventilation_factor(r);
        const OdeConsts o{b.th_s[g], b.th_ak[g], kohler_b(msol), ffactor_fv};
        const double z0 = initialguess_a3(o, r, b.th_a3[g]);
        // ucrit1 || ucrit2, the critical timestep only evaluated when ucrit1 fails
        const bool ucrit1 = first_unique_a3(o, r, z0, b.th_u3[g]);
        double crit = 0.0;
        uint32_t ni = 0;
        if (ucrit1 || below_critical_timestep(o, p.cond_delt, crit)) {
          bool conv = false, conv1 = false;
          double z1 = 0.0;
          GEval e = eval_g(o, p.cond_delt, r, z0);
#pragma unroll 1
          for (int it = 0; it < 2; ++it) {  // one copy of the iteration: a smaller hot loop
            e = nr_iterate(cfg, o, p.cond_delt, r, e, conv, ni);
            if (it == 0) {
              conv1 = conv;
              z1 = e.z;
            }
          }
          if (!conv) {
            b.zres[i] = conv1 ? -z1 : e.z;  // where pass B's restart continues
            b.ffv[i] = ffactor_fv;
          }
          if (conv) {
            const double rnew = max_dryradius(sqrt(e.z), msol);  // change_radius
            b.dm[i] = (condensate_mass(rnew, msol, w) - condensate_mass(r, msol, w)) *
                      (double)c.sd.xi[i];
            b.its[i] = ni;
            c.sd.r[i] = rnew;
          } else {
            defer = true;  // restart from z0 until converged (impliciteuler.cpp:136-140)
          }
        } else {
          defer = true;
          key = deferred_key(p.cond_delt, fmax(crit, p.cond_minsubdelt), true);
          b.ffv[i] = ffactor_fv;  // pass B's sub-stepping solve starts from it
        }
      }
    }
    const uint32_t pos = warp_append(&b.ctr[0], defer);
    {  // restarts (key 0) lead the sorted list; their number bounds the surrogate's rows
      const unsigned rm = __ballot_sync(0xFFFFFFFFu, defer && key == 0u);
      if (rm && (threadIdx.x & 31) == (unsigned)(__ffs(rm) - 1)) atomicAdd(&b.ctr[9], __popc(rm));
    }
    if (defer) {
      b.lkeys[pos] = key;
      b.lvals[pos] = i;
    }
  }
}

// ---- pass B: the deferred solves, in order of cost ----
template <int MINB>
__global__ void __launch_bounds__(256, MINB)
k_cond_b(const __grid_constant__ DevCtx c, const __grid_constant__ BatchScratch b) {
  const cleo_b200_params& p = c.p;
  const uint32_t nl = b.ctr[0];
  const NewtonCfg cfg{p.maxniters, p.rtol, p.atol};
  for (uint32_t jr = blockIdx.x * blockDim.x + threadIdx.x; jr < nl;
       jr += gridDim.x * blockDim.x) {
    // the list is sorted by ascending cost: the most expensive solves start first, so that the
    // longest sub-stepping ones do not run alone at the end
    const uint32_t j = nl - 1 - jr;
    const uint32_t i = b.lvals[j];
    const uint32_t g = c.sd.gbx[i];
    const Where w{c.err, g, i};
    const double r = c.sd.r[i], msol = c.sd.msol[i];
    const double akoh = b.th_ak[g], bkoh = kohler_b(msol);
    uint32_t ni = 0;
    const double seed = p.nr_seed == CLEO_NRSEED_MLP ? b.dm[i] : 0.0;
    double newr;
    if (b.lkeys[j] == 0u && cfg.maxniters >= 2) {
      // a direct solve whose two iterations in pass A did not converge: the restart continues
      // from them (resume_restart), unless the surrogate's seed converges first
      const OdeConsts o{b.th_s[g], akoh, bkoh, b.ffv[i]};  // pass A's th_ff / ventilation
      ni = 2;
      double rsqrd = 0.0;
      bool done = false;
      if (seed_ok(seed)) {
        const double z0 = initialguess_a3(o, r, b.th_a3[g]);
        const bool ucrit1 = first_unique_a3(o, r, z0, b.th_u3[g]);
        const GEval e0 = eval_g(o, p.cond_delt, r, z0);
        const GEval es = eval_g(o, p.cond_delt, r, seed);
        done = fabs(es.g) < fabs(e0.g) && integrate_seeded(cfg, o, p.cond_delt, r, es, ni, rsqrd) &&
               seeded_root_ok(o, ucrit1, rsqrd);
      }
      if (!done) {
        const int code = resume_restart(cfg, o, p.cond_delt, r, b.zres[i], ni, rsqrd);
        if (code) w.fail(code);
      }
      newr = sqrt(rsqrd);
    } else {
      // (b.ffv: pass A's th_ff / ventilation_factor(r), what solve_condensation computes first)
      newr = solve_condensation_fv(cfg, p.cond_delt, p.cond_minsubdelt, b.th_s[g], akoh, bkoh,
                                   b.ffv[i], r, seed, ni, w);
    }
    const double rnew = max_dryradius(newr, msol);
    b.dm[i] = (condensate_mass(rnew, msol, w) - condensate_mass(r, msol, w)) * (double)c.sd.xi[i];
    b.its[i] = ni;
    c.sd.r[i] = rnew;
  }
}

// ---- the pair terminal velocity of every superdroplet (for the warp kernel), a thread each:
// the same pair_tv the kernel would evaluate, with every lane busy ----
__global__ void __launch_bounds__(256) k_b_tv(const __grid_constant__ DevCtx c,
                                              const __grid_constant__ BatchScratch b) {
  const uint32_t n = c.counters[0];
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    if (c.sd.gbx[i] < c.ngbxs) b.tv[i] = pair_tv(c.p, c.sd.r[i]);
}

// ---- size buckets of the gridboxes that hold superdroplets ----
__global__ void k_b_classify(const __grid_constant__ DevCtx c, const __grid_constant__ BatchScratch b) {
  const uint32_t ng = c.ngbxs;
  for (uint32_t g0 = blockIdx.x * blockDim.x; g0 < ng; g0 += gridDim.x * blockDim.x) {
    const uint32_t g = g0 + threadIdx.x;
    const uint32_t n = g < ng ? c.gcount[g] : 0u;
    // buckets: warp kernel's 64-slot variant, its 128-slot variant (65 .. small_max), CTA per
    // gridbox in shared memory, CTA per gridbox with global scratch
    const uint32_t lo = b.small_max < SMALL_MAX ? b.small_max : SMALL_MAX;
    const int bk = (n == 0) ? -1
                 : (n <= lo ? 0 : (n <= b.small_max ? 1 : (n <= b.medium_max ? 2 : 3)));
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const uint32_t pos = warp_append(&b.ctr[1 + q], bk == q);
      if (bk == q) {
        b.bucket[(size_t)q * ng + pos] = g;
        // the warp kernel reads its gridboxes' ranges and RNG slots with the list entry
        if (q < 2) b.brec[(size_t)q * ng + pos] = make_uint4(g, c.gstart[g], n, b.slot[g]);
      }
    }
  }
}

// reduction of the condensed mass and iterations of one gridbox + state update and budgets
// (effect_on_thermodynamic_state, condensation.cpp:72-80 and :126-138; monitor, condensation.hpp:149)
__device__ __forceinline__ void cond_commit(const DevCtx& c, uint32_t g, double totmass,
                                            unsigned long long totits) {
  if (c.p.do_alter_thermo) {
    const double R0cubed_VOL0 = R0 * R0 * R0 / VOL0;
    const double totrho = totmass / c.volume[g] * R0cubed_VOL0;
    const double rho_dry = dry_air_density(c.press[g], c.temp[g], c.qvap[g]);
    const double dq = totrho / rho_dry;
    c.qvap[g] -= dq;
    c.qcond[g] += dq;
    c.temp[g] += (Latent_v / moist_specifc_heat(c.qvap[g], c.qcond[g])) * dq;
  }
  c.cond_mass[g] += totmass;
  c.nr_iters[g] += totits;
}

// ---- the gridboxes' share of a condensation sub-step after its solves ----
// The condensed mass of each gridbox's superdroplets added in their order (warp_batch_sums, the
// reference's sequential reduction, condensation.cpp:29-35), their Newton iterations, then the
// state update (cond_commit). Empty gridboxes commit a zero change, as the reference's do.
// Gridboxes of more than SEQ_BIG superdroplets are listed for k_b_commit_big instead.
__global__ void __launch_bounds__(SEQ_THREADS) k_b_commit(const __grid_constant__ DevCtx c, const __grid_constant__ BatchScratch b) {
  __shared__ double dbuf[SEQ_THREADS / 32][SEQ_WIN];
  __shared__ uint32_t ubuf[SEQ_THREADS / 32][SEQ_WIN];
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  const int wib = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (uint32_t g0 = warp * 32; g0 < c.ngbxs; g0 += nwarps * 32) {
    const uint32_t nb = c.ngbxs - g0 < 32 ? c.ngbxs - g0 : 32;
    const bool own = (uint32_t)lane < nb;
    const bool big = own && c.gcount[g0 + lane] > SEQ_BIG;
    const uint32_t pos = warp_append(&b.ctr[10], big);
    if (big) b.big[pos] = g0 + lane;
    double m;
    unsigned long long it;
    if (b.qm) {  // qcond from the moved superdroplets first (k_b_qcond's sums, from pass A)
      warp_batch_sums(
          c, g0, nb, dbuf[wib], ubuf[wib], [&](uint32_t i) { return b.qm[i]; },
          [](uint32_t) { return 0u; }, m, it, true);
      if (own && !big) set_qcond(c, g0 + lane, m);
    }
    // (positions past a gridbox's valid superdroplets are loaded but not added)
    warp_batch_sums(
        c, g0, nb, dbuf[wib], ubuf[wib], [&](uint32_t i) { return b.dm[i]; },
        [&](uint32_t i) { return b.its[i]; }, m, it, true);
    if (own && !big) cond_commit(c, g0 + lane, m, it);
  }
}
// the listed gridboxes of more than SEQ_BIG superdroplets, a warp each (the same sums and
// updates as k_b_commit's lanes make)
__global__ void __launch_bounds__(SEQ_THREADS) k_b_commit_big(const __grid_constant__ DevCtx c, const __grid_constant__ BatchScratch b) {
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  const uint32_t nbig = b.ctr[10];
  for (uint32_t j = warp; j < nbig; j += nwarps) {
    const uint32_t g = b.big[j];
    const uint32_t s = c.gstart[g], e = s + c.gcount[g];
    double mq, md;
    unsigned long long it;
    warp_seq_sums(s, e, b.qm, b.dm, b.its, mq, md, it);
    if ((threadIdx.x & 31) == 0) {
      if (b.qm) set_qcond(c, g, mq);  // qcond from the moved superdroplets first
      cond_commit(c, g, md, it);
    }
  }
}

// One pair (2jj, 2jj+1) of the shuffled gridbox, collisions.hpp:140-158, on the drops at indexes
// a and bb of the staged arrays (tvA, tvB: their pair_tv). The probability and the first random
// number decide whether the pair's collision happens, which is rare; only then does the
// out-of-line collide_enact draw the second number (the generator is counter based, so drawing it
// only then gives the same number) and enact the collision on the staged drops. Pairs that do not
// collide leave the staged arrays untouched, and the pair loop keeps few registers live.
static __device__ __noinline__ uint32_t collide_enact(const cleo_b200_params& p,
                                                      unsigned long long* sx, double* sr,
                                                      double* sm, uint32_t i1, uint32_t i2,
                                                      double prob, double phi_coll, uint64_t key,
                                                      uint64_t slot_out, double tv1, double tv2,
                                                      const Where& w) {
  Drop d1{sx[i1], sr[i1], sm[i1]};
  Drop d2{sx[i2], sr[i2], sm[i2]};
  const double phi_out = cleo_rng_to_unit(cleo_rng_u64(key, slot_out));
  // the pair's terminal velocities are the flag's too when both are Simmel's (pair_tv)
  const bool tv_known = p.coll_prob == CLEO_PROB_LONG && p.flag_tv == CLEO_TV_SIMMEL;
  const uint32_t nn = enact_collision(p, d1, d2, prob, phi_coll, phi_out, w, tv_known, tv1, tv2);
  sx[i1] = d1.xi;
  sr[i1] = d1.r;
  sm[i1] = d1.msol;
  sx[i2] = d2.xi;
  sr[i2] = d2.r;
  sm[i2] = d2.msol;
  return nn;
}
// whether enact_collision changes anything: coalescence (alone or in CoalBuRe) when its gamma
// (coalescence_gamma, whose min with xi1 / xi2 >= 1 keeps it nonzero) is nonzero, breakup when
// phi_coll is below the fractional probability
__device__ __forceinline__ bool collision_happens(const cleo_b200_params& p, double prob,
                                                  double phi_coll) {
  if (p.coll_enact == CLEO_ENACT_BREAKUP) return phi_coll < (prob - floor(prob));
  uint64_t gamma = (uint64_t)floor(prob);
  if (phi_coll < (prob - (double)gamma)) ++gamma;
  return gamma != 0;
}
__device__ __forceinline__ uint32_t collide_pair(const cleo_b200_params& p, unsigned long long* sx,
                                                 double* sr, double* sm, uint32_t a, uint32_t bb,
                                                 double tvA, double tvB, double scale_p,
                                                 double VOLUME, uint64_t key, uint64_t slot_pairs,
                                                 uint32_t jj, const Where& w) {
  const unsigned long long xa = sx[a], xb = sx[bb];
  const bool swap = xa < xb;  // d1 is the droplet of larger xi
  const uint32_t i1 = swap ? bb : a, i2 = swap ? a : bb;
  const double tv1 = swap ? tvB : tvA, tv2 = swap ? tvA : tvB;
  const double prob_jk = pair_prob_tv(p, sr[i1], sr[i2], tv1, tv2, VOLUME);
  const double large_xi = (double)(swap ? xb : xa);
  const double prob = scale_p * large_xi * prob_jk;
  const double phi_coll = cleo_rng_to_unit(cleo_rng_u64(key, slot_pairs + 2ull * jj));
  if (!collision_happens(p, prob, phi_coll)) return 0;
  return collide_enact(p, sx, sr, sm, i1, i2, prob, phi_coll, key, slot_pairs + 2ull * jj + 1,
                       tv1, tv2, w);
}

// Fisher-Yates (shuffle.hpp:80-87) applies swap(p[i], p[J[i]]) for i = n-1 down to 1 to the
// identity. The element that ends at position k started at the position reached from k by
// applying the transpositions (s, J[s]) for s = 1, 2, ..., n-1 (the swaps in reverse order), so
// every thread can find the origin of its own positions without the sequential loop.
template <class JT>
__device__ __forceinline__ uint32_t fy_origin(const JT* J, uint32_t n, uint32_t k) {
  uint32_t pos = k;
  for (uint32_t s = 1; s < n; ++s) {
    const uint32_t j = J[s];
    pos = (pos == s) ? j : ((pos == j) ? s : pos);
  }
  return pos;
}

// ---- small gridboxes: persistent, one warp per gridbox ----
// CAP (64 or 128) is the number of per-warp slots; every lane holds CAP / 32 of them.
// Radius, solute mass and multiplicity of each gridbox are staged in shared memory by bulk
// copies (TMA, cp.async.bulk) into one of two buffers per warp: the next gridbox's copies are
// in flight while the current one is processed. A copy starts at the even element at or below
// the gridbox's first superdroplet (16-byte alignment) and covers an even number of elements, so
// it may read one element past the range (the SoA arrays carry two elements of padding).
using mlp::fence_async_smem;
using mlp::mbar_init;
using mlp::mbar_wait_bounded;
using mlp::MBAR_TRIES;
using mlp::smem_u32;

// The 64-slot variant stages all seven 8-byte fields (r, msol, xi, coordinates, id), so its
// write-back reads shared memory instead of gathering the coordinates and ids from global memory
// in shuffled order; the 128-slot variant stages r, msol and xi (seven fields of 128 slots would
// leave room for fewer CTAs per SM than its registers allow). Both stage the pair terminal
// velocities k_b_tv computed (the last field).
template <int CAP>
struct SmallLayout {
  static constexpr bool ALL = CAP <= 64;
  static constexpr uint32_t NF = ALL ? 8 : 4;  // staged fields per buffer
  static constexpr uint32_t F_TV = NF - 1;
  static constexpr uint32_t BUF = CAP + 2;  // elements per staged field
  static constexpr uint32_t FIELD = BUF * 8;
  static constexpr uint32_t OFF_P = 2 * NF * FIELD;
  static constexpr uint32_t OFF_J = OFF_P + CAP;
  static constexpr uint32_t OFF_F = OFF_J + CAP;  // first index of each swap target (chains)
  static constexpr uint32_t OFF_BAR = (OFF_F + CAP + 15) / 16 * 16;
  static constexpr uint32_t WARP_BYTES = OFF_BAR + 16;
  static constexpr uint32_t BYTES = WARP_BYTES * B_WARPS;
  static_assert(FIELD % 16 == 0 && WARP_BYTES % 16 == 0, "bulk-copy buffers must be aligned");
};

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes,
                                         uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(smem_u32(dst)),
      "l"(__cvta_generic_to_global(src)), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

template <int MINB, int CAP>
__global__ void __launch_bounds__(B_THREADS, MINB)
k_b_small(const __grid_constant__ DevCtx c, const __grid_constant__ BatchScratch b, int q) {
  using L = SmallLayout<CAP>;
  constexpr int H = CAP / 32;
  static_assert(CAP % 32 == 0 && CAP <= 255, "slot indices are stored as bytes");
  const uint32_t t_sdm = *b.tsdm;
  extern __shared__ __align__(16) unsigned char smem_small[];
  const cleo_b200_params& p = c.p;
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  unsigned char* wsm = smem_small + wib * L::WARP_BYTES;
  uint8_t* s_p = wsm + L::OFF_P;
  uint8_t* s_j = wsm + L::OFF_J;
  uint8_t* s_f = wsm + L::OFF_F;
  uint64_t* bar = reinterpret_cast<uint64_t*>(wsm + L::OFF_BAR);
  const auto field = [&](int buf, int f) { return wsm + (buf * L::NF + f) * L::FIELD; };
  const uint32_t count = b.ctr[1 + q];
  const uint4* list = b.brec + (size_t)q * c.ngbxs;  // {gridbox, start, count, RNG slot}
  // stage a gridbox's fields into buffer buf (lane 0)
  const auto stage = [&](int buf, const uint4& rec) {
    const uint32_t base = rec.y, n = rec.z;
    const uint32_t a0 = base & ~1u;
    const uint32_t bytes = ((n + (base & 1u) + 1u) & ~1u) * 8u;
    fence_async_smem();  // earlier generic accesses of the buffer precede the async writes
    mbar_expect_tx(&bar[buf], L::NF * bytes);
    bulk_g2s(field(buf, 0), c.sd.r + a0, bytes, &bar[buf]);
    bulk_g2s(field(buf, 1), c.sd.msol + a0, bytes, &bar[buf]);
    bulk_g2s(field(buf, 2), c.sd.xi + a0, bytes, &bar[buf]);
    bulk_g2s(field(buf, L::F_TV), b.tv + a0, bytes, &bar[buf]);
    if constexpr (L::ALL) {
      bulk_g2s(field(buf, 3), c.sd.c3 + a0, bytes, &bar[buf]);
      bulk_g2s(field(buf, 4), c.sd.c1 + a0, bytes, &bar[buf]);
      bulk_g2s(field(buf, 5), c.sd.c2 + a0, bytes, &bar[buf]);
      bulk_g2s(field(buf, 6), c.sd.id + a0, bytes, &bar[buf]);
    }
  };
  // static assignment (item = warp + k * warps): no shared counter; a gridbox's list record is
  // loaded two gridboxes ahead and its copies are issued one gridbox ahead
  const uint32_t nwarps = gridDim.x * B_WARPS;
  uint32_t item = blockIdx.x * B_WARPS + wib;
  const uint4 none = make_uint4(0u, 0u, 0u, 0u);
  uint4 rec_next = item < count ? list[item] : none;
  uint4 rec_after = item + nwarps < count ? list[item + nwarps] : none;
  uint32_t parity = 0;  // bit k: the phase of bar[k] to wait for
  int cur = 0;
  if (lane == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    if (item < count) stage(0, rec_next);
  }
  __syncwarp();
  for (; item < count; item += nwarps) {
    const uint4 rec = rec_next;
    const uint32_t g = rec.x, base = rec.y, n = rec.z;
    const bool has_next = item + nwarps < count;
    rec_next = rec_after;
    rec_after = item + 2 * nwarps < count ? list[item + 2 * nwarps] : none;
    // the next gridbox's copies go out before this one's wait
    if (has_next && lane == 0) stage(cur ^ 1, rec_next);
    const double VOLUME = c.volume[g] * VOL0;  // issued before the wait
    if (!mbar_wait_bounded(&bar[cur], (parity >> cur) & 1u, MBAR_TRIES)) {
      // the step fails with CLEO_ERR_TIMEOUT; before the warp leaves, the copies still in flight
      // into either buffer get a bounded wait to land
      if (lane == 0) Where{c.err, g, base}.fail(CLEO_ERR_TIMEOUT);
      mbar_wait_bounded(&bar[cur], (parity >> cur) & 1u, MBAR_TRIES);
      if (has_next) mbar_wait_bounded(&bar[cur ^ 1], (parity >> (cur ^ 1)) & 1u, MBAR_TRIES);
      return;
    }
    parity ^= 1u << cur;
    const uint32_t off = base & 1u;
    double* s_r = reinterpret_cast<double*>(field(cur, 0)) + off;
    double* s_m = reinterpret_cast<double*>(field(cur, 1)) + off;
    unsigned long long* s_x = reinterpret_cast<unsigned long long*>(field(cur, 2)) + off;
    const double* s_tv = reinterpret_cast<const double*>(field(cur, L::F_TV)) + off;
    const uint64_t key = cleo_rng_key(p.seed, t_sdm, g);
    const uint64_t slot = rec.w;
    for (uint32_t k = 1 + lane; k < n; k += 32)
      s_j[k] = (uint8_t)cleo_rng_range(cleo_rng_u64(key, slot + (n - 1 - k)), 0, (uint64_t)k + 1);
    __syncwarp();
    {
      // origins of the shuffled positions (what fy_origin computes), by chains: tracing position
      // k through the swaps, nothing happens before swap k, swap k takes it to J[k], and after
      // that it moves only to a later index s whose J[s] equals its current position. With
      // FIRST[v] (the first index s >= 1 with J[s] == v) and NEXTSAME[s] (the next index after s
      // with the same J value), the origin of k is the end of the chain J[k] -> NEXTSAME[k] ->
      // FIRST[.] -> ... (0 -> FIRST[0] -> ... for k = 0), about ln n lookups instead of n - 1
      // swaps. Both tables are built from the index groups of 32, last group first, with
      // __match_any_sync.
      constexpr uint32_t NONE = 0xFFu;
      for (uint32_t v = lane; v < n; v += 32) s_f[v] = (uint8_t)NONE;
      __syncwarp();
      uint32_t nsame[H];
#pragma unroll
      for (int h = H - 1; h >= 0; --h) {
        nsame[h] = NONE;
        if (32u * h >= n) continue;  // uniform across the warp
        const uint32_t sidx = lane + 32u * h;
        const bool act = sidx >= 1 && sidx < n;
        const uint32_t v = act ? (uint32_t)s_j[sidx] : 0x100u + lane;  // inactive: unique
        const unsigned peers = __match_any_sync(0xFFFFFFFFu, v);
        const unsigned higher = peers & ~((2u << lane) - 1u);
        if (act) nsame[h] = higher ? 32u * h + __ffs(higher) - 1 : (uint32_t)s_f[v];
        __syncwarp();
        if (act && lane == __ffs(peers) - 1) s_f[v] = (uint8_t)sidx;
        __syncwarp();
      }
#pragma unroll
      for (int h = 0; h < H; ++h) {
        const uint32_t k = lane + 32u * h;
        if (k < n) {
          uint32_t cur = k == 0 ? 0u : (uint32_t)s_j[k];
          uint32_t nx = k == 0 ? (uint32_t)s_f[0] : nsame[h];
          while (nx != NONE) {  // strictly increasing, so at most n hops
            cur = nx;
            nx = s_f[cur];
          }
          s_p[k] = (uint8_t)cur;
        }
      }
    }
    __syncwarp();
    const uint64_t slot_pairs = slot + (n >= 1 ? n - 1 : 0);
    const uint32_t npairs = n / 2;
    const double scale_p = (double)n * ((double)n - 1.0) / (2.0 * (double)npairs);
    uint32_t nnull = 0;
    for (uint32_t jj = lane; jj < npairs; jj += 32) {
      const uint32_t a = s_p[2 * jj], bb = s_p[2 * jj + 1];
      const Where w{c.err, g, (uint64_t)base + 2 * jj};
      nnull += collide_pair(p, s_x, s_r, s_m, a, bb, s_tv[a], s_tv[bb], scale_p, VOLUME, key,
                            slot_pairs, jj, w);
    }
    __syncwarp();
    const uint32_t totnull = warp_sum_u(nnull);
    const uint32_t nvalid = n - totnull;
    // destinations: valid superdroplets in shuffled order, then the nulls (collisions.hpp:240-248)
    uint32_t src[H], q[H];
    double c3v[L::ALL ? 1 : H], c1v[L::ALL ? 1 : H], c2v[L::ALL ? 1 : H];
    unsigned long long idv[L::ALL ? 1 : H];
    uint32_t cval = 0, cnull = 0;
#pragma unroll
    for (int h = 0; h < H; ++h) {
      if (32u * h >= n) break;  // uniform across the warp
      const uint32_t k = lane + 32 * h;
      const bool act = k < n;
      src[h] = act ? s_p[k] : 0;
      const bool valid = act && s_x[src[h]] != 0;
      const unsigned mv = __ballot_sync(0xFFFFFFFFu, valid);
      const unsigned mn = __ballot_sync(0xFFFFFFFFu, act && !valid);
      const unsigned lt = (1u << lane) - 1u;
      q[h] = valid ? cval + __popc(mv & lt) : nvalid + cnull + __popc(mn & lt);
      cval += __popc(mv);
      cnull += __popc(mn);
      if constexpr (!L::ALL) {
        if (act) {
          const uint32_t s = base + src[h];
          c3v[h] = c.sd.c3[s];
          c1v[h] = c.sd.c1[s];
          c2v[h] = c.sd.c2[s];
          idv[h] = c.sd.id[s];
        }
      }
    }
    __syncwarp();
#pragma unroll
    for (int h = 0; h < H; ++h) {
      const uint32_t k = lane + 32 * h;
      if (k < n) {
        const uint32_t o = base + q[h];
        c.sd.r[o] = s_r[src[h]];
        c.sd.msol[o] = s_m[src[h]];
        c.sd.xi[o] = s_x[src[h]];
        c.sd.gbx[o] = q[h] < nvalid ? g : OOB;
        if constexpr (L::ALL) {
          c.sd.c3[o] = reinterpret_cast<const double*>(field(cur, 3))[off + src[h]];
          c.sd.c1[o] = reinterpret_cast<const double*>(field(cur, 4))[off + src[h]];
          c.sd.c2[o] = reinterpret_cast<const double*>(field(cur, 5))[off + src[h]];
          c.sd.id[o] = reinterpret_cast<const unsigned long long*>(field(cur, 6))[off + src[h]];
        } else {
          c.sd.c3[o] = c3v[h];
          c.sd.c1[o] = c1v[h];
          c.sd.c2[o] = c2v[h];
          c.sd.id[o] = idv[h];
        }
      }
    }
    __syncwarp();  // every lane is done with buffer cur before it is staged into again
    if (lane == 0) {
      c.gcount[g] = nvalid;
      b.slot[g] = (uint32_t)(slot_pairs + 2ull * npairs);
    }
    cur ^= 1;
  }
}

// Origins of the shuffled positions of a gridbox of n (2 .. CHAIN_MAX) superdroplets for a whole
// CTA, by the chains the warp kernel follows (see k_b_small): FIRST[v] = the first swap index s
// with J[s] = v, NEXT[s] = the next swap index after s with the same J value. The pairs
// (J[s], s), s = 1 .. n-1, are ordered by a bitonic sort of the 32-bit keys J[s] << 16 | s in
// shared memory (`keys`, a power of two >= n - 1 entries), so that equal values lie together in
// increasing s; FIRST and NEXT (n entries each, any memory) are read off the sorted keys, and
// each thread then walks the chains of its positions (about ln n lookups each). P receives the
// origins, as fy_origin computes them. Ends with a barrier.
constexpr uint32_t CHAIN_MAX = 16384;  // keys of up to 16384 swaps: 64 KB of shared memory
// the keys, FIRST and NEXT of up to CHAIN_MAX swaps in shared memory (192 KB): the chain walks'
// dependent lookups stay on chip
constexpr uint32_t LARGE_SMEM = CHAIN_MAX * 4 * 3;
constexpr uint32_t LARGE_THREADS = 1024;  // a gridbox of thousands: four times B_THREADS
__device__ void cta_fy_origins(const uint32_t* J, uint32_t n, uint32_t* keys, uint32_t* FIRST,
                               uint32_t* NEXT, uint32_t* P) {
  constexpr uint32_t NONE = 0xFFFFFFFFu;
  const uint32_t tid = threadIdx.x, nt = blockDim.x;
  const uint32_t m = n - 1;  // swaps s = 1 .. n-1
  uint32_t mp = 1;
  while (mp < m) mp <<= 1;
  for (uint32_t i = tid; i < mp; i += nt) keys[i] = i < m ? (J[i + 1] << 16) | (i + 1) : NONE;
  for (uint32_t v = tid; v < n; v += nt) FIRST[v] = NEXT[v] = NONE;
  __syncthreads();
  for (uint32_t k = 2; k <= mp; k <<= 1) {
    for (uint32_t j = k >> 1; j > 0; j >>= 1) {
      for (uint32_t i = tid; i < mp; i += nt) {
        const uint32_t l = i ^ j;
        if (l > i) {
          const uint32_t a = keys[i], bk = keys[l];
          if ((a > bk) == ((i & k) == 0)) {
            keys[i] = bk;
            keys[l] = a;
          }
        }
      }
      __syncthreads();
    }
  }
  for (uint32_t i = tid; i < m; i += nt) {
    const uint32_t v = keys[i] >> 16, sidx = keys[i] & 0xFFFFu;
    if (i == 0 || (keys[i - 1] >> 16) != v) FIRST[v] = sidx;
    if (i + 1 < m && (keys[i + 1] >> 16) == v) NEXT[sidx] = keys[i + 1] & 0xFFFFu;
  }
  __syncthreads();
  for (uint32_t k = tid; k < n; k += nt) {
    uint32_t cur = k == 0 ? 0u : J[k];
    uint32_t nx = k == 0 ? FIRST[0] : NEXT[k];
    while (nx != NONE) {  // strictly increasing, so at most n hops
      cur = nx;
      nx = FIRST[cur];
    }
    P[k] = cur;
  }
  __syncthreads();
}

// ---- medium and large gridboxes: one CTA per gridbox ----
// medium: staged in shared memory with the non-staged fields permuted through registers;
// large: staged in global scratch arrays, the shuffle's chain tables in LARGE_SMEM of shared memory.
template <bool LARGE>
__global__ void __launch_bounds__(LARGE ? LARGE_THREADS : B_THREADS)
k_b_cta(const __grid_constant__ DevCtx c, const __grid_constant__ BatchScratch b) {
  const uint32_t t_sdm = *b.tsdm;
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ uint32_t shw[40];
  __shared__ uint32_t s_item;
  __shared__ uint64_t s_bar;  // completion of the medium path's bulk copies
  constexpr uint32_t PT = MEDIUM_MAX / B_THREADS;  // superdroplets per thread (medium)
  constexpr uint32_t NT = LARGE ? LARGE_THREADS : B_THREADS;  // threads of the block
  constexpr uint32_t MBUF = MEDIUM_MAX + 2;        // staged elements per field (medium)
  const cleo_b200_params& p = c.p;
  const int tid = threadIdx.x;
  const uint32_t q_idx = LARGE ? 3 : 2;
  const uint32_t count = b.ctr[1 + q_idx];
  const uint32_t* list = b.bucket + (size_t)q_idx * c.ngbxs;
  uint32_t bar_parity = 0;
  if (!LARGE) {
    if (tid == 0) mbar_init(&s_bar, 1);
    __syncthreads();
  }
  while (true) {
    if (tid == 0) s_item = atomicAdd(&b.ctr[5 + q_idx], 1u);
    __syncthreads();
    const uint32_t item = s_item;
    __syncthreads();
    if (item >= count) break;
    const uint32_t g = list[item];
    const uint32_t base = c.gstart[g];
    const uint32_t n = c.gcount[g];
    const uint64_t key = cleo_rng_key(p.seed, t_sdm, g);
    const uint64_t slot = b.slot[g];
    // medium: r, msol, xi staged in shared memory by bulk copies (TMA) from the even element at
    // or below the gridbox's first superdroplet (16-byte alignment; the SoA arrays' padding
    // covers the element a copy may read past the range); large: global scratch
    const uint32_t off = base & 1u;
    double* Sr = LARGE ? c.scr_r + base : reinterpret_cast<double*>(smem) + off;
    double* Sm = LARGE ? c.scr_m + base : reinterpret_cast<double*>(smem) + MBUF + off;
    unsigned long long* Sx = LARGE ? c.scr_x + base
                                   : reinterpret_cast<unsigned long long*>(smem) + 2 * MBUF + off;
    uint32_t* P = LARGE ? c.scr_p + base : reinterpret_cast<uint32_t*>(smem + 24 * MBUF);
    uint32_t* J = LARGE ? c.scr_j + base
                        : reinterpret_cast<uint32_t*>(smem + 24 * MBUF + 4 * MEDIUM_MAX);
    // the pair terminal velocities k_b_tv computed (medium: copied to shared memory after the five
    // staged arrays; large: read per pair)
    double* Stv = LARGE ? nullptr : reinterpret_cast<double*>(smem + 24 * MBUF + 8 * MEDIUM_MAX);
    if (!LARGE) {
      if (tid == 0) {  // the previous gridbox's accesses ended at the barriers above
        const uint32_t bytes = ((n + off + 1u) & ~1u) * 8u;
        const uint32_t a0 = base & ~1u;
        fence_async_smem();
        mbar_expect_tx(&s_bar, 3u * bytes);
        bulk_g2s(smem, c.sd.r + a0, bytes, &s_bar);
        bulk_g2s(smem + 8 * MBUF, c.sd.msol + a0, bytes, &s_bar);
        bulk_g2s(smem + 16 * MBUF, c.sd.xi + a0, bytes, &s_bar);
      }
      // every thread waits with a bound; the outcome is agreed by the whole block
      const bool ok = __syncthreads_and(mbar_wait_bounded(&s_bar, bar_parity, MBAR_TRIES) ? 1 : 0);
      if (!ok) {
        if (tid == 0) Where{c.err, g, base}.fail(CLEO_ERR_TIMEOUT);
        mbar_wait_bounded(&s_bar, bar_parity, MBAR_TRIES);  // let the copies in flight land
        return;
      }
      bar_parity ^= 1u;
    }
    for (uint32_t k = tid; k < n; k += NT) {
      if (LARGE) {
        Sr[k] = c.sd.r[base + k];
        Sm[k] = c.sd.msol[base + k];
        Sx[k] = c.sd.xi[base + k];
      } else {
        Stv[k] = b.tv[base + k];  // k_b_tv's pair terminal velocity of the same radius
      }
      if (k >= 1) J[k] = (uint32_t)cleo_rng_range(cleo_rng_u64(key, slot + (n - 1 - k)), 0, (uint64_t)k + 1);
    }
    __syncthreads();
    if (n <= FY_PARALLEL_MAX) {  // every thread traces its own positions
      for (uint32_t k = tid; k < n; k += NT) P[k] = fy_origin(J, n, k);
    } else if (LARGE && n <= CHAIN_MAX) {  // chains, as in the warp kernel (keys in smem)
      cta_fy_origins(J, n, reinterpret_cast<uint32_t*>(smem),
                     reinterpret_cast<uint32_t*>(smem) + CHAIN_MAX,
                     reinterpret_cast<uint32_t*>(smem) + 2 * CHAIN_MAX, P);
    } else {
      for (uint32_t k = tid; k < n; k += NT) P[k] = k;
      __syncthreads();
      if (tid == 0) {
        for (uint32_t it = n > 0 ? n - 1 : 0; it > 0; --it) {
          const uint32_t j = J[it];
          const uint32_t t = P[it];
          P[it] = P[j];
          P[j] = t;
        }
      }
    }
    __syncthreads();
    const uint64_t slot_pairs = slot + (n >= 1 ? n - 1 : 0);
    const uint32_t npairs = n / 2;
    const double scale_p = (double)n * ((double)n - 1.0) / (2.0 * (double)npairs);
    const double VOLUME = c.volume[g] * VOL0;
    uint32_t nnull = 0;
    for (uint32_t jj = tid; jj < npairs; jj += NT) {
      const uint32_t a = P[2 * jj], bb = P[2 * jj + 1];
      const Where w{c.err, g, (uint64_t)base + 2 * jj};
      const double tvA = LARGE ? b.tv[base + a] : Stv[a];
      const double tvB = LARGE ? b.tv[base + bb] : Stv[bb];
      nnull += collide_pair(p, Sx, Sr, Sm, a, bb, tvA, tvB, scale_p, VOLUME, key, slot_pairs, jj,
                            w);
    }
    const uint32_t totnull = block_sum(nnull, shw);
    const uint32_t nvalid = n - totnull;
    uint32_t cval = 0, cnull = 0;
    // destination of shuffled position k; J becomes the inverse map q -> source
    for (uint32_t k0 = 0; k0 < n; k0 += NT) {
      const uint32_t k = k0 + tid;
      const bool act = k < n;
      const uint32_t src = act ? P[k] : 0;
      const bool valid = act && Sx[src] != 0;
      uint32_t tv, tn;
      const uint32_t ev = block_excl_scan(valid ? 1u : 0u, shw, tv);
      const uint32_t en = block_excl_scan((act && !valid) ? 1u : 0u, shw, tn);
      if (act) J[valid ? (cval + ev) : (nvalid + cnull + en)] = src;
      cval += tv;
      cnull += tn;
    }
    __syncthreads();
    if (LARGE) {
      for (uint32_t q = tid; q < n; q += NT) {
        const uint32_t s = base + J[q], o = base + q;
        c.scr_c3[o] = c.sd.c3[s];
        c.scr_c1[o] = c.sd.c1[s];
        c.scr_c2[o] = c.sd.c2[s];
        c.scr_id[o] = c.sd.id[s];
      }
      __syncthreads();
      for (uint32_t q = tid; q < n; q += NT) {
        const uint32_t o = base + q;
        const uint32_t src = J[q];
        c.sd.r[o] = Sr[src];
        c.sd.msol[o] = Sm[src];
        c.sd.xi[o] = Sx[src];
        c.sd.gbx[o] = q < nvalid ? g : OOB;
        c.sd.c3[o] = c.scr_c3[o];
        c.sd.c1[o] = c.scr_c1[o];
        c.sd.c2[o] = c.scr_c2[o];
        c.sd.id[o] = c.scr_id[o];
      }
    } else {
      double c3v[PT], c1v[PT], c2v[PT];
      unsigned long long idv[PT];
#pragma unroll
      for (uint32_t h = 0; h < PT; ++h) {
        const uint32_t q = tid + h * B_THREADS;
        if (q < n) {
          const uint32_t s = base + J[q];
          c3v[h] = c.sd.c3[s];
          c1v[h] = c.sd.c1[s];
          c2v[h] = c.sd.c2[s];
          idv[h] = c.sd.id[s];
        }
      }
      __syncthreads();
#pragma unroll
      for (uint32_t h = 0; h < PT; ++h) {
        const uint32_t q = tid + h * B_THREADS;
        if (q < n) {
          const uint32_t o = base + q;
          const uint32_t src = J[q];
          c.sd.r[o] = Sr[src];
          c.sd.msol[o] = Sm[src];
          c.sd.xi[o] = Sx[src];
          c.sd.gbx[o] = q < nvalid ? g : OOB;
          c.sd.c3[o] = c3v[h];
          c.sd.c1[o] = c1v[h];
          c.sd.c2[o] = c2v[h];
          c.sd.id[o] = idv[h];
        }
      }
    }
    __syncthreads();
    if (tid == 0) {
      c.gcount[g] = nvalid;
      b.slot[g] = (uint32_t)(slot_pairs + 2ull * npairs);
    }
  }
}

// reset of the per-gridbox slot offsets at the start of an SDM step and of the bucket counters
// the device copy of the SDM step time: set before a step whose time the device does not hold,
// advanced by the last kernel of every step (so one captured step graph serves every step)
__global__ void k_b_set_t(BatchScratch b, uint32_t t) { *b.tsdm = t; }
// the SDM step's end: its start time advanced; with zero_slot0 (a one-gridbox domain, whose step
// has no per-gridbox reset) the gridbox's RNG slot is reset for the next step here
__global__ void k_b_advance_t(BatchScratch b, uint32_t dt, int zero_slot0) {
  *b.tsdm += dt;
  if (zero_slot0) b.slot[0] = 0;
}

__global__ void k_b_reset(const __grid_constant__ DevCtx c, const __grid_constant__ BatchScratch b, int slots) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (slots)
    for (uint32_t g = i; g < c.ngbxs; g += gridDim.x * blockDim.x) b.slot[g] = 0;
  if (i < 8) b.ctr[1 + i] = 0;  // bucket counts and heads
}

}  // namespace
