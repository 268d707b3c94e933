// batched_types.cuh — sizes and scratch of the batched microphysics schedule (batched.cuh).
#pragma once

#include <cstdint>

namespace {

constexpr uint32_t SMALL_MAX = 64;   // default limit of the warp kernel
constexpr uint32_t WARP_MAX = 128;   // largest gridbox the warp kernel's 128-slot variant holds
constexpr uint32_t MEDIUM_MAX = 1024;
// r, msol, xi (each with two elements of slack for the bulk copies' alignment), P, J, Simmel
// velocity
constexpr uint32_t MEDIUM_SMEM = 24 * (MEDIUM_MAX + 2) + 16 * MEDIUM_MAX;
constexpr uint32_t FY_PARALLEL_MAX = 256;  // gridboxes up to this size shuffle in parallel
constexpr int B_THREADS = 256;
constexpr int B_WARPS = B_THREADS / 32;

struct BatchScratch {
  double* th_s;      // per gridbox supersaturation ratio
  double* th_ff;     // per gridbox diffusion factor
  double* th_ak;     // per gridbox Kohler factor akoh (kohler_a)
  double* th_a3;     // per gridbox activation_a3(akoh)
  double* th_u3;     // per gridbox unique_a3(akoh)
  double* dm;        // per superdroplet condensed mass x xi
  uint32_t* its;     // per superdroplet Newton iterations
  double* qm;        // per superdroplet condensate mass x xi before the solves, when the first
                     // condensation sub-step after motion also gives qcond (else null)
  double* tv;        // per superdroplet pair terminal velocity (pair_tv) for the warp kernel,
                     // two elements of padding for its bulk copies
  double* zres;      // per deferred direct solve: pass A's iterate that pass B resumes from
  double* ffv;       // per deferred solve: pass A's diffusion factor over the ventilation factor
  uint32_t* lkeys;   // cost keys of deferred solves
  uint32_t* lvals;   // positions of deferred solves
  uint32_t* bucket;  // [4][ngbxs] gridbox lists per size bucket
  uint4* brec;       // [2][ngbxs] the warp kernel's buckets as {gridbox, start, count, RNG slot}
  uint32_t* slot;    // per gridbox RNG slot offset within the SDM step
  uint32_t* ctr;     // [0] deferred solves, [1..4] bucket counts, [5..8] bucket heads,
                     // [9] restarts among the deferred solves, [10] big gridboxes (commit)
  uint32_t* big;     // gridboxes whose condensation commit takes a warp each (k_b_commit_big)
  uint32_t* tsdm;    // the SDM step's start time (keys the injected random numbers)
  uint32_t small_max;   // gridboxes with 1..small_max superdroplets: warp kernel (<= WARP_MAX)
  uint32_t medium_max;  // small_max..medium_max: CTA kernel in shared memory (<= MEDIUM_MAX)
};

// scratch of the one-gridbox collision path (onebox.cuh)
constexpr uint32_t OB_NONE = 0xFFFFFFFFu;

struct OneBox {
  uint32_t* J;      // swap draws, index s (1 .. n-1)
  uint32_t* cnt;    // per value: bucket size, then (scanned) bucket start; n + 1 entries
  uint32_t* fill;   // per value: placement cursor
  uint32_t* bkt;    // bucket contents (swap indexes), n entries
  uint32_t* first;  // per value
  uint32_t* next;   // per swap index
  uint32_t* P;      // origin of shuffled position k
  uint32_t* vflag;  // 1 for a valid superdroplet at shuffled position q, scanned; n + 1 entries
  uint32_t* tsums;  // the scans' tile totals
  uint32_t* nnull;  // nulls made by this sub-step's collisions
  uint32_t* ninv;   // superdroplets left with multiplicity 0 (the flags' zeros)
  uint32_t* nstep;  // the gridbox's count at the step's start (for k_ob_commit)
};

}  // namespace
