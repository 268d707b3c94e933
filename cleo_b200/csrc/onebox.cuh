// onebox.cuh — collisions of a domain of one gridbox (the box model) across the whole GPU.
//
// A box model puts all its superdroplets (thousands) in one gridbox, so the per-gridbox kernels
// of batched.cuh run it on one CTA. Here each phase of the gridbox's collision step is a kernel
// over all its superdroplets or pairs, with the same results (collisions.hpp:140-248):
//   k_ob_draw    thread per swap index s >= 1: J[s], the Fisher-Yates draw (shuffle.hpp:80-87),
//                counted per value J (cnt, all zero on entry)
//   (exclusive scan of cnt: the start of each value's bucket; k_ob_scan, one block, when the
//   store's slots allow; k_ob_front does these four phases in one block for stores of up to
//   OB_FRONT_MAX slots)
//   k_ob_place   thread per s: s into its value's bucket (unordered)
//   k_ob_chains  thread per value v: its bucket sorted (increasing s), FIRST[v] and NEXT[s] (the
//                chains of the warp kernel: FIRST[v] the first swap index with J = v, NEXT[s] the
//                next one after s with the same value)
//   k_ob_pairs   thread per pair (2jj, 2jj+1) of the shuffled order: the origins P of its two
//                positions (the end of the chain J[k] -> NEXT[k] -> FIRST[.] -> ..., 0 ->
//                FIRST[0] -> ... for k = 0), collide_pair on those superdroplets in place (pairs
//                are disjoint), nulls counted, then the two valid flags in shuffled order (its
//                own pair's collision is the only one that touches them); the thread after the
//                last pair takes an odd last position and the flags' end entry
//   (exclusive scan of the flags)
//   k_ob_gather  thread per destination: valid superdroplets in shuffled order, then the nulls,
//                into scratch; it also clears cnt and fill for the next step. k_ob_commit copies
//                the records back and sets the count and RNG slot
// The host takes this path for domains of one gridbox; every array is sized by the store's slots.
#pragma once

namespace {

__global__ void k_ob_draw(const __grid_constant__ DevCtx c, const __grid_constant__ BatchScratch b,
                          OneBox o) {
  const uint32_t n = c.gcount[0];
  const uint64_t key = cleo_rng_key(c.p.seed, *b.tsdm, 0);
  const uint64_t slot = b.slot[0];
  for (uint32_t s = 1 + blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
    const uint32_t j =
        (uint32_t)cleo_rng_range(cleo_rng_u64(key, slot + (n - 1 - s)), 0, (uint64_t)s + 1);
    o.J[s] = j;
    atomicAdd(&o.cnt[j], 1u);
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    *o.nnull = 0;
    *o.ninv = 0;
  }
}
// exclusive scan in place of a[0 .. n] (n = the gridbox's count) by one block, for n + 1 <=
// OB_SCAN_MAX: each warp takes a chunk of OB_SCAN_CHUNK consecutive entries, read 32 at a time
// (coalesced) and scanned with a carry, then the chunks' totals are scanned across the warps.
// With skip set, the scan is left out while *skip is 0 (no flag to count).
constexpr uint32_t OB_SCAN_ROUNDS = 16;
constexpr uint32_t OB_SCAN_CHUNK = 32 * OB_SCAN_ROUNDS;
constexpr uint32_t OB_SCAN_MAX = (SCAN_THREADS / 32) * OB_SCAN_CHUNK;
__global__ void __launch_bounds__(SCAN_THREADS) k_ob_scan(const __grid_constant__ DevCtx c,
                                                          uint32_t* __restrict__ a,
                                                          const uint32_t* __restrict__ skip) {
  __shared__ uint32_t wsum[SCAN_THREADS / 32];
  if (skip && *skip == 0) return;
  const uint32_t m = c.gcount[0] + 1;
  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t c0 = warp * OB_SCAN_CHUNK;
  uint32_t ex[OB_SCAN_ROUNDS], carry = 0;
#pragma unroll
  for (uint32_t r = 0; r < OB_SCAN_ROUNDS; ++r) {
    const uint32_t k = c0 + 32 * r + lane;
    const uint32_t x = k < m ? a[k] : 0u;
    uint32_t inc = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, inc, o);
      if ((int)lane >= o) inc += y;
    }
    ex[r] = carry + inc - x;
    carry += __shfl_sync(0xFFFFFFFFu, inc, 31);
  }
  if (lane == 0) wsum[warp] = carry;
  __syncthreads();
  if (warp == 0) {
    const uint32_t t = wsum[lane];
    uint32_t inc = t;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, inc, o);
      if ((int)lane >= o) inc += y;
    }
    wsum[lane] = inc - t;  // exclusive over the warps' chunks
  }
  __syncthreads();
  const uint32_t off = wsum[warp];
#pragma unroll
  for (uint32_t r = 0; r < OB_SCAN_ROUNDS; ++r) {
    const uint32_t k = c0 + 32 * r + lane;
    if (k < m) a[k] = off + ex[r];
  }
}
__global__ void k_ob_place(const __grid_constant__ DevCtx c, OneBox o) {
  const uint32_t n = c.gcount[0];
  for (uint32_t s = 1 + blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
    const uint32_t v = o.J[s];
    o.bkt[o.cnt[v] + atomicAdd(&o.fill[v], 1u)] = s;
  }
}
__global__ void k_ob_chains(const __grid_constant__ DevCtx c, OneBox o) {
  const uint32_t n = c.gcount[0];
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
    const uint32_t a = o.cnt[v], e = o.cnt[v + 1];
    for (uint32_t i = a + 1; i < e; ++i) {  // insertion sort: buckets hold a few indexes
      const uint32_t x = o.bkt[i];
      uint32_t j = i;
      while (j > a && o.bkt[j - 1] > x) {
        o.bkt[j] = o.bkt[j - 1];
        --j;
      }
      o.bkt[j] = x;
    }
    o.first[v] = a < e ? o.bkt[a] : OB_NONE;
    for (uint32_t i = a; i < e; ++i) o.next[o.bkt[i]] = i + 1 < e ? o.bkt[i + 1] : OB_NONE;
  }
}
// The front of the step (k_ob_draw, the counts' scan, k_ob_place, k_ob_chains and the chain
// walks: the same values) in one block for a store of up to OB_FRONT_MAX slots, the tables in
// shared memory: cnt and fill (n + 1 each; fill then holds FIRST), J, the buckets and NEXT as
// 16-bit indexes (n each). The origins P go to global memory, so k_ob_pairs reads them instead of
// walking the chains in global memory. Five phases, four launches, become one launch.
constexpr uint32_t OB_FRONT_THREADS = 1024;
constexpr uint32_t OB_FRONT_MAX = 16000;
constexpr size_t ob_front_smem(uint32_t slots) {
  return (size_t)(slots + 1) * 8 + (size_t)slots * 6 + 16;
}
__global__ void __launch_bounds__(OB_FRONT_THREADS)
k_ob_front(const __grid_constant__ DevCtx c, const __grid_constant__ BatchScratch b, OneBox o) {
  extern __shared__ __align__(16) unsigned char ob_smem[];
  __shared__ uint32_t wsum[32];
  const uint32_t n = c.gcount[0];
  uint32_t* cnt = reinterpret_cast<uint32_t*>(ob_smem);
  uint32_t* fill = cnt + (n + 1);
  uint16_t* J = reinterpret_cast<uint16_t*>(fill + (n + 1));
  uint16_t* bkt = J + n;    // the n - 1 swap indexes by value
  uint16_t* nxt = bkt + n;  // NEXT
  uint32_t* first = fill;   // FIRST, once the placement is done with fill
  const uint32_t t = threadIdx.x;
  for (uint32_t v = t; v <= n; v += blockDim.x) {
    cnt[v] = 0u;
    fill[v] = 0u;
  }
  if (t == 0) {
    *o.nnull = 0;
    *o.ninv = 0;
  }
  __syncthreads();
  const uint64_t key = cleo_rng_key(c.p.seed, *b.tsdm, 0);
  const uint64_t slot = b.slot[0];
  for (uint32_t s = 1 + t; s < n; s += blockDim.x) {
    const uint32_t j =
        (uint32_t)cleo_rng_range(cleo_rng_u64(key, slot + (n - 1 - s)), 0, (uint64_t)s + 1);
    J[s] = (uint16_t)j;
    atomicAdd(&cnt[j], 1u);
  }
  __syncthreads();
  {  // exclusive scan of cnt[0 .. n]: thread t its contiguous share, then across the block
    const uint32_t m = n + 1, per = (m + blockDim.x - 1) / blockDim.x;
    const uint32_t lo = t * per < m ? t * per : m;
    const uint32_t hi = lo + per < m ? lo + per : m;
    uint32_t sum = 0;
    for (uint32_t i = lo; i < hi; ++i) sum += cnt[i];
    uint32_t total;
    uint32_t run = block_exclusive_scan_1024(sum, wsum, total);
    for (uint32_t i = lo; i < hi; ++i) {
      const uint32_t x = cnt[i];
      cnt[i] = run;
      run += x;
    }
  }
  __syncthreads();
  for (uint32_t s = 1 + t; s < n; s += blockDim.x) {
    const uint32_t v = J[s];
    bkt[cnt[v] + atomicAdd(&fill[v], 1u)] = (uint16_t)s;
  }
  __syncthreads();
  constexpr uint16_t NONE16 = 0xFFFFu;  // no index: n <= OB_FRONT_MAX < 2^16 - 1
  for (uint32_t v = t; v < n; v += blockDim.x) {
    const uint32_t a = cnt[v], e = cnt[v + 1];
    for (uint32_t i = a + 1; i < e; ++i) {  // insertion sort: buckets hold a few indexes
      const uint16_t x = bkt[i];
      uint32_t j = i;
      while (j > a && bkt[j - 1] > x) {
        bkt[j] = bkt[j - 1];
        --j;
      }
      bkt[j] = x;
    }
    first[v] = a < e ? (uint32_t)bkt[a] : OB_NONE;  // fill[v] is no longer needed
    for (uint32_t i = a; i < e; ++i) nxt[bkt[i]] = i + 1 < e ? bkt[i + 1] : NONE16;
  }
  __syncthreads();
  for (uint32_t k = t; k < n; k += blockDim.x) {  // the chain walks (ob_origin's)
    uint32_t cur = k == 0 ? 0u : (uint32_t)J[k];
    uint32_t nx = k == 0 ? first[0] : (nxt[k] == NONE16 ? OB_NONE : (uint32_t)nxt[k]);
    while (nx != OB_NONE) {  // strictly increasing, so at most n hops
      cur = nx;
      nx = first[cur];
    }
    o.P[k] = cur;
  }
}
// the origin of shuffled position k (what fy_origin computes), by the chains (first: FIRST[])
__device__ __forceinline__ uint32_t ob_origin(const OneBox& o, const uint32_t* first, uint32_t k) {
  uint32_t cur = k == 0 ? 0u : o.J[k];
  uint32_t nx = k == 0 ? first[0] : o.next[k];
  while (nx != OB_NONE) {  // strictly increasing, so at most n hops
    cur = nx;
    nx = first[cur];
  }
  return cur;
}
// walked: the origins P are in global memory already (k_ob_front), else found here by the chains
__global__ void k_ob_pairs(const __grid_constant__ DevCtx c, const __grid_constant__ BatchScratch b,
                           OneBox o, int walked) {
  const uint32_t n = c.gcount[0], base = c.gstart[0];
  const uint32_t npairs = n / 2;
  const uint32_t* first = o.first;
  const uint64_t key = cleo_rng_key(c.p.seed, *b.tsdm, 0);
  const uint64_t slot_pairs = (uint64_t)b.slot[0] + (n >= 1 ? n - 1 : 0);
  const double scale_p = (double)n * ((double)n - 1.0) / (2.0 * (double)npairs);
  const double VOLUME = c.volume[0] * VOL0;
  uint32_t nnull = 0, ninv = 0;
  for (uint32_t jj = blockIdx.x * blockDim.x + threadIdx.x; jj <= npairs;
       jj += gridDim.x * blockDim.x) {
    if (jj < npairs) {
      uint32_t a, bb;
      if (walked) {
        a = o.P[2 * jj];
        bb = o.P[2 * jj + 1];
      } else {
        a = ob_origin(o, first, 2 * jj);
        bb = ob_origin(o, first, 2 * jj + 1);
        o.P[2 * jj] = a;
        o.P[2 * jj + 1] = bb;
      }
      const Where w{c.err, 0u, (uint64_t)base + 2 * jj};
      nnull += collide_pair(c.p, c.sd.xi + base, c.sd.r + base, c.sd.msol + base, a, bb,
                            b.tv[base + a], b.tv[base + bb], scale_p, VOLUME, key, slot_pairs,
                            jj, w);
      const uint32_t fa = c.sd.xi[base + a] != 0 ? 1u : 0u;
      const uint32_t fb = c.sd.xi[base + bb] != 0 ? 1u : 0u;
      o.vflag[2 * jj] = fa;
      o.vflag[2 * jj + 1] = fb;
      ninv += 2u - fa - fb;
    } else {  // an odd last position (no pair) and the flags' end entry
      if (n & 1u) {
        const uint32_t p = walked ? o.P[n - 1] : ob_origin(o, first, n - 1);
        o.P[n - 1] = p;
        const uint32_t f = c.sd.xi[base + p] != 0 ? 1u : 0u;
        o.vflag[n - 1] = f;
        ninv += 1u - f;
      }
      o.vflag[n] = 0u;
    }
  }
  if (nnull) atomicAdd(o.nnull, nnull);
  if (ninv) atomicAdd(o.ninv, ninv);
}
// destinations after the exclusive scan of vflag: valid superdroplets in shuffled order first,
// then the nulls (collisions.hpp:240-248); the records into scratch. cnt and fill, used up by
// the chains, are cleared for the next step (k_ob_draw and k_ob_place count into them).
__global__ void k_ob_gather(const __grid_constant__ DevCtx c, OneBox o) {
  const uint32_t n = c.gcount[0], base = c.gstart[0];
  const uint32_t nvalid = n - *o.nnull;
  const uint32_t ninv = *o.ninv;
  if (blockIdx.x == 0 && threadIdx.x == 0) *o.nstep = n;  // k_ob_commit updates the count
  for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q <= n; q += gridDim.x * blockDim.x) {
    o.cnt[q] = 0u;
    o.fill[q] = 0u;
    if (q == n) continue;
    // valid ones before shuffled position q (the scan of the flags; q itself when all are valid,
    // the scan then left out)
    const uint32_t before = ninv ? o.vflag[q] : q;
    const uint32_t i = base + o.P[q];
    const bool valid = c.sd.xi[i] != 0;
    const uint32_t d = valid ? before : nvalid + (q - before);
    const uint32_t t = base + d;
    c.scr_r[t] = c.sd.r[i];
    c.scr_m[t] = c.sd.msol[i];
    c.scr_x[t] = c.sd.xi[i];
    c.scr_c3[t] = c.sd.c3[i];
    c.scr_c1[t] = c.sd.c1[i];
    c.scr_c2[t] = c.sd.c2[i];
    c.scr_id[t] = c.sd.id[i];
  }
}
// the records back from scratch; the gridbox's count and RNG slot after the step (its count at
// the step's start comes from k_ob_gather, so no thread reads the count this kernel sets)
__global__ void k_ob_commit(const __grid_constant__ DevCtx c, const __grid_constant__ BatchScratch b,
                            OneBox o) {
  const uint32_t n = *o.nstep, base = c.gstart[0];
  const uint32_t nvalid = n - *o.nnull;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    const uint64_t slot_pairs = (uint64_t)b.slot[0] + (n >= 1 ? n - 1 : 0);
    c.gcount[0] = nvalid;
    b.slot[0] = (uint32_t)(slot_pairs + 2ull * (n / 2));
  }
  for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
    const uint32_t t = base + q;
    c.sd.r[t] = c.scr_r[t];
    c.sd.msol[t] = c.scr_m[t];
    c.sd.xi[t] = c.scr_x[t];
    c.sd.c3[t] = c.scr_c3[t];
    c.sd.c1[t] = c.scr_c1[t];
    c.sd.c2[t] = c.scr_c2[t];
    c.sd.id[t] = c.scr_id[t];
    c.sd.gbx[t] = q < nvalid ? 0u : OOB;
  }
}

}  // namespace
