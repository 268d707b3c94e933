// onebox.cuh — collisions of a domain of one gridbox (the box model) across the whole GPU.
//
// A box model puts all its superdroplets (thousands) in one gridbox, so the per-gridbox kernels
// of batched.cuh run it on one CTA. Here each phase of the gridbox's collision step is a kernel
// over all its superdroplets or pairs, with the same results (collisions.hpp:140-248):
//   k_ob_draw    thread per swap index s >= 1: J[s], the Fisher-Yates draw (shuffle.hpp:80-87),
//                counted per value J (cnt)
//   (exclusive scan of cnt: the start of each value's bucket)
//   k_ob_place   thread per s: s into its value's bucket (unordered)
//   k_ob_chains  thread per value v: its bucket sorted (increasing s), FIRST[v] and NEXT[s] (the
//                chains of the warp kernel: FIRST[v] the first swap index with J = v, NEXT[s] the
//                next one after s with the same value)
//   k_ob_origin  thread per position k: the origin P[k] of the element the shuffle leaves at k,
//                the end of the chain J[k] -> NEXT[k] -> FIRST[.] -> ... (0 -> FIRST[0] -> ... for
//                k = 0)
//   k_ob_pairs   thread per pair (2jj, 2jj+1) of the shuffled order: collide_pair on the
//                superdroplets in place (pairs are disjoint), nulls counted
//   k_ob_flags   the valid flags in shuffled order (then their exclusive scan)
//   k_ob_gather  thread per destination: valid superdroplets in shuffled order, then the nulls,
//                into scratch; k_ob_commit copies them back and sets the count and RNG slot
// The host takes this path for domains of one gridbox; every array is sized by the store's slots.
#pragma once

namespace {

__global__ void k_ob_draw(const __grid_constant__ DevCtx c, const __grid_constant__ BatchScratch b,
                          OneBox o) {
  const uint32_t n = c.gcount[0];
  const uint64_t key = cleo_rng_key(c.p.seed, *b.tsdm, 0);
  const uint64_t slot = b.slot[0];
  for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s <= n; s += gridDim.x * blockDim.x) {
    o.cnt[s] = 0;  // n + 1 entries (the scan's total after the last); k_ob_count adds to them
    o.fill[s] = 0;
  }
  for (uint32_t s = 1 + blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x)
    o.J[s] = (uint32_t)cleo_rng_range(cleo_rng_u64(key, slot + (n - 1 - s)), 0, (uint64_t)s + 1);
  if (blockIdx.x == 0 && threadIdx.x == 0) *o.nnull = 0;
}
__global__ void k_ob_count(const __grid_constant__ DevCtx c, OneBox o) {
  const uint32_t n = c.gcount[0];
  for (uint32_t s = 1 + blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x)
    atomicAdd(&o.cnt[o.J[s]], 1u);
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
__global__ void k_ob_origin(const __grid_constant__ DevCtx c, OneBox o) {
  const uint32_t n = c.gcount[0];
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    uint32_t cur = k == 0 ? 0u : o.J[k];
    uint32_t nx = k == 0 ? o.first[0] : o.next[k];
    while (nx != OB_NONE) {  // strictly increasing, so at most n hops
      cur = nx;
      nx = o.first[cur];
    }
    o.P[k] = cur;
  }
}
__global__ void k_ob_pairs(const __grid_constant__ DevCtx c, const __grid_constant__ BatchScratch b,
                           OneBox o) {
  const uint32_t n = c.gcount[0], base = c.gstart[0];
  const uint32_t npairs = n / 2;
  const uint64_t key = cleo_rng_key(c.p.seed, *b.tsdm, 0);
  const uint64_t slot_pairs = (uint64_t)b.slot[0] + (n >= 1 ? n - 1 : 0);
  const double scale_p = (double)n * ((double)n - 1.0) / (2.0 * (double)npairs);
  const double VOLUME = c.volume[0] * VOL0;
  uint32_t nnull = 0;
  for (uint32_t jj = blockIdx.x * blockDim.x + threadIdx.x; jj < npairs;
       jj += gridDim.x * blockDim.x) {
    const uint32_t a = o.P[2 * jj], bb = o.P[2 * jj + 1];
    const Where w{c.err, 0u, (uint64_t)base + 2 * jj};
    nnull += collide_pair(c.p, c.sd.xi + base, c.sd.r + base, c.sd.msol + base, a, bb,
                          b.tv[base + a], b.tv[base + bb], scale_p, VOLUME, key, slot_pairs, jj, w);
  }
  if (nnull) atomicAdd(o.nnull, nnull);
}
__global__ void k_ob_flags(const __grid_constant__ DevCtx c, OneBox o) {
  const uint32_t n = c.gcount[0], base = c.gstart[0];
  for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q <= n; q += gridDim.x * blockDim.x)
    o.vflag[q] = q < n && c.sd.xi[base + o.P[q]] != 0 ? 1u : 0u;
}
// destinations after the exclusive scan of vflag: valid superdroplets in shuffled order first,
// then the nulls (collisions.hpp:240-248); the records into scratch
__global__ void k_ob_gather(const __grid_constant__ DevCtx c, OneBox o) {
  const uint32_t n = c.gcount[0], base = c.gstart[0];
  const uint32_t nvalid = n - *o.nnull;
  for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
    const uint32_t before = o.vflag[q];  // valid ones before shuffled position q
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
__global__ void k_ob_commit(const __grid_constant__ DevCtx c, const __grid_constant__ BatchScratch b,
                            OneBox o) {
  const uint32_t n = c.gcount[0], base = c.gstart[0];
  const uint32_t nvalid = n - *o.nnull;
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
__global__ void k_ob_finish(const __grid_constant__ DevCtx c, const __grid_constant__ BatchScratch b,
                            OneBox o) {
  const uint32_t n = c.gcount[0];
  const uint32_t npairs = n / 2;
  const uint64_t slot_pairs = (uint64_t)b.slot[0] + (n >= 1 ? n - 1 : 0);
  c.gcount[0] = n - *o.nnull;
  b.slot[0] = (uint32_t)(slot_pairs + 2ull * npairs);
}

}  // namespace
