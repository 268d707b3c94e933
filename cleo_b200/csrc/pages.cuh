// pages.cuh — the paged layout of the superdroplet store and the re-sort after motion.
//
// Layout. Gridboxes are grouped in pages of PAGE_GBXS consecutive indexes; page p owns the slots
// [pstart[p], pstart[p + 1]) of the SoA buffers: its gridboxes' superdroplets packed in gridbox
// order from pstart[p] (gridbox g: its gcount[g] valid superdroplets from gstart[g], then any null
// ones its collisions left), then free slots up to the page's end ("holes": sdgbxindex out of
// range, xi 0, sdid HOLE_ID). Every kernel that runs over slots already skips an out-of-range
// sdgbxindex; holes lie together at page ends, so whole warps skip them.
//
// Full sort (upload, or when many superdroplets moved): a stable radix sort of all slots by key
// (gridbox, out-of-domain, hole), then every page is written packed with PAGE_SLACK free slots
// after it, out-of-domain superdroplets are appended to the out-of-domain store and holes are
// dropped.
//
// Re-sort after motion (CLEO re-sorts every superdroplet by gridbox after each motion step,
// sortsupers.hpp:93-226; stable). Movers are the valid superdroplets whose gridbox changed and
// the null ones collisions left. Stably sorted by key (in position order, so by their place in
// CLEO's array), they are copied out to a mover buffer; every page that movers leave or enter is
// rewritten in place: gridbox g of it becomes, in order, the movers into g from positions before
// its range, its stayers, the movers into g from positions after it (what the full stable sort
// gives), the page's remaining slots holes. Pages nobody leaves or enters are not touched. If a
// page would outgrow its slots, all pages are rewritten into the other buffer with fresh slack
// and copied back (k_pg_plan decides on the device; both paths are in every captured step and
// the one not taken returns at once).
#pragma once

constexpr uint32_t PAGE_GBXS = 64;   // gridboxes per page (a multiple of 32)
constexpr uint32_t PAGE_SLACK = 64;  // free slots after each page at a full sort
constexpr unsigned long long HOLE_ID = ~0ull;

__device__ __forceinline__ bool is_hole(const Fields& f, uint32_t i) { return f.id[i] == HOLE_ID; }

// sort key of a slot: its gridbox, ngbxs for an out-of-domain or null superdroplet, ngbxs + 1 for
// a hole
__device__ __forceinline__ uint32_t slot_key(const DevCtx& c, uint32_t i) {
  const uint32_t g = c.sd.gbx[i];
  if (g < c.ngbxs) return g;
  return is_hole(c.sd, i) ? c.ngbxs + 1 : c.ngbxs;
}

__device__ __forceinline__ void set_hole(const Fields& f, uint32_t o) {
  f.gbx[o] = OOB;
  f.c3[o] = 0.0;
  f.c1[o] = 0.0;
  f.c2[o] = 0.0;
  f.xi[o] = 0;
  f.r[o] = 0.0;
  f.msol[o] = 0.0;
  f.id[o] = HOLE_ID;
}
__device__ __forceinline__ void copy_rec(const Fields& s, uint32_t i, const Fields& d, uint32_t o) {
  d.gbx[o] = s.gbx[i];
  d.c3[o] = s.c3[i];
  d.c1[o] = s.c1[i];
  d.c2[o] = s.c2[i];
  d.xi[o] = s.xi[i];
  d.r[o] = s.r[i];
  d.msol[o] = s.msol[i];
  d.id[o] = s.id[i];
}

// first index in a[0, n) with a[i] >= v (a ascending)
__device__ __forceinline__ uint32_t lower_bound_u32(const uint32_t* a, uint32_t n, uint32_t v) {
  uint32_t lo = 0, len = n;
  while (len > 0) {
    const uint32_t half = len >> 1;
    if (a[lo + half] < v) {
      lo += half + 1;
      len -= half + 1;
    } else {
      len = half;
    }
  }
  return lo;
}
// the page whose slots hold position i: the last p with pstart[p] <= i
__device__ __forceinline__ uint32_t page_of_slot(const DevCtx& c, uint32_t i) {
  const uint32_t q = lower_bound_u32(c.pstart, c.npages + 1, i + 1);  // first pstart > i
  return q - 1;
}

// ---- full sort ----
__global__ void k_keys_paged(const __grid_constant__ DevCtx c, uint32_t* __restrict__ keys,
                             uint32_t* __restrict__ vals) {
  const uint32_t n = c.counters[0];
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    keys[i] = slot_key(c, i);
    vals[i] = i;
  }
}
// gp[k] = first sorted position with key >= k, k = 0 .. ngbxs + 1 (findrefs.hpp:54-126)
__global__ void k_lower_bounds(const __grid_constant__ DevCtx c, const uint32_t* __restrict__ keys,
                               uint32_t* __restrict__ gp) {
  const uint32_t n = c.counters[0];
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < c.ngbxs + 2;
       k += gridDim.x * blockDim.x)
    gp[k] = lower_bound_u32(keys, n, k);
}
// slots of each page: its superdroplets plus the slack (scanned into pstart)
__global__ void k_pg_sizes_full(const __grid_constant__ DevCtx c, const uint32_t* __restrict__ gp,
                                uint32_t* __restrict__ psize) {
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < c.npages;
       p += gridDim.x * blockDim.x) {
    const uint32_t lo = p * PAGE_GBXS, hi = min(lo + PAGE_GBXS, c.ngbxs);
    psize[p] = gp[hi] - gp[lo] + PAGE_SLACK;
  }
}
// the in-domain superdroplets (sorted positions j < gp[ngbxs]) into their pages of dst
__global__ void __launch_bounds__(256)
k_gather_paged(const __grid_constant__ DevCtx c, Fields src, Fields dst,
               const uint32_t* __restrict__ keys, const uint32_t* __restrict__ perm,
               const uint32_t* __restrict__ gp) {
  const uint32_t nd = gp[c.ngbxs];
  for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < nd; j += gridDim.x * blockDim.x) {
    const uint32_t p = keys[j] / PAGE_GBXS;
    copy_rec(src, perm[j], dst, c.pstart[p] + (j - gp[p * PAGE_GBXS]));
  }
}
// holes after each page's superdroplets; the gridboxes' ranges; the store's ends
__global__ void k_pg_fill_full(const __grid_constant__ DevCtx c, Fields dst,
                               const uint32_t* __restrict__ gp) {
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x, nt = gridDim.x * blockDim.x;
  for (uint32_t p = tid; p < c.npages; p += nt) {
    const uint32_t lo = p * PAGE_GBXS, hi = min(lo + PAGE_GBXS, c.ngbxs);
    for (uint32_t o = c.pstart[p] + (gp[hi] - gp[lo]); o < c.pstart[p + 1]; ++o) set_hole(dst, o);
  }
  for (uint32_t g = tid; g < c.ngbxs; g += nt) {
    const uint32_t p = g / PAGE_GBXS;
    c.gstart[g] = c.pstart[p] + (gp[g] - gp[p * PAGE_GBXS]);
    c.gcount[g] = gp[g + 1] - gp[g];
  }
}
// out-of-domain and null superdroplets (sorted keys == ngbxs) appended to the out-of-domain store
__global__ void k_grave_sorted(const __grid_constant__ DevCtx c, Fields src,
                               const uint32_t* __restrict__ perm, const uint32_t* __restrict__ gp) {
  const uint32_t a = gp[c.ngbxs], b = gp[c.ngbxs + 1], ng0 = c.counters[2];
  for (uint32_t j = a + blockIdx.x * blockDim.x + threadIdx.x; j < b; j += gridDim.x * blockDim.x)
    copy_rec(src, perm[j], c.grave, ng0 + (j - a));
}
__global__ void k_full_commit(const __grid_constant__ DevCtx c, const uint32_t* __restrict__ gp) {
  const uint32_t total = c.pstart[c.npages];
  c.counters[2] += gp[c.ngbxs + 1] - gp[c.ngbxs];
  c.counters[0] = total;
  c.counters[1] = gp[c.ngbxs];
  c.gstart[c.ngbxs] = total;
  c.gstart[c.ngbxs + 1] = total;
}

// ---- re-sort after motion ----
// pg_ctr: [0] pages touched, [1] a page outgrows its slots (repack), [2] movers into the
// out-of-domain store (their first sorted index), [3] the re-sort's stamp (counts re-sorts)
__global__ void k_pg_reset(const __grid_constant__ DevCtx c) {
  c.pg_ctr[0] = 0;
  c.pg_ctr[1] = 0;
  c.pg_ctr[2] = 0;
  c.pg_ctr[3] += 1;
}
// the movers' records, in their sorted order
__global__ void __launch_bounds__(256)
k_mv_gather(const __grid_constant__ DevCtx c, Fields src, const uint32_t* __restrict__ mvp,
            const uint32_t* __restrict__ m_ptr) {
  const uint32_t m = *m_ptr;
  for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < m; j += gridDim.x * blockDim.x)
    copy_rec(src, mvp[j], c.mvrec, j);
}
__device__ __forceinline__ void touch_page(const DevCtx& c, uint32_t p) {
  if (atomicExch(&c.pg_flag[p], 1u) == 0u) c.pg_list[atomicAdd(&c.pg_ctr[0], 1u)] = p;
}
// the pages movers leave or enter
__global__ void k_pg_touch(const __grid_constant__ DevCtx c, const uint32_t* __restrict__ mk,
                           const uint32_t* __restrict__ mvp, const uint32_t* __restrict__ m_ptr) {
  const uint32_t m = *m_ptr;
  for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < m; j += gridDim.x * blockDim.x) {
    const uint32_t k = mk[j];
    if (k < c.ngbxs) touch_page(c, k / PAGE_GBXS);
    touch_page(c, page_of_slot(c, mvp[j]));
    if (j == 0) c.pg_ctr[2] = lower_bound_u32(mk, m, c.ngbxs);
  }
}

// each gridbox's run of sorted movers [mv_lo, mv_hi), stamped with this re-sort's stamp (a
// gridbox whose stamp is older has no arrivals)
__global__ void k_mv_runs(const __grid_constant__ DevCtx c, const uint32_t* __restrict__ mk,
                          const uint32_t* __restrict__ m_ptr) {
  const uint32_t m = *m_ptr, stamp = c.pg_ctr[3];
  for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < m; j += gridDim.x * blockDim.x) {
    const uint32_t k = mk[j];
    if (k >= c.ngbxs) continue;
    if (j == 0 || mk[j - 1] != k) {
      c.mv_lo[k] = j;
      c.mv_stamp[k] = stamp;
    }
    if (j + 1 == m || mk[j + 1] != k) c.mv_hi[k] = j + 1;
  }
}

// One page's new content, worked out by a CTA: per gridbox (a warp each) its stayers counted and
// the sorted movers into it, split at its old start (plan_page); then where each gridbox goes
// (place_page) and which gridboxes are rewritten.
struct PagePlan {
  uint32_t b[PAGE_GBXS];   // old start
  uint32_t oc[PAGE_GBXS];  // old count
  uint32_t ns[PAGE_GBXS];  // stayers
  uint32_t lo[PAGE_GBXS];  // first sorted mover into the gridbox
  uint32_t nl[PAGE_GBXS];  // movers from positions before its old start
  uint32_t na[PAGE_GBXS];  // movers into it
  uint32_t st[PAGE_GBXS];  // new start (absolute slot)
  uint8_t rw[PAGE_GBXS];   // rewritten (content or start changes)
  uint32_t total;          // new count of the page
};
__device__ void plan_page(const DevCtx& c, uint32_t p, const uint32_t* mvp, PagePlan& pl) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  const uint32_t g0 = p * PAGE_GBXS, ng = min(PAGE_GBXS, c.ngbxs - g0);
  for (uint32_t q = warp; q < ng; q += nw) {
    const uint32_t g = g0 + q;
    const uint32_t b = c.gstart[g], n = c.gcount[g];
    uint32_t nst = 0;
    for (uint32_t k0 = 0; k0 < n; k0 += 32) {
      const uint32_t k = k0 + lane;
      nst += __popc(__ballot_sync(0xFFFFFFFFu, k < n && c.sd.gbx[b + k] == g));
    }
    // the movers into g (k_mv_runs), sorted by position: those before its old start lead
    const bool has = c.mv_stamp[g] == c.pg_ctr[3];
    const uint32_t lo = has ? c.mv_lo[g] : 0u, na = has ? c.mv_hi[g] - lo : 0u;
    uint32_t nl = 0;
    for (uint32_t t = lane; t < na; t += 32) nl += mvp[lo + t] < b ? 1u : 0u;
    nl = __reduce_add_sync(0xFFFFFFFFu, nl);
    if (lane == 0) {
      pl.b[q] = b;
      pl.oc[q] = n;
      pl.ns[q] = nst;
      pl.lo[q] = lo;
      pl.na[q] = na;
      pl.nl[q] = nl;
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t s = 0;
    for (uint32_t q = 0; q < ng; ++q) s += pl.ns[q] + pl.na[q];
    pl.total = s;
  }
  __syncthreads();
}
// Where the page's gridboxes go in [pbase, pend). In place (keep), each keeps its start unless
// the one before it now reaches past it, so that a superdroplet moving between neighbouring
// gridboxes rewrites those two and the free slots stay where superdroplets left; when that does
// not fit (or into a fresh page), the gridboxes are packed from pbase. A gridbox is rewritten
// when superdroplets left or entered it or its start moved; the others stay where they are.
__device__ void place_page(const DevCtx& c, uint32_t p, uint32_t pbase, uint32_t pend, bool keep,
                           PagePlan& pl) {
  if (threadIdx.x == 0) {
    const uint32_t ng = min(PAGE_GBXS, c.ngbxs - p * PAGE_GBXS);
    bool fits = false;
    if (keep) {
      uint32_t e = pbase;
      for (uint32_t q = 0; q < ng; ++q) {
        const uint32_t s = max(pl.b[q], e);
        pl.st[q] = s;
        e = s + pl.ns[q] + pl.na[q];
      }
      fits = e <= pend;
    }
    if (!fits) {
      uint32_t e = pbase;
      for (uint32_t q = 0; q < ng; ++q) {
        pl.st[q] = e;
        e += pl.ns[q] + pl.na[q];
      }
    }
    for (uint32_t q = 0; q < ng; ++q)
      pl.rw[q] = (!keep || pl.ns[q] != pl.oc[q] || pl.na[q] != 0 || pl.st[q] != pl.b[q]) ? 1 : 0;
  }
  __syncthreads();
}
// the stayers of the rewritten gridboxes, compacted into the scratch fields at their old ranges
__device__ void stage_page(const DevCtx& c, uint32_t p, const PagePlan& pl) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  const uint32_t g0 = p * PAGE_GBXS, ng = min(PAGE_GBXS, c.ngbxs - g0);
  const Fields& S = c.sd;
  for (uint32_t q = warp; q < ng; q += nw) {
    if (!pl.rw[q]) continue;  // uniform across the warp
    const uint32_t g = g0 + q, b = pl.b[q], n = pl.oc[q];
    uint32_t nst = 0;
    for (uint32_t k0 = 0; k0 < n; k0 += 32) {
      const uint32_t k = k0 + lane;
      const bool st = k < n && S.gbx[b + k] == g;
      const unsigned bal = __ballot_sync(0xFFFFFFFFu, st);
      if (st) {
        const uint32_t o = b + nst + __popc(bal & ((1u << lane) - 1u));
        const uint32_t i = b + k;
        c.scr_c3[o] = S.c3[i];
        c.scr_c1[o] = S.c1[i];
        c.scr_c2[o] = S.c2[i];
        c.scr_x[o] = S.xi[i];
        c.scr_r[o] = S.r[i];
        c.scr_m[o] = S.msol[i];
        c.scr_id[o] = S.id[i];
      }
      nst += __popc(bal);
    }
  }
  __syncthreads();
}

// whether every touched page still fits its slots (else pg_ctr[1] = 1: repack)
__global__ void __launch_bounds__(256)
k_pg_plan(const __grid_constant__ DevCtx c, const uint32_t* __restrict__ mk,
          const uint32_t* __restrict__ mvp, const uint32_t* __restrict__ m_ptr) {
  __shared__ PagePlan pl;
  const uint32_t np = c.pg_ctr[0];
  for (uint32_t it = blockIdx.x; it < np; it += gridDim.x) {
    const uint32_t p = c.pg_list[it];
    plan_page(c, p, mvp, pl);
    if (threadIdx.x == 0 && pl.total > c.pstart[p + 1] - c.pstart[p]) atomicExch(&c.pg_ctr[1], 1u);
    __syncthreads();
  }
}

// A page written from its plan: REPACK = false rewrites the touched pages in place (taken when no
// page outgrows its slots), REPACK = true writes every page packed into dst at the new page starts
// (taken when one does; then dst is copied back). Every slot of the page outside its gridboxes'
// new ranges is left a hole.
template <bool REPACK>
__global__ void __launch_bounds__(256, 4)  // (256) alone caps it at 32 registers, with spills
k_pg_write(const __grid_constant__ DevCtx c, Fields dst, const uint32_t* __restrict__ mk,
           const uint32_t* __restrict__ mvp, const uint32_t* __restrict__ m_ptr,
           const uint32_t* __restrict__ pnew) {
  __shared__ PagePlan pl;
  if ((c.pg_ctr[1] != 0) != REPACK) return;  // the other path is taken
  const uint32_t np = REPACK ? c.npages : c.pg_ctr[0];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  const Fields& M = c.mvrec;
  for (uint32_t it = blockIdx.x; it < np; it += gridDim.x) {
    const uint32_t p = REPACK ? it : c.pg_list[it];
    plan_page(c, p, mvp, pl);
    const uint32_t g0 = p * PAGE_GBXS, ng = min(PAGE_GBXS, c.ngbxs - g0);
    const uint32_t base = pnew[p], end = pnew[p + 1];
    place_page(c, p, base, end, !REPACK, pl);
    stage_page(c, p, pl);
    for (uint32_t q = warp; q < ng; q += nw) {
      const uint32_t g = g0 + q, ns = pl.st[q];
      const uint32_t nl = pl.nl[q], nst = pl.ns[q], na = pl.na[q], lo = pl.lo[q], b = pl.b[q];
      if (pl.rw[q]) {
        for (uint32_t t = lane; t < na + nst; t += 32) {
          const bool arrival = t < nl || t >= nl + nst;
          const uint32_t o = ns + t;
          if (arrival) {
            copy_rec(M, lo + (t < nl ? t : t - nst), dst, o);
          } else {
            const uint32_t i = b + (t - nl);
            dst.gbx[o] = g;
            dst.c3[o] = c.scr_c3[i];
            dst.c1[o] = c.scr_c1[i];
            dst.c2[o] = c.scr_c2[i];
            dst.xi[o] = c.scr_x[i];
            dst.r[o] = c.scr_r[i];
            dst.msol[o] = c.scr_m[i];
            dst.id[o] = c.scr_id[i];
          }
        }
      }
      // the free slots after the gridbox, up to the next one's start (or the page's end), and
      // before the first one
      const uint32_t gap_end = q + 1 < ng ? pl.st[q + 1] : end;
      for (uint32_t o = ns + na + nst + lane; o < gap_end; o += 32) set_hole(dst, o);
      if (q == 0)
        for (uint32_t o = base + lane; o < ns; o += 32) set_hole(dst, o);
    }
    __syncthreads();  // every warp has read the page's old starts from pl
    for (uint32_t q = threadIdx.x; q < ng; q += blockDim.x) {
      c.gstart[g0 + q] = pl.st[q];
      c.gcount[g0 + q] = pl.ns[q] + pl.na[q];
    }
    if (!REPACK && threadIdx.x == 0) c.pg_flag[p] = 0;
    __syncthreads();
  }
}
// repack path: page sizes for the new starts (every page: its new count plus the slack)
__global__ void __launch_bounds__(256)
k_pg_sizes_repack(const __grid_constant__ DevCtx c, const uint32_t* __restrict__ mk,
                  const uint32_t* __restrict__ mvp, const uint32_t* __restrict__ m_ptr,
                  uint32_t* __restrict__ psize) {
  __shared__ PagePlan pl;
  if (c.pg_ctr[1] == 0) return;
  for (uint32_t p = blockIdx.x; p < c.npages; p += gridDim.x) {
    plan_page(c, p, mvp, pl);
    if (threadIdx.x == 0) psize[p] = pl.total + PAGE_SLACK;
    __syncthreads();
  }
}
// repack path: the rewritten store back into the current buffer, the new page starts
__global__ void __launch_bounds__(256)
k_pg_copy_back(const __grid_constant__ DevCtx c, Fields src, const uint32_t* __restrict__ pnew) {
  if (c.pg_ctr[1] == 0) return;
  const uint32_t total = pnew[c.npages];
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x)
    copy_rec(src, i, c.sd, i);
}
__global__ void k_pg_commit(const __grid_constant__ DevCtx c, const uint32_t* __restrict__ pnew) {
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x, nt = gridDim.x * blockDim.x;
  const bool repack = c.pg_ctr[1] != 0;
  if (repack) {
    for (uint32_t p = tid; p <= c.npages; p += nt) c.pstart[p] = pnew[p];
    for (uint32_t i = tid; i < c.pg_ctr[0]; i += nt) c.pg_flag[c.pg_list[i]] = 0;
  }
  if (tid == 0) {
    const uint32_t total = repack ? pnew[c.npages] : c.counters[0];
    c.counters[0] = total;
    c.gstart[c.ngbxs] = total;
    c.gstart[c.ngbxs + 1] = total;
  }
}
// movers out of the domain (and null ones) appended to the out-of-domain store
__global__ void k_grave_movers(const __grid_constant__ DevCtx c, const uint32_t* __restrict__ m_ptr) {
  const uint32_t m = *m_ptr, a = c.pg_ctr[2], ng0 = c.counters[2];
  for (uint32_t j = a + blockIdx.x * blockDim.x + threadIdx.x; j < m; j += gridDim.x * blockDim.x)
    copy_rec(c.mvrec, j, c.grave, ng0 + (j - a));
}
__global__ void k_grave_movers_commit(const __grid_constant__ DevCtx c,
                                      const uint32_t* __restrict__ m_ptr) {
  c.counters[2] += *m_ptr - c.pg_ctr[2];
}
