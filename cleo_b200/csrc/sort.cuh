// sort.cuh — stable counting sort of superdroplets by gridbox index on the GPU.
//
// Replaces SortSupersBySdgbxindex (libs/gridboxes/sortsupers.hpp:93-226): the reference builds a
// histogram of sdgbxindex (out-of-domain keys share the last bucket), an exclusive scan and a
// scatter with atomic_fetch_add, which is stable only on the Serial backend. Here the scatter is
// made stable on the GPU by a least-significant-digit radix sort of (key, position) pairs with
// 8-bit digits: per digit pass, every tile of 4096 keys counts its digits (upsweep), the
// digit-major table of tile counts is scanned, and each tile ranks its keys stably with warp
// match/ballot (downsweep). No block waits on another block.
#pragma once

#include <cstdint>

namespace cleo {

constexpr int RS_THREADS = 256;
constexpr int RS_ITEMS = 16;
constexpr int RS_TILE = RS_THREADS * RS_ITEMS;
constexpr int RS_WARPS = RS_THREADS / 32;
constexpr int SCAN_THREADS = 1024;
constexpr int SCAN_ITEMS = 4;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;

// per-tile digit counts; hist is digit-major: hist[d * ntiles + tile]. With small_n > 0 the
// pass does nothing for n <= small_n (k_rs_small sorts those in one block).
__global__ void __launch_bounds__(RS_THREADS)
k_rs_upsweep(const uint32_t* __restrict__ keys, const uint32_t* __restrict__ n_ptr, int shift,
             uint32_t* __restrict__ hist, uint32_t ntiles, uint32_t small_n = 0) {
  __shared__ uint32_t cnt[256];
  const uint32_t n = *n_ptr;
  if (small_n > 0 && n <= small_n) return;
  for (int i = threadIdx.x; i < 256; i += RS_THREADS) cnt[i] = 0;
  __syncthreads();
  const uint32_t tile = blockIdx.x;
  const uint64_t base = (uint64_t)tile * RS_TILE;
#pragma unroll
  for (int k = 0; k < RS_ITEMS; ++k) {
    const uint64_t idx = base + (uint64_t)k * RS_THREADS + threadIdx.x;
    if (idx < n) atomicAdd(&cnt[(keys[idx] >> shift) & 255u], 1u);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < 256; i += RS_THREADS) hist[(uint64_t)i * ntiles + tile] = cnt[i];
}

// stable scatter of one digit pass
__global__ void __launch_bounds__(RS_THREADS)
k_rs_downsweep(const uint32_t* __restrict__ kin, const uint32_t* __restrict__ vin,
               const uint32_t* __restrict__ n_ptr, int shift, const uint32_t* __restrict__ offs,
               uint32_t ntiles, uint32_t* __restrict__ kout, uint32_t* __restrict__ vout,
               uint32_t small_n = 0) {
  __shared__ uint32_t wcount[RS_WARPS][256];
  __shared__ uint32_t dbase[256];
  const uint32_t n = *n_ptr;
  const uint32_t tile = blockIdx.x;
  const uint64_t base = (uint64_t)tile * RS_TILE;
  if (base >= n || (small_n > 0 && n <= small_n)) return;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int i = threadIdx.x; i < RS_WARPS * 256; i += RS_THREADS) (&wcount[0][0])[i] = 0;
  for (int i = threadIdx.x; i < 256; i += RS_THREADS) dbase[i] = offs[(uint64_t)i * ntiles + tile];
  __syncthreads();
  const unsigned lt = (1u << lane) - 1u;
  uint32_t kk[RS_ITEMS], vv[RS_ITEMS], rk[RS_ITEMS];
  // warp w owns the contiguous chunk [w*32*ITEMS, (w+1)*32*ITEMS) of the tile, read in rounds of
  // 32 consecutive keys: rank order = array order
#pragma unroll
  for (int j = 0; j < RS_ITEMS; ++j) {
    const uint64_t idx = base + (uint64_t)warp * 32 * RS_ITEMS + (uint64_t)j * 32 + lane;
    const bool valid = idx < n;
    kk[j] = valid ? kin[idx] : 0u;
    vv[j] = valid ? vin[idx] : 0u;
    const uint32_t d = valid ? ((kk[j] >> shift) & 255u) : 256u;
    const unsigned peers = __match_any_sync(0xFFFFFFFFu, d);
    const int leader = __ffs(peers) - 1;
    uint32_t prev = 0;
    if (valid) prev = wcount[warp][d];
    __syncwarp();
    if (valid && lane == leader) wcount[warp][d] = prev + __popc(peers);
    __syncwarp();
    rk[j] = valid ? (prev + __popc(peers & lt)) : 0xFFFFFFFFu;
  }
  __syncthreads();
  for (int d = threadIdx.x; d < 256; d += RS_THREADS) {
    uint32_t s = 0;
#pragma unroll
    for (int w = 0; w < RS_WARPS; ++w) {
      const uint32_t c = wcount[w][d];
      wcount[w][d] = s;
      s += c;
    }
  }
  __syncthreads();
#pragma unroll
  for (int j = 0; j < RS_ITEMS; ++j) {
    if (rk[j] != 0xFFFFFFFFu) {
      const uint32_t d = (kk[j] >> shift) & 255u;
      const uint32_t pos = dbase[d] + wcount[warp][d] + rk[j];
      kout[pos] = kk[j];
      vout[pos] = vv[j];
    }
  }
}

// The same stable LSD sort for n <= RS_SMALL_MAX pairs (device count) in one block of
// RS_SMALL_THREADS: `bits` key bits in 8-bit passes between (k0, v0) and (k1, v1), leaving the
// result where the multi-tile passes would (in (k0, v0) after an even number of passes). Returns
// at once for larger n, which the multi-tile passes sort.
constexpr int RS_SMALL_THREADS = 1024;
constexpr int RS_SMALL_WARPS = RS_SMALL_THREADS / 32;
constexpr uint32_t RS_SMALL_MAX = (uint32_t)RS_SMALL_THREADS * RS_ITEMS;  // 16384
__global__ void __launch_bounds__(RS_SMALL_THREADS)
k_rs_small(uint32_t* __restrict__ k0, uint32_t* __restrict__ v0, uint32_t* __restrict__ k1,
           uint32_t* __restrict__ v1, const uint32_t* __restrict__ n_ptr, uint32_t bits,
           uint32_t unsorted_max = 0) {
  __shared__ uint32_t wcount[RS_SMALL_WARPS][256];
  __shared__ uint32_t dbase[256];
  __shared__ uint32_t wsum[8];
  const uint32_t n = *n_ptr;
  if (n > RS_SMALL_MAX || n <= unsorted_max) return;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const unsigned lt = (1u << lane) - 1u;
  uint32_t* K[2] = {k0, k1};
  uint32_t* V[2] = {v0, v1};
  int cur = 0;
  for (uint32_t shift = 0; shift < bits; shift += 8) {
    for (int i = threadIdx.x; i < RS_SMALL_WARPS * 256; i += RS_SMALL_THREADS)
      (&wcount[0][0])[i] = 0;
    __syncthreads();
    uint32_t kk[RS_ITEMS], vv[RS_ITEMS], rk[RS_ITEMS];
#pragma unroll
    for (int j = 0; j < RS_ITEMS; ++j) {  // array order = rank order, as in k_rs_downsweep
      const uint32_t idx = (uint32_t)warp * 32 * RS_ITEMS + (uint32_t)j * 32 + lane;
      const bool valid = idx < n;
      kk[j] = valid ? K[cur][idx] : 0u;
      vv[j] = valid ? V[cur][idx] : 0u;
      const uint32_t d = valid ? ((kk[j] >> shift) & 255u) : 256u;
      const unsigned peers = __match_any_sync(0xFFFFFFFFu, d);
      const int leader = __ffs(peers) - 1;
      uint32_t prev = 0;
      if (valid) prev = wcount[warp][d];
      __syncwarp();
      if (valid && lane == leader) wcount[warp][d] = prev + __popc(peers);
      __syncwarp();
      rk[j] = valid ? (prev + __popc(peers & lt)) : 0xFFFFFFFFu;
    }
    __syncthreads();
    // digit d = thread d < 256: its per-warp offsets, then the exclusive scan of the digit totals
    // over the first 8 warps
    const uint32_t d = threadIdx.x;
    uint32_t tot = 0, x = 0;
    if (d < 256) {
      for (int w = 0; w < RS_SMALL_WARPS; ++w) {
        const uint32_t c = wcount[w][d];
        wcount[w][d] = tot;
        tot += c;
      }
      x = tot;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
        if (lane >= o) x += y;
      }
      if (lane == 31) wsum[warp] = x;
    }
    __syncthreads();
    if (d < 256) {
      uint32_t before = 0;
      for (int w = 0; w < warp; ++w) before += wsum[w];
      dbase[d] = before + x - tot;
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < RS_ITEMS; ++j) {
      if (rk[j] != 0xFFFFFFFFu) {
        const uint32_t dg = (kk[j] >> shift) & 255u;
        const uint32_t pos = dbase[dg] + wcount[warp][dg] + rk[j];
        K[1 - cur][pos] = kk[j];
        V[1 - cur][pos] = vv[j];
      }
    }
    __syncthreads();  // this pass's writes before the next pass reads them
    cur ^= 1;
  }
}

// ---- exclusive scan of u32 (reduce-then-scan over tiles of SCAN_TILE) ----
// The scan kernels take an optional gate: with gate set they do nothing while *gate <= gate_max
// (the digit tables of a multi-tile radix pass that k_rs_small replaces).
__device__ __forceinline__ uint32_t block_exclusive_scan_1024(uint32_t v, uint32_t* wsum,
                                                              uint32_t& total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) wsum[warp] = x;
  __syncthreads();
  if (warp == 0) {
    uint32_t s = (lane < (int)(blockDim.x >> 5)) ? wsum[lane] : 0u;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, s, o);
      if (lane >= o) s += y;
    }
    wsum[lane] = s;  // inclusive over warps
  }
  __syncthreads();
  total = wsum[(blockDim.x >> 5) - 1];
  const uint32_t before = warp > 0 ? wsum[warp - 1] : 0u;
  __syncthreads();
  return before + x - v;
}

// phase 1: scan each tile, write the tile's total
__global__ void __launch_bounds__(SCAN_THREADS)
k_scan_tiles(const uint32_t* in, uint32_t* out, uint64_t n,  // in == out: scanned in place
             uint32_t* __restrict__ tile_sums, const uint32_t* gate = nullptr,
             uint32_t gate_max = 0) {
  __shared__ uint32_t wsum[32];
  if (gate && *gate <= gate_max) return;
  const uint64_t base = (uint64_t)blockIdx.x * SCAN_TILE + (uint64_t)threadIdx.x * SCAN_ITEMS;
  uint32_t v[SCAN_ITEMS], s = 0;
#pragma unroll
  for (int k = 0; k < SCAN_ITEMS; ++k) {
    v[k] = (base + k < n) ? in[base + k] : 0u;
    s += v[k];
  }
  uint32_t total;
  uint32_t run = block_exclusive_scan_1024(s, wsum, total);
#pragma unroll
  for (int k = 0; k < SCAN_ITEMS; ++k) {
    if (base + k < n) out[base + k] = run;
    run += v[k];
  }
  if (threadIdx.x == 0) tile_sums[blockIdx.x] = total;
}

// phase 2: one block scans the tile totals (exclusive, in place); *grand gets the total
__global__ void __launch_bounds__(SCAN_THREADS)
k_scan_sums(uint32_t* __restrict__ sums, uint32_t nsums, uint32_t* __restrict__ grand,
            const uint32_t* gate = nullptr, uint32_t gate_max = 0) {
  __shared__ uint32_t wsum[32];
  if (gate && *gate <= gate_max) return;
  uint32_t carry = 0;
  for (uint32_t start = 0; start < nsums; start += SCAN_THREADS) {
    const uint32_t i = start + threadIdx.x;
    const uint32_t v = i < nsums ? sums[i] : 0u;
    uint32_t total;
    const uint32_t ex = block_exclusive_scan_1024(v, wsum, total);
    if (i < nsums) sums[i] = carry + ex;
    carry += total;
  }
  if (threadIdx.x == 0 && grand) *grand = carry;
}

// phase 3: add the scanned tile totals
__global__ void k_scan_add(uint32_t* __restrict__ out, uint64_t n,
                           const uint32_t* __restrict__ tile_sums, const uint32_t* gate = nullptr,
                           uint32_t gate_max = 0) {
  if (gate && *gate <= gate_max) return;
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] += tile_sums[i / SCAN_TILE];
}

}  // namespace cleo
