// sort_static.cu — the stable sort of superdroplets by gridbox index, without allocating memory.
//
// Some callers of this library cannot call cudaMalloc while they run: a host model that reserves
// all of its device memory at start-up and forbids allocation inside its time loop (allocation
// would also synchronise the whole device in the middle of a coupling step), or a caller whose
// device memory is owned by another framework's pool. For them, this file provides one entry point
// that sorts with scratch memory held in a file-scope device array instead of allocating it.
//
// The scratch array is SCRATCH_BYTES (about 16.3 MiB) and lives in every GPU that loads the
// library until the process exits. It bounds one call to SORT_STATIC_MAX superdroplets. Under
// CUDA's lazy module loading the driver allocates it when this file's code first reaches a
// device, which is the first call's cudaGetSymbolAddress; hence the set-up call with n = 0 that
// callers make at start-up, before they reserve device memory or enter their time loop.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <mutex>

#include "../../include/cleo_b200.h"

namespace {
#include "sort.cuh"  // the radix-sort kernels, given internal linkage in this translation unit
}

namespace {

constexpr uint32_t SORT_STATIC_MAX = 1u << 20;  // superdroplets per call
constexpr uint32_t TILES_MAX = (SORT_STATIC_MAX + cleo::RS_TILE - 1) / cleo::RS_TILE;
constexpr uint32_t HIST_MAX = 256 * TILES_MAX;
constexpr uint32_t SCAN_SUMS_MAX = (HIST_MAX + cleo::SCAN_TILE - 1) / cleo::SCAN_TILE + 1;
// layout (u32 words): keys[2][MAX], vals[2][MAX], hist[HIST_MAX], scan sums, n
constexpr size_t OFF_KEYS0 = 0;
constexpr size_t OFF_KEYS1 = OFF_KEYS0 + SORT_STATIC_MAX;
constexpr size_t OFF_VALS0 = OFF_KEYS1 + SORT_STATIC_MAX;
constexpr size_t OFF_VALS1 = OFF_VALS0 + SORT_STATIC_MAX;
constexpr size_t OFF_HIST = OFF_VALS1 + SORT_STATIC_MAX;
constexpr size_t OFF_SUMS = OFF_HIST + HIST_MAX;
constexpr size_t OFF_N = OFF_SUMS + SCAN_SUMS_MAX;
constexpr size_t SCRATCH_WORDS = OFF_N + 64;
constexpr size_t SCRATCH_BYTES = SCRATCH_WORDS * sizeof(uint32_t);
static_assert(SCRATCH_BYTES < (17u << 20), "the static scratch stays under 17 MiB");

// The scratch memory. In host code this name is only a stand-in for the device symbol: the host
// uses the address returned by cudaGetSymbolAddress, never the name itself.
static __device__ __align__(256) uint32_t g_sort_scratch[SCRATCH_WORDS];

constexpr int MAX_DEVICES = 64;
std::mutex g_setup_mutex;
uint32_t* g_scratch_ptr[MAX_DEVICES] = {};

// keys = min(sdgbxindex, ngbxs) (out-of-domain keys share the last bucket, sortsupers.hpp:44-48)
__global__ void k_static_keys(const uint32_t* __restrict__ gbx, uint32_t n, uint32_t ngbxs,
                              uint32_t* __restrict__ keys, uint32_t* __restrict__ vals,
                              uint32_t* __restrict__ n_slot) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0) *n_slot = n;
  if (i < n) {
    const uint32_t g = gbx[i];
    keys[i] = g < ngbxs ? g : ngbxs;
    vals[i] = i;
  }
}

__global__ void k_static_out(const uint32_t* __restrict__ keys, const uint32_t* __restrict__ vals,
                             uint32_t n, uint32_t ngbxs, uint32_t* __restrict__ order,
                             uint32_t* __restrict__ gstart) {
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += stride) order[j] = vals[j];
  if (!gstart) return;
  // gstart[k] = first sorted position with key >= k, k = 0 .. ngbxs + 1
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < ngbxs + 2; k += stride) {
    uint32_t lo = 0, len = n;
    while (len > 0) {
      const uint32_t half = len >> 1;
      if (keys[lo + half] < k) {
        lo += half + 1;
        len -= half + 1;
      } else {
        len = half;
      }
    }
    gstart[k] = lo;
  }
}

// Once per device, with that device current: the device address of the scratch array.
int scratch_for_current_device(uint32_t** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= MAX_DEVICES) return CLEO_ERR_CUDA;
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_ptr[dev]) {
    uint32_t* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress((void**)&p, g_sort_scratch);
    if (e != cudaSuccess || !p) {
      fprintf(stderr, "cleo_b200: cudaGetSymbolAddress of the sort scratch failed: %s\n",
              cudaGetErrorString(e));
      return CLEO_ERR_CUDA;
    }
    g_scratch_ptr[dev] = p;
  }
  *out = g_scratch_ptr[dev];
  return CLEO_OK;
}

}  // namespace

extern "C" int cleo_b200_sort_by_gridbox_static(const uint32_t* d_sdgbxindex, uint32_t n,
                                                uint32_t ngbxs, uint32_t* d_order,
                                                uint32_t* d_gstart, void* stream) {
  // n = 0: the set-up call a caller makes at start-up (the pointers may be NULL)
  if (n > 0 && (!d_sdgbxindex || !d_order)) return CLEO_ERR_ARGUMENT;
  if (n > SORT_STATIC_MAX) {
    fprintf(stderr,
            "cleo_b200_sort_by_gridbox_static: %u superdroplets exceed the static scratch limit "
            "of %u\n", n, SORT_STATIC_MAX);
    return CLEO_ERR_CAPACITY;
  }
  if (ngbxs >= 0xFFFFFFFEu) return CLEO_ERR_ARGUMENT;
  uint32_t* base = nullptr;
  const int rc = scratch_for_current_device(&base);
  if (rc != CLEO_OK) return rc;
  if (n == 0) {
    if (d_gstart && cudaMemsetAsync(d_gstart, 0, ((size_t)ngbxs + 2) * 4, (cudaStream_t)stream) != cudaSuccess)
      return CLEO_ERR_CUDA;
    return CLEO_OK;
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  uint32_t* keys[2] = {base + OFF_KEYS0, base + OFF_KEYS1};
  uint32_t* vals[2] = {base + OFF_VALS0, base + OFF_VALS1};
  uint32_t* hist = base + OFF_HIST;
  uint32_t* sums = base + OFF_SUMS;
  uint32_t* n_slot = base + OFF_N;
  // every word the passes read is written first in this call (keys/vals for [0, n), the whole
  // digit table by the upsweep), so nothing left by an earlier call needs clearing
  k_static_keys<<<(n + 255) / 256, 256, 0, s>>>(d_sdgbxindex, n, ngbxs, keys[0], vals[0], n_slot);
  uint32_t bits = 0;
  while (bits < 32 && (((uint64_t)1 << bits) <= (uint64_t)ngbxs)) ++bits;
  const uint32_t key_bits = bits == 0 ? 8 : ((bits + 7) / 8) * 8;
  const uint32_t nt = (n + cleo::RS_TILE - 1) / cleo::RS_TILE;
  const uint64_t nh = (uint64_t)256 * nt;
  const uint32_t nscan = (uint32_t)((nh + cleo::SCAN_TILE - 1) / cleo::SCAN_TILE);
  int cur = 0;
  for (uint32_t shift = 0; shift < key_bits; shift += 8) {
    cleo::k_rs_upsweep<<<nt, cleo::RS_THREADS, 0, s>>>(keys[cur], n_slot, (int)shift, hist, nt);
    cleo::k_scan_tiles<<<nscan, cleo::SCAN_THREADS, 0, s>>>(hist, hist, nh, sums);
    cleo::k_scan_sums<<<1, cleo::SCAN_THREADS, 0, s>>>(sums, nscan, nullptr);
    cleo::k_scan_add<<<(unsigned)((nh + 255) / 256), 256, 0, s>>>(hist, nh, sums);
    cleo::k_rs_downsweep<<<nt, cleo::RS_THREADS, 0, s>>>(keys[cur], vals[cur], n_slot, (int)shift,
                                                         hist, nt, keys[1 - cur], vals[1 - cur]);
    cur = 1 - cur;
  }
  const uint32_t outn = n > ngbxs + 2 ? n : ngbxs + 2;
  unsigned blocks = (outn + 255) / 256;
  if (blocks > 148 * 32) blocks = 148 * 32;
  k_static_out<<<blocks, 256, 0, s>>>(keys[cur], vals[cur], n, ngbxs, d_order, d_gstart);
  return cudaGetLastError() == cudaSuccess ? CLEO_OK : CLEO_ERR_CUDA;
}
