// mlp.cuh — the condensation surrogate: a 7 -> 64 -> 64 -> 1 multilayer perceptron (GELU) that
// predicts the post-step r^2 of ImplicitEuler::solve_condensation (impliciteuler.cpp:35-54) and
// seeds the FP64 Newton-Raphson iteration with it. The reference has no such model; its solver
// starts from ImplicitIterations::initialguess (impliciteuler.cpp:156-170).
//
// Inputs (raw features, float): log r, log msol, s_ratio - 1, T, p, delt (all in the reference's
// dimensionless units) and log(3 b / a), the squared activation radius of the Koehler curve
// (impliciteuler.cpp:75). Output: log(z_new / r^2), z = r^2 the Newton variable. Features and
// target are standardised with per-model means and scales.
//
// Inference uses BF16 weights with FP32 accumulation:
//   layer 1 (7 -> 64): FP32 CUDA-core arithmetic on the BF16-rounded weights, GELU, BF16 result;
//   layer 2 (64 -> 64): tcgen05.mma kind::f16, A = the BF16 hidden layer of 128 samples staged in
//     shared memory, B = W2 (BF16, K-major), D = FP32 accumulator in tensor memory;
//   layer 3 (64 -> 1): FP32 dot product of GELU(D + b2) with the BF16-rounded W3.
// A warp-level mma.sync m16n8k16 kernel and a scalar FP32 kernel compute the same function and
// check the tensor-core path.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "physics.cuh"

namespace cleo {
namespace mlp {

constexpr int NIN = 7;
constexpr int NH = 64;
// parameter vector (FP32 master copy): W1[64][7], b1[64], W2[64][64], b2[64], W3[64], b3
constexpr int OFF_W1 = 0;
constexpr int OFF_B1 = OFF_W1 + NH * NIN;  // 448
constexpr int OFF_W2 = OFF_B1 + NH;        // 512
constexpr int OFF_B2 = OFF_W2 + NH * NH;   // 4608
constexpr int OFF_W3 = OFF_B2 + NH;        // 4672
constexpr int OFF_B3 = OFF_W3 + NH;        // 4736
constexpr int NPARAM = OFF_B3 + 1;         // 4737
// normalisation: feature means [0,7), feature inverse scales [7,14), target mean 14, scale 15
constexpr int NNORM = 16;

// inference constants in one float array (BF16-rounded weights stored as float)
constexpr int FW_W1 = 0;
constexpr int FW_B1 = FW_W1 + NH * NIN;
constexpr int FW_B2 = FW_B1 + NH;
constexpr int FW_W3 = FW_B2 + NH;
constexpr int FW_B3 = FW_W3 + NH;
constexpr int FW_NORM = FW_B3 + 1;
constexpr int NFW = FW_NORM + NNORM;  // 657

// W2 as the B operand of tcgen05.mma: K-major, no swizzle. Core matrices of 8 rows x 16 bytes
// (8 BF16 along K); core (kc, ng) for K chunk kc = k/8 and row group ng = n/8 sits at byte
// (kc * 8 + ng) * 128. Leading byte offset (between K-adjacent cores) 1024, stride byte offset
// (between 8-row groups) 128.
constexpr uint32_t W2_UMMA_BYTES = NH * NH * 2;  // 8192
constexpr uint32_t B_LBO = 8 * 128;
constexpr uint32_t B_SBO = 128;
// The A tile (128 samples x 64 hidden, BF16): core (kc, mg) at (kc * 16 + mg) * 128.
constexpr uint32_t TILE_M = 128;
constexpr uint32_t A_BYTES = TILE_M * NH * 2;  // 16384
constexpr uint32_t A_LBO = 16 * 128;
constexpr uint32_t A_SBO = 128;
constexpr uint32_t TMEM_COLS = 64;  // FP32 accumulator of N = 64 columns, M = 128 lanes

struct Infer {
  const float* fw;        // NFW floats
  const uint4* w2_umma;   // W2_UMMA_BYTES, canonical layout above
  const uint32_t* w2_rm;  // W2 row-major, BF16 pairs: w2_rm[n * 32 + k / 2]
  uint32_t* err;          // device status word: the first cleo_status failure is kept
};

__device__ __forceinline__ float gelu(float x) {
  return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f));
}
__device__ __forceinline__ float gelu_grad(float x) {
  const float cdf = 0.5f * (1.0f + erff(x * 0.70710678118654752f));
  const float pdf = 0.39894228040143268f * expf(-0.5f * x * x);
  return cdf + x * pdf;
}
__device__ __forceinline__ uint32_t pack_bf16x2(float lo, float hi) {
  const uint32_t a = __bfloat16_as_ushort(__float2bfloat16_rn(lo));
  const uint32_t b = __bfloat16_as_ushort(__float2bfloat16_rn(hi));
  return a | (b << 16);
}
__device__ __forceinline__ float bf16_round(float x) {
  return __bfloat162float(__float2bfloat16_rn(x));
}

// raw features of one droplet (Koehler factors as condensation.cpp:49-51). The network is FP32
// with BF16 weights, so the logarithms are taken in single precision: they shape a seed that the
// FP64 Newton iteration then judges, and FP64 logarithms would cost as much as several Newton
// iterations.
__device__ __forceinline__ void raw_features(double r, double msol, double temp, double press,
                                             double s_ratio, double delt, float x[NIN]) {
  double akoh, bkoh;
  kohler_factors(msol, temp, akoh, bkoh);
  x[0] = logf((float)r);
  x[1] = logf((float)msol);
  x[2] = (float)(s_ratio - 1.0);
  x[3] = (float)temp;
  x[4] = (float)press;
  x[5] = (float)delt;
  x[6] = logf((float)(3.0 * bkoh / akoh));
}
// the Newton seed r^2 exp(t) from the network's output t = log(z_new / r^2)
__device__ __forceinline__ double seed_from(double r, float t) { return r * r * (double)expf(t); }

// standardised features from raw ones
__device__ __forceinline__ void normalise(const float* fw, float x[NIN]) {
#pragma unroll
  for (int i = 0; i < NIN; ++i) x[i] = (x[i] - fw[FW_NORM + i]) * fw[FW_NORM + NIN + i];
}
__device__ __forceinline__ float denormalise(const float* fw, float y) {
  return fw[FW_NORM + 14] + fw[FW_NORM + 15] * y;
}
// hidden unit k of layer 1 (FP32 accumulation over the BF16-rounded weights)
__device__ __forceinline__ float hidden1(const float* fw, const float x[NIN], int k) {
  float a = fw[FW_B1 + k];
#pragma unroll
  for (int i = 0; i < NIN; ++i) a += fw[FW_W1 + k * NIN + i] * x[i];
  return gelu(a);
}

// ---- tcgen05 primitives (PTX ISA 8.6+, sm_100a) ----
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;  // descriptor version of sm_100
  return d;                // base offset 0, legacy LBO mode, layout SWIZZLE_NONE (0)
}
// instruction descriptor of kind::f16: D F32, A and B BF16, both K-major, N = 64, M = 128
constexpr uint32_t UMMA_IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((64u >> 3) << 17) |
                                ((128u >> 4) << 24);

__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// bounded wait on an mbarrier phase; false when the bound ran out
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity,
                                                  uint32_t max_tries) {
  for (uint32_t t = 0; t < max_tries; ++t)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols) {  // one full warp
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                   smem_u32(slot)),
               "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {  // one full warp
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols)
               : "memory");
}
__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                          uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(UMMA_IDESC), "r"(accumulate)
      : "memory");
}
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
          smem_u32(bar))
      : "memory");
}
// 32 lanes x 32 bit, 16 consecutive columns per thread
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float v[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
      "%11, %12, %13, %14, %15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
        "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
#pragma unroll
  for (int j = 0; j < 16; ++j) v[j] = __uint_as_float(r[j]);
}
__device__ __forceinline__ void tmem_wait_ld() {
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// shared memory of the tensor-core kernel
constexpr uint32_t SM_A = 0;
constexpr uint32_t SM_B = SM_A + A_BYTES;                             // 16384
constexpr uint32_t SM_FW = SM_B + W2_UMMA_BYTES;                      // 24576
constexpr uint32_t SM_BAR = SM_FW + ((NFW * 4 + 15) / 16) * 16;       // 27216
constexpr uint32_t SM_TSLOT = SM_BAR + 8;
constexpr uint32_t TC_SMEM = 32768;  // rounded up: at most 7 CTAs per SM, 448 of 512 TMEM columns
// persistent grid of the tensor-core kernel: every SM's 7 resident CTAs (tile phases of different
// CTAs overlap: the CUDA-core layers of one with the MMA of another)
constexpr uint32_t TC_GRID_MAX = 148u * 7u;
static_assert(SM_TSLOT + 4 <= TC_SMEM, "tensor-core kernel shared memory");
constexpr uint32_t MBAR_TRIES = 1u << 22;

// One persistent CTA of 128 threads per tile of 128 samples; thread t owns sample row t.
// IO supplies raw features (io.features(i, x)) and consumes the denormalised output
// (io.store(i, t)).
template <class IO>
__global__ void __launch_bounds__(128) k_mlp_tc(Infer w, IO io, uint32_t n) {
  extern __shared__ __align__(1024) uint8_t smem[];
  uint8_t* sA = smem + SM_A;
  uint4* sB = reinterpret_cast<uint4*>(smem + SM_B);
  float* sF = reinterpret_cast<float*>(smem + SM_FW);
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem + SM_BAR);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(smem + SM_TSLOT);
  const uint32_t tid = threadIdx.x, warp = tid >> 5;

  for (uint32_t i = tid; i < W2_UMMA_BYTES / 16; i += 128) sB[i] = w.w2_umma[i];
  for (uint32_t i = tid; i < (uint32_t)NFW; i += 128) sF[i] = w.fw[i];
  if (tid == 0) mbar_init(bar, 1);
  if (warp == 0) tmem_alloc(tslot, TMEM_COLS);
  fence_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tslot;
  const uint32_t a_addr = smem_u32(sA), b_addr = smem_u32(sB);
  uint32_t phase = 0;

  n = io.rows(n);  // an IO may hold its row count in device memory (the same for every thread)
  for (uint32_t tile = blockIdx.x; (size_t)tile * TILE_M < n; tile += gridDim.x) {
    const uint32_t i = tile * TILE_M + tid;
    const bool valid = i < n;
    float x[NIN];
#pragma unroll
    for (int q = 0; q < NIN; ++q) x[q] = 0.0f;
    if (valid) io.features(i, x);
    normalise(sF, x);
    // layer 1 -> BF16 A tile, one 16-byte row segment of a core matrix per K chunk
#pragma unroll 1
    for (uint32_t kc = 0; kc < NH / 8; ++kc) {
      uint4 v;
      v.x = pack_bf16x2(hidden1(sF, x, kc * 8 + 0), hidden1(sF, x, kc * 8 + 1));
      v.y = pack_bf16x2(hidden1(sF, x, kc * 8 + 2), hidden1(sF, x, kc * 8 + 3));
      v.z = pack_bf16x2(hidden1(sF, x, kc * 8 + 4), hidden1(sF, x, kc * 8 + 5));
      v.w = pack_bf16x2(hidden1(sF, x, kc * 8 + 6), hidden1(sF, x, kc * 8 + 7));
      *reinterpret_cast<uint4*>(sA + (kc * 16 + (tid >> 3)) * 128 + (tid & 7) * 16) = v;
    }
    fence_async_smem();
    __syncthreads();
    if (tid == 0) {
      tc_fence_after();
#pragma unroll
      for (uint32_t s = 0; s < NH / 16; ++s)
        umma_bf16(tmem, umma_desc(a_addr + s * 2 * A_LBO, A_LBO, A_SBO),
                  umma_desc(b_addr + s * 2 * B_LBO, B_LBO, B_SBO), s > 0 ? 1u : 0u);
      umma_commit(bar);
    }
    const bool ok = mbar_wait_bounded(bar, phase, MBAR_TRIES);
    if (__syncthreads_or(!ok)) {
      if (tid == 0) atomicCAS(w.err, 0u, (uint32_t)CLEO_ERR_TIMEOUT);
      mbar_wait_bounded(bar, phase, MBAR_TRIES);  // let the MMA in flight finish
      break;
    }
    phase ^= 1u;
    tc_fence_after();
    float y = sF[FW_B3];
#pragma unroll
    for (uint32_t c = 0; c < NH / 16; ++c) {
      float acc[16];
      tmem_ld16(tmem + ((warp * 32u) << 16) + c * 16u, acc);
      tmem_wait_ld();
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        const int col = (int)c * 16 + j;
        y += sF[FW_W3 + col] * gelu(acc[j] + sF[FW_B2 + col]);
      }
    }
    if (valid) io.store(i, denormalise(sF, y));
    tc_fence_before();
    __syncthreads();
  }
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, TMEM_COLS);
}

// Check path 1: warp-level mma.sync m16n8k16 (BF16 in, FP32 accumulate). Each warp evaluates
// 16 samples per iteration; lanes 0-15 compute the hidden layer 1 rows into shared memory.
constexpr int MMA_WARPS = 4;
constexpr int H1_LD = NH + 8;  // BF16 row stride of the staged hidden layer (bank spread)
template <class IO>
__global__ void __launch_bounds__(128) k_mlp_mma(Infer w, IO io, uint32_t n) {
  __shared__ float sF[NFW];
  __shared__ __align__(16) __nv_bfloat16 sH[MMA_WARPS][16][H1_LD];
  for (uint32_t i = threadIdx.x; i < (uint32_t)NFW; i += blockDim.x) sF[i] = w.fw[i];
  __syncthreads();
  const uint32_t lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const uint32_t g = lane >> 2, t = lane & 3;
  const uint32_t nwarps = gridDim.x * MMA_WARPS;
  for (uint32_t tile = blockIdx.x * MMA_WARPS + wid; (size_t)tile * 16 < n; tile += nwarps) {
    const uint32_t base = tile * 16;
    if (lane < 16) {
      const uint32_t i = base + lane;
      float x[NIN];
#pragma unroll
      for (int q = 0; q < NIN; ++q) x[q] = 0.0f;
      if (i < n) io.features(i, x);
      normalise(sF, x);
      for (int k = 0; k < NH; ++k) sH[wid][lane][k] = __float2bfloat16_rn(hidden1(sF, x, k));
    }
    __syncwarp();
    float yg = 0.0f, yg8 = 0.0f;  // partial outputs of rows g and g + 8
#pragma unroll 1
    for (int nt = 0; nt < NH / 8; ++nt) {
      float c0 = 0.f, c1 = 0.f, c2 = 0.f, c3 = 0.f;
#pragma unroll
      for (int ks = 0; ks < NH / 16; ++ks) {
        const int kb = ks * 16;
        const uint32_t a0 = *reinterpret_cast<const uint32_t*>(&sH[wid][g][kb + 2 * t]);
        const uint32_t a1 = *reinterpret_cast<const uint32_t*>(&sH[wid][g + 8][kb + 2 * t]);
        const uint32_t a2 = *reinterpret_cast<const uint32_t*>(&sH[wid][g][kb + 8 + 2 * t]);
        const uint32_t a3 = *reinterpret_cast<const uint32_t*>(&sH[wid][g + 8][kb + 8 + 2 * t]);
        const uint32_t b0 = w.w2_rm[(nt * 8 + g) * 32 + (kb + 2 * t) / 2];
        const uint32_t b1 = w.w2_rm[(nt * 8 + g) * 32 + (kb + 8 + 2 * t) / 2];
        asm volatile(
            "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0, %1, %2, %3}, "
            "{%4, %5, %6, %7}, {%8, %9}, {%0, %1, %2, %3};"
            : "+f"(c0), "+f"(c1), "+f"(c2), "+f"(c3)
            : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
      }
      const int col = nt * 8 + 2 * (int)t;
      yg += sF[FW_W3 + col] * gelu(c0 + sF[FW_B2 + col]) +
            sF[FW_W3 + col + 1] * gelu(c1 + sF[FW_B2 + col + 1]);
      yg8 += sF[FW_W3 + col] * gelu(c2 + sF[FW_B2 + col]) +
             sF[FW_W3 + col + 1] * gelu(c3 + sF[FW_B2 + col + 1]);
    }
    yg += __shfl_xor_sync(0xFFFFFFFFu, yg, 1);
    yg += __shfl_xor_sync(0xFFFFFFFFu, yg, 2);
    yg8 += __shfl_xor_sync(0xFFFFFFFFu, yg8, 1);
    yg8 += __shfl_xor_sync(0xFFFFFFFFu, yg8, 2);
    if (t == 0) {
      if (base + g < n) io.store(base + g, denormalise(sF, sF[FW_B3] + yg));
      if (base + g + 8 < n) io.store(base + g + 8, denormalise(sF, sF[FW_B3] + yg8));
    }
    __syncwarp();
  }
}

// Check path 2: one thread per sample, FP32 CUDA-core arithmetic on the same BF16 operands.
template <class IO>
__global__ void __launch_bounds__(128) k_mlp_fp32(Infer w, IO io, uint32_t n) {
  __shared__ float sF[NFW];
  __shared__ float sW2[NH * NH];
  for (uint32_t i = threadIdx.x; i < (uint32_t)NFW; i += blockDim.x) sF[i] = w.fw[i];
  for (uint32_t i = threadIdx.x; i < (uint32_t)(NH * NH / 2); i += blockDim.x) {
    const uint32_t v = w.w2_rm[i];
    sW2[2 * i] = __bfloat162float(__ushort_as_bfloat16((unsigned short)(v & 0xFFFFu)));
    sW2[2 * i + 1] = __bfloat162float(__ushort_as_bfloat16((unsigned short)(v >> 16)));
  }
  __syncthreads();
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    float x[NIN];
    io.features(i, x);
    normalise(sF, x);
    float h[NH];
#pragma unroll
    for (int k = 0; k < NH; ++k) h[k] = bf16_round(hidden1(sF, x, k));
    float y = sF[FW_B3];
    for (int j = 0; j < NH; ++j) {
      float a = 0.0f;
#pragma unroll
      for (int k = 0; k < NH; ++k) a += sW2[j * NH + k] * h[k];
      y += sF[FW_W3 + j] * gelu(a + sF[FW_B2 + j]);
    }
    io.store(i, denormalise(sF, y));
  }
}

// raw features -> output (the IO of the feature-array entry points)
struct ArrayIO {
  const float* feats;  // [n][NIN]
  float* out;
  __device__ __forceinline__ void features(uint32_t i, float x[NIN]) const {
#pragma unroll
    for (int q = 0; q < NIN; ++q) x[q] = feats[(size_t)i * NIN + q];
  }
  __device__ __forceinline__ void store(uint32_t i, float t) const { out[i] = t; }
  __device__ __forceinline__ uint32_t rows(uint32_t n) const { return n; }
};

}  // namespace mlp
}  // namespace cleo

// library-internal accessor of a model's inference view (defined in mlp.cu)
struct cleo_b200_mlp;
int cleo_mlp_infer_view(const cleo_b200_mlp* m, cleo::mlp::Infer* out);
