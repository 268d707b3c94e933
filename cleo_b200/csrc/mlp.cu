// mlp.cu — training and inference entry points of the condensation surrogate (see mlp.cuh).
//
// Training runs on the GPU with this file's own kernels: a forward/backward kernel computes the
// gradient of the mean squared error of the standardised target over a minibatch (FP32,
// deterministic: each CTA reduces its 128 samples in a fixed order into its own partial row, and
// the Adam kernel sums the rows in block order), and an Adam kernel updates the FP32 master
// weights. After every change of the weights a packing kernel writes the BF16 inference copies.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "../../include/cleo_b200.h"
#include "mlp.cuh"

using namespace cleo;
using namespace cleo::mlp;

struct cleo_b200_mlp {
  int device = 0;
  cudaStream_t stream = nullptr;
  float* params = nullptr;  // NPARAM FP32 master weights
  float* adam_m = nullptr;
  float* adam_v = nullptr;
  float* norm = nullptr;  // NNORM
  float* fw = nullptr;    // NFW inference constants
  uint4* w2_umma = nullptr;
  uint32_t* w2_rm = nullptr;
  uint32_t* err = nullptr;
  DevError* phys_err = nullptr;
  float* partial = nullptr;  // [cap_blocks][NPARAM]
  float* loss_partial = nullptr;
  double* stats = nullptr;  // [cap_stat_blocks][32]
  uint32_t cap_blocks = 0, cap_stat_blocks = 0;
  uint64_t adam_t = 0;
};

namespace {

#define MLP_TRY(x)                                                                     \
  do {                                                                                 \
    cudaError_t e_ = (x);                                                              \
    if (e_ != cudaSuccess) {                                                           \
      fprintf(stderr, "cleo_b200 mlp: %s failed: %s\n", #x, cudaGetErrorString(e_)); \
      return CLEO_ERR_CUDA;                                                            \
    }                                                                                  \
  } while (0)

constexpr int TR_LD = 65;  // padded row of the per-sample activations
constexpr size_t TR_SMEM =
    (size_t)(NPARAM + 4 * 128 * TR_LD + 128 * 8 + 2 * 128) * sizeof(float);  // 157188 B

// ---- features, standardisation targets and the Newton branch of each droplet ----
__global__ void k_mlp_features(uint32_t n, const double* __restrict__ radius,
                               const double* __restrict__ msol, const double* __restrict__ temp,
                               const double* __restrict__ press,
                               const double* __restrict__ s_ratio,
                               const double* __restrict__ delt,
                               const double* __restrict__ radius_new, float* __restrict__ feats,
                               float* __restrict__ target, uint8_t* __restrict__ direct,
                               DevError* err) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    float x[NIN];
    raw_features(radius[i], msol[i], temp[i], press[i], s_ratio[i], delt[i], x);
#pragma unroll
    for (int q = 0; q < NIN; ++q) feats[(size_t)i * NIN + q] = x[q];
    if (target) target[i] = (float)(2.0 * log(radius_new[i] / radius[i]));
    if (direct) {
      // the branch of solve_condensation (impliciteuler.cpp:35-54) that a seed applies to
      const Where w{err, OOB, i};
      const double T = temp[i];
      const double psat = saturation_pressure(T, w);
      const double ffactor = diffusion_factor(press[i], T, psat);
      double akoh, bkoh;
      kohler_factors(msol[i], T, akoh, bkoh);
      const OdeConsts o{s_ratio[i], akoh, bkoh, ffactor / ventilation_factor(radius[i])};
      const double z0 = initialguess(o, radius[i]);
      direct[i] = (first_unique_criteria(o, radius[i], z0) || delt[i] <= critical_timestep(o))
                      ? 1
                      : 0;
    }
  }
}

// per-block sums and sums of squares of the 7 features and the target (FP64)
__global__ void k_mlp_stats(uint32_t n, const float* __restrict__ feats,
                            const float* __restrict__ target, double* __restrict__ out) {
  __shared__ double red[256];
  double s[8], q[8];
#pragma unroll
  for (int c = 0; c < 8; ++c) s[c] = q[c] = 0.0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      const double v = c < NIN ? (double)feats[(size_t)i * NIN + c] : (double)target[i];
      s[c] += v;
      q[c] += v * v;
    }
  }
  for (int c = 0; c < 16; ++c) {
    red[threadIdx.x] = c < 8 ? s[c] : q[c - 8];
    __syncthreads();
    for (int h = 128; h > 0; h >>= 1) {
      if ((int)threadIdx.x < h) red[threadIdx.x] += red[threadIdx.x + h];
      __syncthreads();
    }
    if (threadIdx.x == 0) out[blockIdx.x * 32 + c] = red[0];
    __syncthreads();
  }
}

// ---- forward + backward over 128 samples per CTA ----
// Loss L = inv_count * sum_s (y_s - t_s)^2 over the standardised target t. random != 0 draws
// the samples uniformly (with replacement) from [0, n) by the counter generator keyed by
// (seed, step); otherwise sample = slot.
__global__ void __launch_bounds__(128)
k_mlp_fwdbwd(const float* __restrict__ params, const float* __restrict__ norm,
             const float* __restrict__ feats, const float* __restrict__ target, uint32_t n,
             uint32_t count, uint64_t seed, uint32_t step, int random,
             float* __restrict__ partial, float* __restrict__ loss_partial, float inv_count) {
  extern __shared__ float sm[];
  float* W = sm;
  float* H1 = W + NPARAM;        // hidden 1 after GELU
  float* D2 = H1 + 128 * TR_LD;  // GELU'(a2), then dL/da2
  float* D1 = D2 + 128 * TR_LD;  // GELU'(a1), then dL/da1
  float* H2 = D1 + 128 * TR_LD;  // hidden 2 after GELU
  float* X = H2 + 128 * TR_LD;   // standardised features, row of 8
  float* DY = X + 128 * 8;       // dL/dy
  float* LS = DY + 128;          // per-sample loss
  const uint32_t tid = threadIdx.x;
  for (uint32_t i = tid; i < (uint32_t)NPARAM; i += 128) W[i] = params[i];
  __syncthreads();

  const uint32_t slot = blockIdx.x * 128 + tid;
  const bool valid = slot < count;
  uint32_t j = slot;
  if (random)
    j = (uint32_t)cleo_rng_mulhi(cleo_rng_u64(cleo_rng_key(seed, step, 0x4D4C50u), slot), n);
  float x[NIN];
  float t = 0.0f;
#pragma unroll
  for (int q = 0; q < NIN; ++q)
    x[q] = valid ? (feats[(size_t)j * NIN + q] - norm[q]) * norm[NIN + q] : 0.0f;
  if (valid) t = (target[j] - norm[14]) / norm[15];

  float h1[NH];
#pragma unroll
  for (int k = 0; k < NH; ++k) {
    float a = W[OFF_B1 + k];
#pragma unroll
    for (int i = 0; i < NIN; ++i) a += W[OFF_W1 + k * NIN + i] * x[i];
    h1[k] = gelu(a);
    H1[tid * TR_LD + k] = h1[k];
    D1[tid * TR_LD + k] = gelu_grad(a);
  }
  float y = W[OFF_B3];
#pragma unroll 2
  for (int jj = 0; jj < NH; ++jj) {
    float a = W[OFF_B2 + jj];
#pragma unroll
    for (int k = 0; k < NH; ++k) a += W[OFF_W2 + jj * NH + k] * h1[k];
    const float h2 = gelu(a);
    H2[tid * TR_LD + jj] = h2;
    D2[tid * TR_LD + jj] = gelu_grad(a);
    y += W[OFF_W3 + jj] * h2;
  }
  const float d = valid ? (y - t) : 0.0f;
  LS[tid] = d * d * inv_count;
  const float dy = 2.0f * d * inv_count;
  DY[tid] = dy;
  float da2[NH];
#pragma unroll
  for (int jj = 0; jj < NH; ++jj) {
    da2[jj] = dy * W[OFF_W3 + jj] * D2[tid * TR_LD + jj];
    D2[tid * TR_LD + jj] = da2[jj];
  }
#pragma unroll 2
  for (int k = 0; k < NH; ++k) {
    float dh = 0.0f;
#pragma unroll
    for (int jj = 0; jj < NH; ++jj) dh += W[OFF_W2 + jj * NH + k] * da2[jj];
    D1[tid * TR_LD + k] *= dh;
  }
#pragma unroll
  for (int q = 0; q < NIN; ++q) X[tid * 8 + q] = x[q];
  __syncthreads();

  // parameter gradients, summed over the 128 samples in sample order
  float* out = partial + (size_t)blockIdx.x * NPARAM;
  {
    const int j0 = (int)(tid >> 3) * 4, k0 = (int)(tid & 7) * 8;
    float acc[4][8];
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
      for (int c = 0; c < 8; ++c) acc[r][c] = 0.0f;
    for (int s = 0; s < 128; ++s) {
      float a[4], b[8];
#pragma unroll
      for (int r = 0; r < 4; ++r) a[r] = D2[s * TR_LD + j0 + r];
#pragma unroll
      for (int c = 0; c < 8; ++c) b[c] = H1[s * TR_LD + k0 + c];
#pragma unroll
      for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int c = 0; c < 8; ++c) acc[r][c] += a[r] * b[c];
    }
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
      for (int c = 0; c < 8; ++c) out[OFF_W2 + (j0 + r) * NH + k0 + c] = acc[r][c];
  }
  if (tid < 64) {
    float gb = 0.0f, gw = 0.0f;
    for (int s = 0; s < 128; ++s) {
      gb += D2[s * TR_LD + tid];
      gw += DY[s] * H2[s * TR_LD + tid];
    }
    out[OFF_B2 + tid] = gb;
    out[OFF_W3 + tid] = gw;
  } else {
    const int k = (int)tid - 64;
    float gb = 0.0f;
    for (int s = 0; s < 128; ++s) gb += D1[s * TR_LD + k];
    out[OFF_B1 + k] = gb;
  }
  for (uint32_t e = tid; e < (uint32_t)(NH * NIN); e += 128) {
    const int k = (int)e / NIN, i = (int)e % NIN;
    float g = 0.0f;
    for (int s = 0; s < 128; ++s) g += D1[s * TR_LD + k] * X[s * 8 + i];
    out[OFF_W1 + e] = g;
  }
  if (tid == 0) {
    float gb = 0.0f, l = 0.0f;
    for (int s = 0; s < 128; ++s) {
      gb += DY[s];
      l += LS[s];
    }
    out[OFF_B3] = gb;
    loss_partial[blockIdx.x] = l;
  }
}

// sum of the partial rows (block order), then an optional Adam update
__global__ void k_mlp_adam(float* __restrict__ params, float* __restrict__ m,
                           float* __restrict__ v, const float* __restrict__ partial,
                           uint32_t nblk, float lr_eff, float eps_eff, float beta1, float beta2,
                           int apply, float* __restrict__ grad_out,
                           const float* __restrict__ loss_partial, float* __restrict__ loss_out) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0 && loss_out) {
    float l = 0.0f;
    for (uint32_t b = 0; b < nblk; ++b) l += loss_partial[b];
    *loss_out = l;
  }
  if (i >= (uint32_t)NPARAM) return;
  float g = 0.0f;
  for (uint32_t b = 0; b < nblk; ++b) g += partial[(size_t)b * NPARAM + i];
  if (grad_out) grad_out[i] = g;
  if (!apply) return;
  const float mi = beta1 * m[i] + (1.0f - beta1) * g;
  const float vi = beta2 * v[i] + (1.0f - beta2) * g * g;
  m[i] = mi;
  v[i] = vi;
  params[i] -= lr_eff * mi / (sqrtf(vi) + eps_eff);
}

// BF16 inference copies of the master weights
__global__ void k_mlp_pack(const float* __restrict__ params, const float* __restrict__ norm,
                           float* __restrict__ fw, uint16_t* __restrict__ w2_umma,
                           uint32_t* __restrict__ w2_rm) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < (uint32_t)(NH * NH)) {
    const uint32_t nn = i / NH, k = i % NH;
    const uint16_t b = __bfloat16_as_ushort(__float2bfloat16_rn(params[OFF_W2 + i]));
    w2_umma[((k / 8) * 8 + nn / 8) * 64 + (nn % 8) * 8 + (k % 8)] = b;
    if ((k & 1) == 0)
      w2_rm[nn * 32 + k / 2] = pack_bf16x2(params[OFF_W2 + i], params[OFF_W2 + i + 1]);
  }
  if (i < (uint32_t)(NH * NIN)) fw[FW_W1 + i] = bf16_round(params[OFF_W1 + i]);
  if (i < (uint32_t)NH) {
    fw[FW_B1 + i] = params[OFF_B1 + i];
    fw[FW_B2 + i] = params[OFF_B2 + i];
    fw[FW_W3 + i] = bf16_round(params[OFF_W3 + i]);
  }
  if (i == 0) fw[FW_B3] = params[OFF_B3];
  if (i < (uint32_t)NNORM) fw[FW_NORM + i] = norm[i];
}

int pack(cleo_b200_mlp* m) {
  k_mlp_pack<<<(NH * NH + 255) / 256, 256, 0, m->stream>>>(
      m->params, m->norm, m->fw, reinterpret_cast<uint16_t*>(m->w2_umma), m->w2_rm);
  MLP_TRY(cudaGetLastError());
  return CLEO_OK;
}

int ensure_blocks(cleo_b200_mlp* m, uint32_t nblk) {
  if (nblk <= m->cap_blocks) return CLEO_OK;
  MLP_TRY(cudaStreamSynchronize(m->stream));
  cudaFree(m->partial);
  cudaFree(m->loss_partial);
  m->partial = nullptr;
  m->loss_partial = nullptr;
  m->cap_blocks = 0;
  MLP_TRY(cudaMalloc(&m->partial, (size_t)nblk * NPARAM * sizeof(float)));
  MLP_TRY(cudaMalloc(&m->loss_partial, (size_t)nblk * sizeof(float)));
  m->cap_blocks = nblk;
  return CLEO_OK;
}

int set_fwdbwd_smem() {  // the attribute is per function and device: set before each use
  MLP_TRY(cudaFuncSetAttribute(k_mlp_fwdbwd, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)TR_SMEM));
  return CLEO_OK;
}

uint64_t splitmix(uint64_t& s) {
  uint64_t z = (s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

bool bad_mlp(const cleo_b200_mlp* m) { return m == nullptr || m->params == nullptr; }

}  // namespace

int cleo_mlp_infer_view(const cleo_b200_mlp* m, Infer* out) {
  if (bad_mlp(m) || !out) return CLEO_ERR_ARGUMENT;
  out->fw = m->fw;
  out->w2_umma = m->w2_umma;
  out->w2_rm = m->w2_rm;
  out->err = m->err;
  return CLEO_OK;
}

extern "C" {

int cleo_b200_mlp_create(void* stream, uint64_t seed, cleo_b200_mlp** out) {
  if (!out) return CLEO_ERR_ARGUMENT;
  *out = nullptr;
  cleo_b200_mlp* m = new cleo_b200_mlp();
  MLP_TRY(cudaGetDevice(&m->device));
  m->stream = static_cast<cudaStream_t>(stream);
  int rc = CLEO_OK;
  auto al = [&](void** p, size_t bytes) {
    if (rc == CLEO_OK && cudaMalloc(p, bytes) != cudaSuccess) rc = CLEO_ERR_CUDA;
  };
  al((void**)&m->params, NPARAM * sizeof(float));
  al((void**)&m->adam_m, NPARAM * sizeof(float));
  al((void**)&m->adam_v, NPARAM * sizeof(float));
  al((void**)&m->norm, NNORM * sizeof(float));
  al((void**)&m->fw, NFW * sizeof(float));
  al((void**)&m->w2_umma, W2_UMMA_BYTES);
  al((void**)&m->w2_rm, NH * NH / 2 * sizeof(uint32_t));
  al((void**)&m->err, sizeof(uint32_t));
  al((void**)&m->phys_err, sizeof(DevError));
  if (rc != CLEO_OK) {
    cleo_b200_mlp_destroy(m);
    return rc;
  }
  // Glorot-uniform weights, zero biases, identity standardisation
  std::vector<float> p(NPARAM, 0.0f);
  uint64_t st = seed ^ 0x6D6C702D696E6974ull;
  auto uni = [&](float a) {
    const double u = (double)(splitmix(st) >> 11) * (1.0 / 9007199254740992.0);
    return (float)((2.0 * u - 1.0) * a);
  };
  const float a1 = std::sqrt(6.0f / (NIN + NH)), a2 = std::sqrt(6.0f / (NH + NH)),
              a3 = std::sqrt(6.0f / (NH + 1));
  for (int i = 0; i < NH * NIN; ++i) p[OFF_W1 + i] = uni(a1);
  for (int i = 0; i < NH * NH; ++i) p[OFF_W2 + i] = uni(a2);
  for (int i = 0; i < NH; ++i) p[OFF_W3 + i] = uni(a3);
  float nrm[NNORM];
  for (int i = 0; i < NIN; ++i) {
    nrm[i] = 0.0f;
    nrm[NIN + i] = 1.0f;
  }
  nrm[14] = 0.0f;
  nrm[15] = 1.0f;
  rc = cleo_b200_mlp_set_params(m, p.data(), nrm);
  if (rc != CLEO_OK) {
    cleo_b200_mlp_destroy(m);
    return rc;
  }
  *out = m;
  return CLEO_OK;
}

int cleo_b200_mlp_destroy(cleo_b200_mlp* m) {
  if (!m) return CLEO_OK;
  if (m->stream) cudaStreamSynchronize(m->stream);
  cudaFree(m->params);
  cudaFree(m->adam_m);
  cudaFree(m->adam_v);
  cudaFree(m->norm);
  cudaFree(m->fw);
  cudaFree(m->w2_umma);
  cudaFree(m->w2_rm);
  cudaFree(m->err);
  cudaFree(m->phys_err);
  cudaFree(m->partial);
  cudaFree(m->loss_partial);
  cudaFree(m->stats);
  delete m;
  return CLEO_OK;
}

int cleo_b200_mlp_set_params(cleo_b200_mlp* m, const float* params, const float* norm) {
  if (bad_mlp(m) || !params || !norm) return CLEO_ERR_ARGUMENT;
  MLP_TRY(cudaMemcpyAsync(m->params, params, NPARAM * sizeof(float), cudaMemcpyHostToDevice,
                          m->stream));
  MLP_TRY(cudaMemcpyAsync(m->norm, norm, NNORM * sizeof(float), cudaMemcpyHostToDevice,
                          m->stream));
  MLP_TRY(cudaMemsetAsync(m->adam_m, 0, NPARAM * sizeof(float), m->stream));
  MLP_TRY(cudaMemsetAsync(m->adam_v, 0, NPARAM * sizeof(float), m->stream));
  MLP_TRY(cudaMemsetAsync(m->err, 0, sizeof(uint32_t), m->stream));
  MLP_TRY(cudaMemsetAsync(m->phys_err, 0, sizeof(DevError), m->stream));
  m->adam_t = 0;
  const int rc = pack(m);
  if (rc != CLEO_OK) return rc;
  MLP_TRY(cudaStreamSynchronize(m->stream));
  return CLEO_OK;
}

int cleo_b200_mlp_get_params(cleo_b200_mlp* m, float* params, float* norm) {
  if (bad_mlp(m)) return CLEO_ERR_ARGUMENT;
  if (params)
    MLP_TRY(cudaMemcpyAsync(params, m->params, NPARAM * sizeof(float), cudaMemcpyDeviceToHost,
                            m->stream));
  if (norm)
    MLP_TRY(cudaMemcpyAsync(norm, m->norm, NNORM * sizeof(float), cudaMemcpyDeviceToHost,
                            m->stream));
  MLP_TRY(cudaStreamSynchronize(m->stream));
  return CLEO_OK;
}

int cleo_b200_mlp_features(cleo_b200_mlp* m, size_t n, const double* d_radius,
                           const double* d_msol, const double* d_temp, const double* d_press,
                           const double* d_s_ratio, const double* d_delt,
                           const double* d_radius_new, float* d_features, float* d_target,
                           uint8_t* d_direct) {
  if (bad_mlp(m) || n > 0xFFFFFFFFull) return CLEO_ERR_ARGUMENT;
  if (n == 0) return CLEO_OK;
  if (!d_radius || !d_msol || !d_temp || !d_press || !d_s_ratio || !d_delt || !d_features ||
      (d_target && !d_radius_new))
    return CLEO_ERR_ARGUMENT;
  const uint32_t nb = (uint32_t)std::min<size_t>((n + 255) / 256, 148 * 16);
  k_mlp_features<<<nb, 256, 0, m->stream>>>((uint32_t)n, d_radius, d_msol, d_temp, d_press,
                                            d_s_ratio, d_delt, d_radius_new, d_features,
                                            d_target, d_direct, m->phys_err);
  MLP_TRY(cudaGetLastError());
  DevError e{};
  MLP_TRY(cudaMemcpyAsync(&e, m->phys_err, sizeof(e), cudaMemcpyDeviceToHost, m->stream));
  MLP_TRY(cudaStreamSynchronize(m->stream));
  return e.code != 0 ? e.code : CLEO_OK;
}

int cleo_b200_mlp_fit_normalisation(cleo_b200_mlp* m, size_t n, const float* d_features,
                                    const float* d_target) {
  if (bad_mlp(m) || n == 0 || n > 0xFFFFFFFFull || !d_features || !d_target)
    return CLEO_ERR_ARGUMENT;
  const uint32_t nb = (uint32_t)std::min<size_t>((n + 255) / 256, 148 * 4);
  if (nb > m->cap_stat_blocks) {
    MLP_TRY(cudaStreamSynchronize(m->stream));
    cudaFree(m->stats);
    m->stats = nullptr;
    m->cap_stat_blocks = 0;
    MLP_TRY(cudaMalloc(&m->stats, (size_t)nb * 32 * sizeof(double)));
    m->cap_stat_blocks = nb;
  }
  k_mlp_stats<<<nb, 256, 0, m->stream>>>((uint32_t)n, d_features, d_target, m->stats);
  MLP_TRY(cudaGetLastError());
  std::vector<double> h((size_t)nb * 32);
  MLP_TRY(cudaMemcpyAsync(h.data(), m->stats, h.size() * sizeof(double), cudaMemcpyDeviceToHost,
                          m->stream));
  MLP_TRY(cudaStreamSynchronize(m->stream));
  double s[8] = {0}, q[8] = {0};
  for (uint32_t b = 0; b < nb; ++b)
    for (int c = 0; c < 8; ++c) {
      s[c] += h[b * 32 + c];
      q[c] += h[b * 32 + 8 + c];
    }
  float nrm[NNORM];
  for (int c = 0; c < 8; ++c) {
    const double mean = s[c] / (double)n;
    double var = q[c] / (double)n - mean * mean;
    if (!(var > 1e-24)) var = 1.0;  // a constant input carries no information: leave unscaled
    const double sd = std::sqrt(var);
    if (c < NIN) {
      nrm[c] = (float)mean;
      nrm[NIN + c] = (float)(1.0 / sd);
    } else {
      nrm[14] = (float)mean;
      nrm[15] = (float)sd;
    }
  }
  MLP_TRY(cudaMemcpyAsync(m->norm, nrm, sizeof(nrm), cudaMemcpyHostToDevice, m->stream));
  const int rc = pack(m);
  if (rc != CLEO_OK) return rc;
  MLP_TRY(cudaStreamSynchronize(m->stream));
  return CLEO_OK;
}

int cleo_b200_mlp_loss_grad(cleo_b200_mlp* m, size_t n, const float* d_features,
                            const float* d_target, float* d_grad, float* d_loss) {
  if (bad_mlp(m) || n == 0 || n > (1u << 24) || !d_features || !d_target || !d_grad)
    return CLEO_ERR_ARGUMENT;
  const uint32_t nb = (uint32_t)((n + 127) / 128);
  int rc = ensure_blocks(m, nb);
  if (rc != CLEO_OK) return rc;
  rc = set_fwdbwd_smem();
  if (rc != CLEO_OK) return rc;
  k_mlp_fwdbwd<<<nb, 128, TR_SMEM, m->stream>>>(m->params, m->norm, d_features, d_target,
                                                (uint32_t)n, (uint32_t)n, 0, 0, 0, m->partial,
                                                m->loss_partial, 1.0f / (float)n);
  MLP_TRY(cudaGetLastError());
  k_mlp_adam<<<(NPARAM + 255) / 256, 256, 0, m->stream>>>(m->params, m->adam_m, m->adam_v,
                                                          m->partial, nb, 0.f, 0.f, 0.f, 0.f, 0,
                                                          d_grad, m->loss_partial, d_loss);
  MLP_TRY(cudaGetLastError());
  MLP_TRY(cudaStreamSynchronize(m->stream));
  return CLEO_OK;
}

int cleo_b200_mlp_train(cleo_b200_mlp* m, size_t n, const float* d_features,
                        const float* d_target, uint32_t steps, uint32_t batch, float lr,
                        uint64_t seed, float* d_loss_per_step) {
  if (bad_mlp(m) || n == 0 || n > 0xFFFFFFFFull || !d_features || !d_target || batch == 0 ||
      batch % 128 != 0 || batch > (1u << 20) || !(lr > 0.0f))
    return CLEO_ERR_ARGUMENT;
  const uint32_t nb = batch / 128;
  int rc = ensure_blocks(m, nb);
  if (rc != CLEO_OK) return rc;
  rc = set_fwdbwd_smem();
  if (rc != CLEO_OK) return rc;
  const double beta1 = 0.9, beta2 = 0.999, eps = 1e-8;
  const uint32_t warm = steps / 50 + 1;
  for (uint32_t s = 0; s < steps; ++s) {
    // linear warm-up, then cosine decay to 2% of lr
    double f = 0.02 + 0.98 * 0.5 * (1.0 + std::cos(3.141592653589793 * (double)s / (double)steps));
    if (s < warm) f *= (double)(s + 1) / (double)warm;
    const uint64_t t = ++m->adam_t;
    const double bc1 = 1.0 - std::pow(beta1, (double)t), bc2 = 1.0 - std::pow(beta2, (double)t);
    const float lr_eff = (float)(lr * f * std::sqrt(bc2) / bc1);
    const float eps_eff = (float)(eps * std::sqrt(bc2));
    k_mlp_fwdbwd<<<nb, 128, TR_SMEM, m->stream>>>(m->params, m->norm, d_features, d_target,
                                                  (uint32_t)n, batch, seed, s, 1, m->partial,
                                                  m->loss_partial, 1.0f / (float)batch);
    k_mlp_adam<<<(NPARAM + 255) / 256, 256, 0, m->stream>>>(
        m->params, m->adam_m, m->adam_v, m->partial, nb, lr_eff, eps_eff, (float)beta1,
        (float)beta2, 1, nullptr, m->loss_partial,
        d_loss_per_step ? d_loss_per_step + s : nullptr);
  }
  MLP_TRY(cudaGetLastError());
  rc = pack(m);
  if (rc != CLEO_OK) return rc;
  MLP_TRY(cudaStreamSynchronize(m->stream));
  return CLEO_OK;
}

int cleo_b200_mlp_infer(cleo_b200_mlp* m, size_t n, const float* d_features, float* d_out,
                        int path) {
  if (bad_mlp(m) || n > 0xFFFFFFFFull || !d_features || !d_out) return CLEO_ERR_ARGUMENT;
  if (n == 0) return CLEO_OK;
  Infer w;
  cleo_mlp_infer_view(m, &w);
  const ArrayIO io{d_features, d_out};
  const uint32_t nn = (uint32_t)n;
  if (path == CLEO_MLP_TCGEN05) {
    const uint32_t tiles = (nn + TILE_M - 1) / TILE_M;
    const uint32_t grid = tiles < TC_GRID_MAX ? tiles : TC_GRID_MAX;
    k_mlp_tc<ArrayIO><<<grid, 128, TC_SMEM, m->stream>>>(w, io, nn);
  } else if (path == CLEO_MLP_MMA_SYNC) {
    const uint32_t tiles = (nn + 15) / 16;
    uint32_t grid = (tiles + MMA_WARPS - 1) / MMA_WARPS;
    if (grid > 148u * 8u) grid = 148u * 8u;
    k_mlp_mma<ArrayIO><<<grid, 128, 0, m->stream>>>(w, io, nn);
  } else if (path == CLEO_MLP_FP32) {
    uint32_t grid = (nn + 127) / 128;
    if (grid > 148u * 8u) grid = 148u * 8u;
    k_mlp_fp32<ArrayIO><<<grid, 128, 0, m->stream>>>(w, io, nn);
  } else {
    return CLEO_ERR_ARGUMENT;
  }
  MLP_TRY(cudaGetLastError());
  uint32_t e = 0;
  MLP_TRY(cudaMemcpyAsync(&e, m->err, sizeof(e), cudaMemcpyDeviceToHost, m->stream));
  MLP_TRY(cudaStreamSynchronize(m->stream));
  return e != 0 ? (int)e : CLEO_OK;
}

}  // extern "C"
