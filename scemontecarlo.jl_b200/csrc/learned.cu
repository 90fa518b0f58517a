// Learned proposal network: the per-site MLP (43 -> 128 -> 128 -> 20, SiLU, BF16
// weights, FP32 accumulate) with its forward, backward and Adam kernels. Every
// matrix product runs on the tcgen05 tensor cores through one GEMM kernel
// (C = A B^T, both operands K-major BF16 staged in shared memory, FP32 accumulator
// in TMEM) whose epilogue fuses the bias, SiLU, SiLU' and the transposed copies the
// backward pass reads. The head (vMF mixture negative log-likelihood and its
// gradient) and the optimiser are plain FP64/FP32 kernels.
//
// The reference has no learned proposal; the C entry points follow the library's
// conventions (int32_t status, scemc_last_error, host buffers).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <numeric>
#include <random>
#include <string>
#include <vector>

#include "mlp.h"
#include "scemc.h"
#include "umma.cuh"
#include "vmf.cuh"

using bf16 = __nv_bfloat16;
using namespace mlpl;

namespace {

int32_t fail(int32_t code, const std::string& m) { return scemc_detail::set_error(code, m.c_str()); }

#define LTRY(x)                                                                      \
  do {                                                                               \
    cudaError_t e_ = (x);                                                            \
    if (e_ != cudaSuccess)                                                           \
      return fail(SCEMC_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_)); \
  } while (0)

constexpr long long kWaitLimitNs = 1000000000ll;  // 1 s for any tensor-core completion

// ---------------------------------------------------------------------------
// GEMM C[M][N] = A[M][K] . B[N][K]^T, one CTA (one warpgroup) per 128-row tile.
// ---------------------------------------------------------------------------
enum GemmMode : int {
  G_STORE = 0,      // C fp32 [M][N]
  G_BIAS_SILU = 1,  // z = acc + bias: C = z (fp32), H = silu(z), HT = H^T (BF16; null skips)
  G_BIAS = 2,       // C = acc + bias (fp32)
  G_DSILU = 3,      // dz = acc * silu'(Zin): H = dz, HT = dz^T (BF16; null skips)
};

struct GemmArgs {
  const bf16* A;
  int64_t lda;
  const bf16* B;
  int64_t ldb;
  int64_t M;
  int N, K;
  int mode;
  float* C;
  int64_t ldc;
  const float* bias;
  bf16* H;
  int64_t ldh;
  bf16* HT;
  int64_t ldht;
  const float* Zin;
  int64_t ldz;
  int* err;
};

constexpr int kKC = 64;  // K columns staged per chunk

// the sweep's fused kernel uses the same form (fast division; 0 for z below about -87)
__device__ __forceinline__ float silu_f(float z) { return __fdividef(z, 1.0f + __expf(-z)); }
__device__ __forceinline__ float dsilu_f(float z) {
  const float s = 1.0f / (1.0f + __expf(-z));
  return s * (1.0f + z * (1.0f - s));
}

__global__ void __launch_bounds__(128) k_umma_gemm(GemmArgs g) {
  __shared__ __align__(1024) uint8_t sA[128 * kKC * 2];
  __shared__ __align__(1024) uint8_t sB[128 * kKC * 2];
  __shared__ __align__(8) uint64_t mbar;
  __shared__ uint32_t tslot;
  const int tid = threadIdx.x, warp = tid >> 5;
  const int64_t m0 = (int64_t)blockIdx.x * 128;
  const int ncols = g.N < 32 ? 32 : g.N;
  if (warp == 0) umma::tmem_alloc(&tslot, (uint32_t)ncols);
  if (tid == 0) umma::mbar_init(&mbar, 1);
  umma::fence_before();
  __syncthreads();
  umma::fence_after();
  const uint32_t tmem = tslot;
  const int kc = g.K < kKC ? g.K : kKC;
  const uint32_t idesc = umma::idesc_bf16_f32(g.N);
  bool ok = true;
  uint32_t phase = 0;
  for (int k0 = 0; k0 < g.K && ok; k0 += kc) {
    // stage the A and B chunks (16-byte pieces) in the K-major canonical layout
    const int pr = kc >> 3;
    for (int p = tid; p < 128 * pr; p += 128) {
      const int row = p / pr, kg = p - row * pr;
      const uint4 v = *reinterpret_cast<const uint4*>(g.A + (m0 + row) * g.lda + k0 + kg * 8);
      *reinterpret_cast<uint4*>(sA + umma::kmajor_offset(row, kg * 8, kc)) = v;
    }
    for (int p = tid; p < g.N * pr; p += 128) {
      const int row = p / pr, kg = p - row * pr;
      const uint4 v = *reinterpret_cast<const uint4*>(g.B + (int64_t)row * g.ldb + k0 + kg * 8);
      *reinterpret_cast<uint4*>(sB + umma::kmajor_offset(row, kg * 8, kc)) = v;
    }
    umma::fence_async_smem();
    __syncthreads();
    if (tid == 0) {
      umma::fence_after();
      const uint32_t a0 = umma::smem_u32(sA), b0 = umma::smem_u32(sB);
      const uint32_t sbo = (uint32_t)(kc / 8) * 128u;
      for (int kk = 0; kk < kc / 16; ++kk) {
        const uint64_t ad = umma::smem_desc(a0 + kk * 256u, 128u, sbo);
        const uint64_t bd = umma::smem_desc(b0 + kk * 256u, 128u, sbo);
        umma::mma_bf16(tmem, ad, bd, idesc, (k0 > 0 || kk > 0) ? 1u : 0u);
      }
      umma::commit(&mbar);
    }
    ok = umma::mbar_wait(&mbar, phase, kWaitLimitNs);
    phase ^= 1u;
    umma::fence_after();
  }
  if (!ok) {
    if (g.err) atomicExch(g.err, 1);
  } else {
    // epilogue: thread tid owns row m0 + tid (TMEM lane tid)
    const int64_t m = m0 + tid;
    const uint32_t lane_base = (uint32_t)(warp * 32) << 16;
    for (int c0 = 0; c0 < g.N; c0 += 8) {
      float v[8];
      umma::tmem_ld8(tmem + lane_base + (uint32_t)c0, v);
      if (m >= g.M) continue;
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const int n = c0 + i;
        float x = v[i];
        if (g.mode == G_STORE) {
          g.C[m * g.ldc + n] = x;
        } else if (g.mode == G_BIAS) {
          g.C[m * g.ldc + n] = x + g.bias[n];
        } else if (g.mode == G_BIAS_SILU) {
          x += g.bias[n];
          if (g.C) g.C[m * g.ldc + n] = x;
          const bf16 h = __float2bfloat16_rn(silu_f(x));
          if (g.H) g.H[m * g.ldh + n] = h;
          if (g.HT) g.HT[(int64_t)n * g.ldht + m] = h;
        } else {  // G_DSILU
          const bf16 h = __float2bfloat16_rn(x * dsilu_f(g.Zin[m * g.ldz + n]));
          if (g.H) g.H[m * g.ldh + n] = h;
          if (g.HT) g.HT[(int64_t)n * g.ldht + m] = h;
        }
      }
    }
  }
  umma::fence_before();
  __syncthreads();
  if (warp == 0) {
    umma::fence_after();
    umma::tmem_free(tmem, (uint32_t)ncols);
  }
}

int32_t gemm(const GemmArgs& g, cudaStream_t st) {
  if (g.M % 128 || (g.N != 32 && g.N != 64 && g.N != 128) || g.K % 16 || (g.K > kKC && g.K % kKC))
    return fail(SCEMC_ERR_ARG, "gemm shape");
  k_umma_gemm<<<(unsigned)(g.M / 128), 128, 0, st>>>(g);
  LTRY(cudaGetLastError());
  return SCEMC_OK;
}

// ---------------------------------------------------------------------------
// small kernels
// ---------------------------------------------------------------------------
// BF16 copies of the masters (and the transposed W2, W3 the backward pass reads)
__global__ void k_to_bf16(const float* P, bf16* W1, bf16* W2, bf16* W2T, bf16* W3, bf16* W3T) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kHid * kHid; i += gridDim.x * blockDim.x) {
    const int r = i / kHid, c = i % kHid;
    const bf16 w2 = __float2bfloat16_rn(P[oW2 + i]);
    W2[i] = w2;
    W2T[c * kHid + r] = w2;
    if (i < kHid * kInPad) W1[i] = __float2bfloat16_rn(P[oW1 + i]);
    if (i < kOutPad * kHid) {
      const int o = i / kHid, h = i % kHid;
      const bf16 w3 = __float2bfloat16_rn(P[oW3 + i]);
      W3[i] = w3;
      W3T[h * kOutPad + o] = w3;
    }
  }
}

// rows of X (n x n_in FP32, host layout; kT last) -> BF16 X [M][64] and X^T [64][M], tau, Y
__global__ void k_rows_in(const float* Xs, const float* Ys, const int32_t* idx, int64_t n_rows, int64_t M, bf16* X,
                          bf16* XT, float* tau, float* Y, int n_in) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < M * kInPad;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t b = i / kInPad;
    const int c = (int)(i % kInPad);
    float v = 0.0f;
    if (b < n_rows && c < n_in) {
      const int64_t src = idx ? idx[b] : b;
      v = Xs[src * n_in + c];
      if (c == n_in - 1) tau[b] = v;
      if (c < 3 && Ys) Y[b * 3 + c] = Ys[src * 3 + c];
    }
    const bf16 h = __float2bfloat16_rn(v);
    X[b * kInPad + c] = h;
    if (XT) XT[(int64_t)c * M + b] = h;
  }
}

// per row: loss and dO (scaled by 1/n), BF16 [M][32] and transposed [32][M]
__global__ void k_head_train(const float* O, const float* tau, const float* Y, int64_t n, int64_t M, bf16* dO,
                             bf16* dOT, double* loss) {
  for (int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; b < M; b += (int64_t)gridDim.x * blockDim.x) {
    float d[kOutPad];
    for (int j = 0; j < kOutPad; ++j) d[j] = 0.0f;
    double l = 0.0;
    if (b < n) {
      const double y[3] = {Y[b * 3], Y[b * 3 + 1], Y[b * 3 + 2]};
      l = vmf::nll_grad(O + b * kOutPad, (double)tau[b], y, 1.0 / (double)n, d);
    }
    loss[b] = l;
    for (int j = 0; j < kOutPad; ++j) {
      const bf16 h = __float2bfloat16_rn(d[j]);
      dO[b * kOutPad + j] = h;
      dOT[(int64_t)j * M + b] = h;
    }
  }
}

// gradient assembly (bias sums over the rows, padded entries zero) and, when lr > 0,
// one Adam step on the FP32 masters
__global__ void k_grad_adam(float* P, float* mom, float* var, float* grad, const float* dW1, const float* dW2,
                            const float* dW3T, const bf16* dZ1T, const bf16* dZ2T, const bf16* dOT, int64_t M,
                            float lr, float c1, float c2, int n_in) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < kParams; i += (int64_t)gridDim.x * blockDim.x) {
    float gv = 0.0f;
    if (i < oB1) {
      gv = ((i % kInPad) < n_in) ? dW1[i] : 0.0f;
    } else if (i < oW2) {
      const bf16* r = dZ1T + (i - oB1) * M;
      for (int64_t b = 0; b < M; ++b) gv += __bfloat162float(r[b]);
    } else if (i < oB2) {
      gv = dW2[i - oW2];
    } else if (i < oW3) {
      const bf16* r = dZ2T + (i - oB2) * M;
      for (int64_t b = 0; b < M; ++b) gv += __bfloat162float(r[b]);
    } else if (i < oB3) {
      const int64_t o = (i - oW3) / kHid, h = (i - oW3) % kHid;
      gv = o < kOut ? dW3T[h * kOutPad + o] : 0.0f;
    } else {
      const int64_t o = i - oB3;
      if (o < kOut) {
        const bf16* r = dOT + o * M;
        for (int64_t b = 0; b < M; ++b) gv += __bfloat162float(r[b]);
      }
    }
    grad[i] = gv;
    if (lr > 0.0f) {
      const float mm = 0.9f * mom[i] + 0.1f * gv;
      const float vv = 0.999f * var[i] + 0.001f * gv * gv;
      mom[i] = mm;
      var[i] = vv;
      P[i] -= lr * (mm / c1) / (sqrtf(vv / c2) + 1e-8f);
    }
  }
}

template <class T>
int32_t dal(T** p, size_t n) {
  LTRY(cudaMalloc(reinterpret_cast<void**>(p), std::max<size_t>(n, 1) * sizeof(T)));
  return SCEMC_OK;
}

void free_work(scemc_mlp* m) {
  void* ps[] = {m->d_X,   m->d_XT,  m->d_H1,  m->d_H1T, m->d_H2,  m->d_H2T, m->d_dO,   m->d_dOT,  m->d_dZ2,
                m->d_dZ2T, m->d_dZ1T, m->d_Z1,  m->d_Z2,  m->d_O,   m->d_tau, m->d_Y,    m->d_dW1,  m->d_dW2,
                m->d_dW3T, m->d_loss};
  for (void* p : ps)
    if (p) cudaFree(p);
  m->d_X = m->d_XT = m->d_H1 = m->d_H1T = m->d_H2 = m->d_H2T = m->d_dO = m->d_dOT = m->d_dZ2 = m->d_dZ2T =
      m->d_dZ1T = nullptr;
  m->d_Z1 = m->d_Z2 = m->d_O = m->d_tau = m->d_Y = m->d_dW1 = m->d_dW2 = m->d_dW3T = nullptr;
  m->d_loss = nullptr;
  m->cap = 0;
}

int32_t ensure_work(scemc_mlp* m, int64_t M) {
  if (m->cap >= M) return SCEMC_OK;
  free_work(m);
  int32_t rc;
  const size_t h = (size_t)M * kHid;
  if ((rc = dal(&m->d_X, (size_t)M * kInPad)) || (rc = dal(&m->d_XT, (size_t)M * kInPad)) ||
      (rc = dal(&m->d_H1, h)) || (rc = dal(&m->d_H1T, h)) || (rc = dal(&m->d_H2, h)) || (rc = dal(&m->d_H2T, h)) ||
      (rc = dal(&m->d_dO, (size_t)M * kOutPad)) || (rc = dal(&m->d_dOT, (size_t)M * kOutPad)) ||
      (rc = dal(&m->d_dZ2, h)) || (rc = dal(&m->d_dZ2T, h)) || (rc = dal(&m->d_dZ1T, h)) || (rc = dal(&m->d_Z1, h)) ||
      (rc = dal(&m->d_Z2, h)) || (rc = dal(&m->d_O, (size_t)M * kOutPad)) || (rc = dal(&m->d_tau, (size_t)M)) ||
      (rc = dal(&m->d_Y, (size_t)M * 3)) || (rc = dal(&m->d_dW1, (size_t)kHid * kInPad)) ||
      (rc = dal(&m->d_dW2, (size_t)kHid * kHid)) || (rc = dal(&m->d_dW3T, (size_t)kHid * kOutPad)) ||
      (rc = dal(&m->d_loss, (size_t)M)))
    return rc;
  m->cap = M;
  return SCEMC_OK;
}

int32_t refresh_bf16(scemc_mlp* m) {
  k_to_bf16<<<64, 256, 0, m->stream>>>(m->d_master, m->d_W1, m->d_W2, m->d_W2T, m->d_W3, m->d_W3T);
  LTRY(cudaGetLastError());
  return SCEMC_OK;
}

GemmArgs ga(const bf16* A, int64_t lda, const bf16* B, int64_t ldb, int64_t M, int N, int K, int mode, int* err) {
  GemmArgs g{};
  g.A = A, g.lda = lda, g.B = B, g.ldb = ldb, g.M = M, g.N = N, g.K = K, g.mode = mode, g.err = err;
  return g;
}

// forward + backward on rows already staged in m->d_X / d_XT / d_tau / d_Y (M rows,
// n valid); gradient into d_grad and, with lr > 0, one Adam step.
int32_t step_rows(scemc_mlp* m, int64_t n, int64_t M, float lr) {
  int32_t rc;
  cudaStream_t st = m->stream;
  GemmArgs g = ga(m->d_X, kInPad, m->d_W1, kInPad, M, kHid, kInPad, G_BIAS_SILU, m->d_err);
  g.C = m->d_Z1, g.ldc = kHid, g.bias = m->d_master + oB1, g.H = m->d_H1, g.ldh = kHid, g.HT = m->d_H1T, g.ldht = M;
  if ((rc = gemm(g, st))) return rc;
  g = ga(m->d_H1, kHid, m->d_W2, kHid, M, kHid, kHid, G_BIAS_SILU, m->d_err);
  g.C = m->d_Z2, g.ldc = kHid, g.bias = m->d_master + oB2, g.H = m->d_H2, g.ldh = kHid, g.HT = m->d_H2T, g.ldht = M;
  if ((rc = gemm(g, st))) return rc;
  g = ga(m->d_H2, kHid, m->d_W3, kHid, M, kOutPad, kHid, G_BIAS, m->d_err);
  g.C = m->d_O, g.ldc = kOutPad, g.bias = m->d_master + oB3;
  if ((rc = gemm(g, st))) return rc;
  k_head_train<<<(unsigned)((M + 127) / 128), 128, 0, st>>>(m->d_O, m->d_tau, m->d_Y, n, M, m->d_dO, m->d_dOT,
                                                             m->d_loss);
  LTRY(cudaGetLastError());
  // dZ2 = (dO W3) * silu'(Z2)
  g = ga(m->d_dO, kOutPad, m->d_W3T, kOutPad, M, kHid, kOutPad, G_DSILU, m->d_err);
  g.Zin = m->d_Z2, g.ldz = kHid, g.H = m->d_dZ2, g.ldh = kHid, g.HT = m->d_dZ2T, g.ldht = M;
  if ((rc = gemm(g, st))) return rc;
  // dZ1 = (dZ2 W2) * silu'(Z1), transposed only
  g = ga(m->d_dZ2, kHid, m->d_W2T, kHid, M, kHid, kHid, G_DSILU, m->d_err);
  g.Zin = m->d_Z1, g.ldz = kHid, g.HT = m->d_dZ1T, g.ldht = M;
  if ((rc = gemm(g, st))) return rc;
  // weight gradients over the M rows: dW3^T = H2^T dO, dW2 = dZ2^T H1, dW1 = dZ1^T X
  g = ga(m->d_H2T, M, m->d_dOT, M, kHid, kOutPad, (int)M, G_STORE, m->d_err);
  g.C = m->d_dW3T, g.ldc = kOutPad;
  if ((rc = gemm(g, st))) return rc;
  g = ga(m->d_dZ2T, M, m->d_H1T, M, kHid, kHid, (int)M, G_STORE, m->d_err);
  g.C = m->d_dW2, g.ldc = kHid;
  if ((rc = gemm(g, st))) return rc;
  g = ga(m->d_dZ1T, M, m->d_XT, M, kHid, kInPad, (int)M, G_STORE, m->d_err);
  g.C = m->d_dW1, g.ldc = kInPad;
  if ((rc = gemm(g, st))) return rc;
  float c1 = 1.0f, c2 = 1.0f;
  if (lr > 0.0f) {
    m->adam_t += 1;
    c1 = 1.0f - powf(0.9f, (float)m->adam_t);
    c2 = 1.0f - powf(0.999f, (float)m->adam_t);
  }
  k_grad_adam<<<(unsigned)((kParams + 255) / 256), 256, 0, st>>>(m->d_master, m->d_m, m->d_v, m->d_grad, m->d_dW1,
                                                                 m->d_dW2, m->d_dW3T, m->d_dZ1T, m->d_dZ2T,
                                                                 m->d_dOT, M, lr, c1, c2, m->n_in);
  LTRY(cudaGetLastError());
  if (lr > 0.0f)
    if ((rc = refresh_bf16(m))) return rc;
  return SCEMC_OK;
}

int32_t check_err(scemc_mlp* m) {
  int e = 0;
  LTRY(cudaMemcpyAsync(&e, m->d_err, sizeof(int), cudaMemcpyDeviceToHost, m->stream));
  LTRY(cudaStreamSynchronize(m->stream));
  if (e) {
    LTRY(cudaMemsetAsync(m->d_err, 0, sizeof(int), m->stream));
    return fail(SCEMC_ERR_TIMEOUT, "a tensor-core completion wait ran out (1 s)");
  }
  return SCEMC_OK;
}

}  // namespace

namespace scemc_detail {
int32_t mlp_forward_dev(const scemc_mlp* m, const bf16* X, int64_t M, bf16* H1, bf16* H2, float* O, cudaStream_t st,
                        int* err) {
  int32_t rc;
  GemmArgs g = ga(X, kInPad, m->d_W1, kInPad, M, kHid, kInPad, G_BIAS_SILU, err);
  g.bias = m->d_master + oB1, g.H = H1, g.ldh = kHid;
  if ((rc = gemm(g, st))) return rc;
  g = ga(H1, kHid, m->d_W2, kHid, M, kHid, kHid, G_BIAS_SILU, err);
  g.bias = m->d_master + oB2, g.H = H2, g.ldh = kHid;
  if ((rc = gemm(g, st))) return rc;
  g = ga(H2, kHid, m->d_W3, kHid, M, kOutPad, kHid, G_BIAS, err);
  g.C = O, g.ldc = kOutPad, g.bias = m->d_master + oB3;
  return gemm(g, st);
}
}  // namespace scemc_detail

extern "C" {

int32_t scemc_mlp_create(uint64_t seed, int32_t n_in, scemc_mlp** out) {
  if (!out) return fail(SCEMC_ERR_ARG, "NULL argument");
  *out = nullptr;
  if (n_in < 2 || n_in > kInPad) return fail(SCEMC_ERR_ARG, "n_in must be 2..64 (inputs, kT last)");
  int dev = 0;
  LTRY(cudaGetDevice(&dev));
  auto* m = new scemc_mlp();
  m->device = dev;
  m->n_in = n_in;
  int32_t rc = SCEMC_OK;
  auto bail = [&](int32_t r) {
    scemc_mlp_destroy(m);
    return r;
  };
  if (cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking) != cudaSuccess)
    return bail(fail(SCEMC_ERR_CUDA, "stream create"));
  if ((rc = dal(&m->d_master, kParams)) || (rc = dal(&m->d_m, kParams)) || (rc = dal(&m->d_v, kParams)) ||
      (rc = dal(&m->d_grad, kParams)) || (rc = dal(&m->d_W1, (size_t)kHid * kInPad)) ||
      (rc = dal(&m->d_W2, (size_t)kHid * kHid)) || (rc = dal(&m->d_W2T, (size_t)kHid * kHid)) ||
      (rc = dal(&m->d_W3, (size_t)kOutPad * kHid)) || (rc = dal(&m->d_W3T, (size_t)kHid * kOutPad)) ||
      (rc = dal(&m->d_err, 1)))
    return bail(rc);
  // He-style initial weights from a seeded generator (host), concentrations
  // starting at softplus(1) kT
  std::vector<float> P(kParams, 0.0f);
  std::mt19937_64 g(seed);
  std::normal_distribution<double> nd(0.0, 1.0);
  for (int r = 0; r < kHid; ++r)
    for (int c = 0; c < n_in; ++c) P[oW1 + r * kInPad + c] = (float)(nd(g) * std::sqrt(2.0 / n_in));
  for (int i = 0; i < kHid * kHid; ++i) P[oW2 + i] = (float)(nd(g) * std::sqrt(2.0 / kHid));
  for (int o = 0; o < kOut; ++o)
    for (int h = 0; h < kHid; ++h) P[oW3 + o * kHid + h] = (float)(nd(g) * std::sqrt(1.0 / kHid) * 0.1);
  for (int k = 0; k < 4; ++k) P[oB3 + 5 * k + 4] = 1.0f;
  if (cudaMemcpy(m->d_master, P.data(), kParams * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemset(m->d_m, 0, kParams * sizeof(float)) != cudaSuccess ||
      cudaMemset(m->d_v, 0, kParams * sizeof(float)) != cudaSuccess ||
      cudaMemset(m->d_err, 0, sizeof(int)) != cudaSuccess)
    return bail(fail(SCEMC_ERR_CUDA, "parameter upload"));
  if ((rc = refresh_bf16(m))) return bail(rc);
  if (cudaStreamSynchronize(m->stream) != cudaSuccess) return bail(fail(SCEMC_ERR_CUDA, "init sync"));
  *out = m;
  return SCEMC_OK;
}

int32_t scemc_mlp_destroy(scemc_mlp* m) {
  if (!m) return SCEMC_OK;
  if (m->stream) cudaStreamSynchronize(m->stream);
  free_work(m);
  void* ps[] = {m->d_master, m->d_m, m->d_v, m->d_grad, m->d_W1, m->d_W2, m->d_W2T, m->d_W3, m->d_W3T, m->d_err};
  for (void* p : ps)
    if (p) cudaFree(p);
  if (m->stream) cudaStreamDestroy(m->stream);
  delete m;
  return SCEMC_OK;
}

int32_t scemc_mlp_get_params(const scemc_mlp* m, float* params) {
  if (!m || !params) return fail(SCEMC_ERR_ARG, "NULL argument");
  LTRY(cudaMemcpyAsync(params, m->d_master, kParams * sizeof(float), cudaMemcpyDeviceToHost, m->stream));
  LTRY(cudaStreamSynchronize(m->stream));
  return SCEMC_OK;
}

int32_t scemc_mlp_set_params(scemc_mlp* m, const float* params) {
  if (!m || !params) return fail(SCEMC_ERR_ARG, "NULL argument");
  LTRY(cudaMemcpyAsync(m->d_master, params, kParams * sizeof(float), cudaMemcpyHostToDevice, m->stream));
  int32_t rc;
  if ((rc = refresh_bf16(m))) return rc;
  LTRY(cudaStreamSynchronize(m->stream));
  return SCEMC_OK;
}

int32_t scemc_mlp_forward(scemc_mlp* m, const float* x, int64_t n, float* out) {
  if (!m || !x || !out || n < 1) return fail(SCEMC_ERR_ARG, "bad forward arguments");
  const int64_t M = (n + 127) / 128 * 128;
  int32_t rc;
  if ((rc = ensure_work(m, M))) return rc;
  float* dx = nullptr;
  LTRY(cudaMallocAsync(reinterpret_cast<void**>(&dx), (size_t)n * m->n_in * sizeof(float), m->stream));
  LTRY(cudaMemcpyAsync(dx, x, (size_t)n * m->n_in * sizeof(float), cudaMemcpyHostToDevice, m->stream));
  k_rows_in<<<256, 256, 0, m->stream>>>(dx, nullptr, nullptr, n, M, m->d_X, nullptr, m->d_tau, nullptr, m->n_in);
  LTRY(cudaGetLastError());
  rc = scemc_detail::mlp_forward_dev(m, m->d_X, M, m->d_H1, m->d_H2, m->d_O, m->stream, m->d_err);
  LTRY(cudaFreeAsync(dx, m->stream));
  if (rc) return rc;
  LTRY(cudaMemcpy2DAsync(out, kOut * sizeof(float), m->d_O, kOutPad * sizeof(float), kOut * sizeof(float), (size_t)n,
                         cudaMemcpyDeviceToHost, m->stream));
  return check_err(m);
}

int32_t scemc_mlp_loss_grad(scemc_mlp* m, const float* x, const float* y, int64_t n, double* loss, float* grad) {
  if (!m || !x || !y || n < 1) return fail(SCEMC_ERR_ARG, "bad loss_grad arguments");
  if (n % 128) return fail(SCEMC_ERR_ARG, "loss_grad needs a multiple of 128 rows");
  int32_t rc;
  if ((rc = ensure_work(m, n))) return rc;
  float *dx = nullptr, *dy = nullptr;
  LTRY(cudaMallocAsync(reinterpret_cast<void**>(&dx), (size_t)n * m->n_in * sizeof(float), m->stream));
  LTRY(cudaMallocAsync(reinterpret_cast<void**>(&dy), (size_t)n * 3 * sizeof(float), m->stream));
  LTRY(cudaMemcpyAsync(dx, x, (size_t)n * m->n_in * sizeof(float), cudaMemcpyHostToDevice, m->stream));
  LTRY(cudaMemcpyAsync(dy, y, (size_t)n * 3 * sizeof(float), cudaMemcpyHostToDevice, m->stream));
  k_rows_in<<<256, 256, 0, m->stream>>>(dx, dy, nullptr, n, n, m->d_X, m->d_XT, m->d_tau, m->d_Y, m->n_in);
  LTRY(cudaGetLastError());
  rc = step_rows(m, n, n, 0.0f);
  LTRY(cudaFreeAsync(dx, m->stream));
  LTRY(cudaFreeAsync(dy, m->stream));
  if (rc) return rc;
  std::vector<double> l(n);
  LTRY(cudaMemcpyAsync(l.data(), m->d_loss, n * sizeof(double), cudaMemcpyDeviceToHost, m->stream));
  if (grad) LTRY(cudaMemcpyAsync(grad, m->d_grad, kParams * sizeof(float), cudaMemcpyDeviceToHost, m->stream));
  if ((rc = check_err(m))) return rc;
  if (loss) *loss = std::accumulate(l.begin(), l.end(), 0.0) / (double)n;
  return SCEMC_OK;
}

int32_t scemc_mlp_train(scemc_mlp* m, const float* x, const float* y, int64_t n, int32_t batch, int32_t epochs,
                        double lr, uint64_t seed, double* epoch_loss) {
  if (!m || !x || !y || n < 1 || epochs < 0 || !(lr > 0.0)) return fail(SCEMC_ERR_ARG, "bad train arguments");
  if (batch < 128 || batch % 128 || batch > n) return fail(SCEMC_ERR_ARG, "batch must be a multiple of 128 <= n");
  int32_t rc;
  if ((rc = ensure_work(m, batch))) return rc;
  float *dx = nullptr, *dy = nullptr;
  int32_t* didx = nullptr;
  LTRY(cudaMalloc(reinterpret_cast<void**>(&dx), (size_t)n * m->n_in * sizeof(float)));
  LTRY(cudaMalloc(reinterpret_cast<void**>(&dy), (size_t)n * 3 * sizeof(float)));
  LTRY(cudaMalloc(reinterpret_cast<void**>(&didx), (size_t)n * sizeof(int32_t)));
  auto cleanup = [&]() {
    cudaStreamSynchronize(m->stream);
    cudaFree(dx);
    cudaFree(dy);
    cudaFree(didx);
  };
  if (cudaMemcpy(dx, x, (size_t)n * m->n_in * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(dy, y, (size_t)n * 3 * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess) {
    cleanup();
    return fail(SCEMC_ERR_CUDA, "dataset upload");
  }
  std::vector<int32_t> perm(n);
  std::iota(perm.begin(), perm.end(), 0);
  std::mt19937_64 g(seed);
  const int64_t steps = n / batch;
  std::vector<double> l(batch);
  for (int e = 0; e < epochs; ++e) {
    std::shuffle(perm.begin(), perm.end(), g);
    if (cudaMemcpyAsync(didx, perm.data(), (size_t)n * sizeof(int32_t), cudaMemcpyHostToDevice, m->stream) !=
        cudaSuccess) {
      cleanup();
      return fail(SCEMC_ERR_CUDA, "permutation upload");
    }
    double acc = 0.0;
    for (int64_t s = 0; s < steps; ++s) {
      k_rows_in<<<256, 256, 0, m->stream>>>(dx, dy, didx + s * batch, batch, batch, m->d_X, m->d_XT, m->d_tau,
                                            m->d_Y, m->n_in);
      if ((rc = step_rows(m, batch, batch, (float)lr))) {
        cleanup();
        return rc;
      }
      if (epoch_loss) {
        cudaMemcpyAsync(l.data(), m->d_loss, batch * sizeof(double), cudaMemcpyDeviceToHost, m->stream);
        cudaStreamSynchronize(m->stream);
        acc += std::accumulate(l.begin(), l.end(), 0.0) / (double)batch;
      }
    }
    if (epoch_loss) epoch_loss[e] = acc / (double)steps;
  }
  rc = check_err(m);
  cleanup();
  return rc;
}

}  // extern "C"
