// Host-side view of the learned proposal's network, shared by the two translation
// units of libscemc_cuda.so (learned.cu owns the network and its training;
// scemc.cu runs it inside the sweep).
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

// Parameter block (FP32 masters, padded shapes), offsets in floats:
// W1 [128][64] (input columns n_in..63 zero; n_in = 43 for 14 environment spins),
// b1 [128], W2 [128][128], b2 [128],
// W3 [32][128] (output rows 20..31 zero), b3 [32].
namespace mlpl {
constexpr int kIn = 43, kInPad = 64, kHid = 128, kOut = 20, kOutPad = 32;
constexpr int64_t oW1 = 0, oB1 = oW1 + kHid * kInPad, oW2 = oB1 + kHid, oB2 = oW2 + kHid * kHid,
                  oW3 = oB2 + kHid, oB3 = oW3 + kOutPad * kHid, kParams = oB3 + kOutPad;
}  // namespace mlpl

struct scemc_mlp {
  int device = 0;
  int32_t n_in = mlpl::kIn;  // inputs per row (kT last), at most kInPad
  cudaStream_t stream = nullptr;
  float* d_master = nullptr;  // kParams FP32
  float* d_m = nullptr;       // Adam moments
  float* d_v = nullptr;
  float* d_grad = nullptr;    // last gradient (kParams)
  int64_t adam_t = 0;
  // BF16 copies used by the tensor-core kernels: W1 [128][64], W2 [128][128],
  // W2T [128][128], W3 [32][128], W3T [128][32]
  __nv_bfloat16 *d_W1 = nullptr, *d_W2 = nullptr, *d_W2T = nullptr, *d_W3 = nullptr, *d_W3T = nullptr;
  // training work buffers for `cap` rows
  int64_t cap = 0;
  __nv_bfloat16 *d_X = nullptr, *d_XT = nullptr, *d_H1 = nullptr, *d_H1T = nullptr, *d_H2 = nullptr,
                *d_H2T = nullptr, *d_dO = nullptr, *d_dOT = nullptr, *d_dZ2 = nullptr, *d_dZ2T = nullptr,
                *d_dZ1T = nullptr;
  float *d_Z1 = nullptr, *d_Z2 = nullptr, *d_O = nullptr, *d_tau = nullptr, *d_Y = nullptr;
  float *d_dW1 = nullptr, *d_dW2 = nullptr, *d_dW3T = nullptr;
  double* d_loss = nullptr;
  int* d_err = nullptr;
};

namespace scemc_detail {
int32_t set_error(int32_t code, const char* msg);
// O [M][32] = MLP(X [M][64]) for M a multiple of 128 (BF16 inputs, FP32 outputs);
// H1 and H2 are [M][128] BF16 scratch. Enqueued on `st`; err is a device flag.
int32_t mlp_forward_dev(const scemc_mlp* m, const __nv_bfloat16* X, int64_t M, __nv_bfloat16* H1,
                        __nv_bfloat16* H2, float* O, cudaStream_t st, int* err);
}  // namespace scemc_detail
