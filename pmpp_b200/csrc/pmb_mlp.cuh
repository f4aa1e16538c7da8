// Internal interfaces of mlp.cu.
#pragma once

#include "pmb_common.cuh"

namespace pmb {

constexpr int kMlpWidth = 64;
// parameter counts: bf16 weights W1 (64x4), W2 (64x64), W3 (64x64), W4 (64);
// FP32 biases b1, b2, b3 (64 each) and b4 (1)
constexpr int kMlpWeights = kMlpWidth * 4 + 2 * kMlpWidth * kMlpWidth + kMlpWidth;
constexpr int kMlpBiases = 3 * kMlpWidth + 1;

struct MlpCond {
  float kscale;  // |k| / k_Nyquist per unit sqrt(n^2) (2 / M for a cubic mesh)
  float a;
  float omega_m;
  float sigma8;
};

int mlp_table(const void* w, const float* b, MlpCond c, int len, float* table, cudaStream_t s);
int mlp_backward(const void* w, const float* b, MlpCond c, int len, const double* tcot, float* grad, cudaStream_t s);
int transfer_cot(const float2* R3, const float2* S_hat, Mesh3 m, SpecTables t, int len, double* out, cudaStream_t s);

}  // namespace pmb
