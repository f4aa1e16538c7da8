// Internal interfaces of integrate.cu.
#pragma once

#include "pmb_common.cuh"

namespace pmb {
int axpy(float* y, const float* x, int64_t n, float f, cudaStream_t s);
int kick_adj(float* vel, const float* acc, const float* vel_cot, float* acc_cot, int64_t n, float k, double* dot,
             cudaStream_t s);
int kick_adj2(float* vel, const float* acc, float* vel_cot, float* acc_cot, int64_t n, float ka, float kb,
              int two, int zero_cot, double* dot_a, double* dot_b, double* dot_f, const float* disp_cot, float dd,
              double* dot_d, cudaStream_t s);
int drift_cot_adj(const float* vel, const float* disp_cot, float* vel_cot, int64_t n, float d, double* dot,
                  cudaStream_t s);
int drift_adj(float* disp, const float* vel, const float* disp_cot, float* vel_cot, int64_t n, float d, double* dot,
              cudaStream_t s);
int dot(const float* a, const float* b, int64_t n, double* out, cudaStream_t s);
int sum(const float* a, int64_t n, double* out, cudaStream_t s);
int set_double(double* p, double v, cudaStream_t s);
}  // namespace pmb
