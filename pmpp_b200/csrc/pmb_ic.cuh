// Internal interfaces of ic.cu.
#pragma once

#include "pmb_common.cuh"

namespace pmb {

struct LinearPowerParams {
  double coef;           // 0.32 * A_s * k_pivot
  double k_pivot;
  double n_s;
  double pi_c2_over_om;  // pi (c/H0)^2 / Omega_m
  double growth2;        // D(a)^2, or 1 without growth
  double box_vol;        // rounded to the working precision by the kernel
};

int white_noise(uint32_t seed, Mesh3 m, float2* out, uint32_t* hashes, cudaStream_t s);
int linear_modes(const float2* in, float2* out, float* amp, Mesh3 m, const float* ktab, const double* tk,
                 const double* tt, int ntab, LinearPowerParams p, cudaStream_t s);
int lpt_strains(const float2* modes, float inv_cell_vol, float2* pot1, float2* strains, Mesh3 m, const float* tab,
                float inv_n, cudaStream_t s);
int lpt_source(const float* s6, float* L, int64_t n, cudaStream_t s);
int lpt_gradients(const float2* pot1, const float2* L_hat, float2* grads, Mesh3 m, const float* tab, float inv_n,
                  cudaStream_t s);
int lpt_displace(const int16_t* pmid, float* disp, float* vel, int64_t n, Mesh3 g, float cell, float spacing,
                 const float* fields, int order, float D1, float V1, float D2, float V2, int64_t* index_out,
                 cudaStream_t s);
int lpt_field_cot(const int64_t* index, const float* disp_cot, const float* vel_cot, int64_t n, int64_t ng,
                  const float* fields, int order, float D1, float V1, float D2, float V2, float* cot, double* dots,
                  cudaStream_t s);
int lpt_grad2_adjoint(const float2* F2, float2* out, Mesh3 m, const float* tab, float post, cudaStream_t s);
int lpt_source_adjoint(const float* s6, const float* Lc, float* c6, int64_t n, cudaStream_t s);
int lpt_modes_adjoint(const float2* F1, const float2* FS, const float* amp, float2* out, Mesh3 m, const float* tab,
                      float scale, cudaStream_t s);
int pk_shells(const float2* spec, Mesh3 m, const float* sinc_tab, int mas_power, int num_shells, double* sums,
              const float2* spec_b, double* sums_b, double* sums_x, cudaStream_t s);
int pk_shells_adjoint(const float2* spec, Mesh3 m, const float* sinc_tab, int mas_power, int num_shells,
                      const double* wshell, float post, float2* out, cudaStream_t s);
int overdensity(const float* rho, float* delta, int64_t n, const double* total, cudaStream_t s);
int shell_stats(Mesh3 m, int num_shells, double* counts, double* ksum, cudaStream_t s);

// float64 instantiations of the same kernels (the reference's x64 build)
int white_noise64(uint32_t seed, Mesh3 m, double2* out, cudaStream_t s);
int linear_modes64(const double2* in, double2* out, Mesh3 m, const double* ktab, const double* tk, const double* tt,
                   int ntab, LinearPowerParams p, cudaStream_t s);
int lpt_strains64(const double2* modes, double inv_cell_vol, double2* pot1, double2* strains, Mesh3 m,
                  const double* tab, double inv_n, cudaStream_t s);
int lpt_source64(const double* s6, double* L, int64_t n, cudaStream_t s);
int lpt_gradients64(const double2* pot1, const double2* L_hat, double2* grads, Mesh3 m, const double* tab,
                    double inv_n, cudaStream_t s);
int lpt_displace64(const int16_t* pmid, double* disp, double* vel, int64_t n, Mesh3 g, double cell, double spacing,
                   const double* fields, int order, double D1, double V1, double D2, double V2, int64_t* index_out,
                   cudaStream_t s);
int lpt_field_cot64(const int64_t* index, const double* disp_cot, const double* vel_cot, int64_t n, int64_t ng,
                    const double* fields, int order, double D1, double V1, double D2, double V2, double* cot,
                    double* dots, cudaStream_t s);
int lpt_grad2_adjoint64(const double2* F2, double2* out, Mesh3 m, const double* tab, double post, cudaStream_t s);
int lpt_source_adjoint64(const double* s6, const double* Lc, double* c6, int64_t n, cudaStream_t s);
int lpt_modes_adjoint64(const double2* F1, const double2* FS, const double* amp, double2* out, Mesh3 m,
                        const double* tab, double scale, cudaStream_t s);
int pk_shells64(const double2* spec, Mesh3 m, const double* sinc_tab, int mas_power, int num_shells, double* sums,
                cudaStream_t s);
int pk_shells_adjoint64(const double2* spec, Mesh3 m, const double* sinc_tab, int mas_power, int num_shells,
                        const double* wshell, double post, double2* out, cudaStream_t s);
int overdensity64(const double* rho, double* delta, int64_t n, const double* total, cudaStream_t s);

}  // namespace pmb
