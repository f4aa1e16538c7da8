// Per-element spectral multipliers shared by the single-simulation kernels
// (spectral.cu) and the persistent ensemble kernels (ensemble.cu).
//
// Reference semantics: nbody/gravity.py:174-196 (particle-Nyquist masks),
// :283-352 (Poisson kernels), :355-391 and core/configuration.py:365-376
// (spectral gradient), corrections/core.py:333-334 (multiplicative transfer).
#pragma once

#include "pmb_common.cuh"
#include "pmb_kernels.cuh"

namespace pmb {

// K(k) = mask(k) * G(k) * T(k) with G = -1/k^2 (0 where k^2 == 0).
// Forward:  phi = (-(S*mask)) / k2 * T ; grad_d = (i c_d) phi,  d = x, y, z.
// The division is done component-wise in float, as the reference's
// complex-by-real division (gravity.py:285, :350-352).
__device__ __forceinline__ float k2_of(const SpecTables& t, int ix, int iy, int iz) {
  const float kx = t.kx[ix], ky = t.ky[iy], kz = t.kz[iz];
  return __fadd_rn(__fadd_rn(__fmul_rn(kx, kx), __fmul_rn(ky, ky)), __fmul_rn(kz, kz));
}

__device__ __forceinline__ float transfer_of(const GreenParams& g, const SpecTables& t, int64_t j, int ix, int iy, int iz,
                                             Mesh3 m) {
  float T = 1.0f;
  if (g.transfer != nullptr) T = g.transfer[j];
  if (g.radial != nullptr) {
    // integer mode numbers: |n|^2 indexes the radial table exactly
    const int nx = ix < (m.nx + 1) / 2 ? ix : ix - m.nx;
    const int ny = iy < (m.ny + 1) / 2 ? iy : iy - m.ny;
    const long long n2 = (long long)nx * nx + (long long)ny * ny + (long long)iz * iz;
    T = __fmul_rn(T, n2 < g.radial_len ? g.radial[n2] : 1.0f);
  }
  return T;
}

// Forward multiplier at half-spectrum cell j = (ix*ny + iy)*(nz/2+1) + iz:
// the three gradient values from the source value v.
__device__ __forceinline__ void green_gradient_value(float2 v, int64_t j, int ix, int iy, int iz, Mesh3 m,
                                                     const SpecTables& t, const GreenParams& g, float2 out[3]) {
  if (t.mx != nullptr) {
    const float mk = __fmul_rn(__fmul_rn(t.mx[ix], t.my[iy]), t.mz[iz]);
    v.x = __fmul_rn(v.x, mk);
    v.y = __fmul_rn(v.y, mk);
  }
  const float k2 = k2_of(t, ix, iy, iz);
  float pr = 0.f, pi = 0.f;
  if (k2 != 0.f) {
    pr = __fdiv_rn(-v.x, k2);
    pi = __fdiv_rn(-v.y, k2);
    if (g.transfer != nullptr || g.radial != nullptr) {
      const float T = transfer_of(g, t, j, ix, iy, iz, m);
      pr = __fmul_rn(pr, T);
      pi = __fmul_rn(pi, T);
    }
  }
  const float c[3] = {t.cx[ix], t.cy[iy], t.cz[iz]};
  const float ps = g.post_scale;
#pragma unroll
  for (int d = 0; d < 3; ++d) out[d] = make_float2(__fmul_rn(-__fmul_rn(c[d], pi), ps), __fmul_rn(__fmul_rn(c[d], pr), ps));
}

// Half-spectrum cell j of the forward multiplier: three gradient spectra
// (channel stride `total`) from one source spectrum.
__device__ __forceinline__ void green_gradient_at(const float2* __restrict__ src, float2* __restrict__ grad, int64_t j,
                                                  int64_t total, int ix, int iy, int iz, Mesh3 m, const SpecTables& t,
                                                  const GreenParams& g) {
  float2 o[3];
  green_gradient_value(src[j], j, ix, iy, iz, m, t, g, o);
#pragma unroll
  for (int d = 0; d < 3; ++d) grad[(int64_t)d * total + j] = o[d];
}

// Adjoint at half-spectrum cell j: S_cot = K * sum_d conj(i c_d) A_d.  The
// force map is a real convolution (H_d Hermitian), so its transpose is the
// correlation with the conjugate multiplier.
__device__ __forceinline__ float2 green_gradient_adjoint_value(const float2 a[3], int64_t j, int ix, int iy, int iz,
                                                               Mesh3 m, const SpecTables& t, const GreenParams& g) {
  const float c[3] = {t.cx[ix], t.cy[iy], t.cz[iz]};
  float ar = 0.f, ai = 0.f;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    ar = __fadd_rn(ar, __fmul_rn(c[d], a[d].y));
    ai = __fsub_rn(ai, __fmul_rn(c[d], a[d].x));
  }
  const float k2 = k2_of(t, ix, iy, iz);
  float pr = 0.f, pi = 0.f;
  if (k2 != 0.f) {
    if (g.transfer != nullptr || g.radial != nullptr) {
      const float T = transfer_of(g, t, j, ix, iy, iz, m);
      ar = __fmul_rn(ar, T);
      ai = __fmul_rn(ai, T);
    }
    pr = __fdiv_rn(-ar, k2);
    pi = __fdiv_rn(-ai, k2);
    if (t.mx != nullptr) {
      const float mk = __fmul_rn(__fmul_rn(t.mx[ix], t.my[iy]), t.mz[iz]);
      pr = __fmul_rn(pr, mk);
      pi = __fmul_rn(pi, mk);
    }
  }
  return make_float2(__fmul_rn(pr, g.post_scale), __fmul_rn(pi, g.post_scale));
}

__device__ __forceinline__ void green_gradient_adjoint_at(const float2* __restrict__ gc, float2* __restrict__ out,
                                                          int64_t j, int64_t total, int ix, int iy, int iz, Mesh3 m,
                                                          const SpecTables& t, const GreenParams& g) {
  const float2 a[3] = {gc[j], gc[total + j], gc[2 * total + j]};
  out[j] = green_gradient_adjoint_value(a, j, ix, iy, iz, m, t, g);
}

}  // namespace pmb
