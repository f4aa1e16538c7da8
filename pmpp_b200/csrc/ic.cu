// Initial conditions and power spectrum on the device:
//  * nested white noise: hashed Gaussian Fourier modes that are identical for
//    shared low-k modes across resolutions (initial_conditions/modes.py:92-268);
//  * linear modes delta(k) = omega(k) sqrt(V P_lin(|k|)) (modes.py:397-454,
//    cosmology/boltzmann.py:428-484), P_lin evaluated in FP64 from the
//    tabulated transfer function;
//  * 2LPT spectral stages and their adjoints (initial_conditions/lpt.py:17-449);
//  * FP64 power-spectrum shell sums (analysis/power_spectrum.py:106-143) and
//    the adjoint of the shell power.
#include <cmath>

#include "pmb_common.cuh"
#include "pmb_ic.cuh"

namespace pmb {

namespace {
unsigned grid_for(int64_t total, int th) {
  int64_t b = (total + th - 1) / th;
  int64_t cap = 148 * 32;
  return (unsigned)(b < cap ? (b > 0 ? b : 1) : cap);
}

struct Idx3 {
  int ix, iy, iz;
};
__device__ __forceinline__ Idx3 unravel_half(int64_t j, Mesh3 m) {
  const int nzh = m.nz / 2 + 1;
  Idx3 r;
  r.iz = (int)(j % nzh);
  const int64_t q = j / nzh;
  r.iy = (int)(q % m.ny);
  r.ix = (int)(q / m.ny);
  return r;
}

__device__ __forceinline__ int fft_mode(int i, int n) { return i < (n + 1) / 2 ? i : i - n; }

// lowbias32 finaliser (modes.py:92-111)
__device__ __forceinline__ uint32_t mix32(uint32_t x) {
  x ^= x >> 16;
  x *= 0x7FEB352Du;
  x ^= x >> 15;
  x *= 0x846CA68Bu;
  x ^= x >> 16;
  return x;
}

// modes.py:114-129
__device__ __forceinline__ uint32_t hash_mode(uint32_t seed, int kx, int ky, int kz, uint32_t salt) {
  uint32_t h = mix32(seed ^ salt);
  h = mix32(h ^ mix32((uint32_t)kx + 0x9E3779B9u));
  h = mix32(h ^ mix32((uint32_t)ky + 0x85EBCA6Bu));
  h = mix32(h ^ mix32((uint32_t)kz + 0xC2B2AE35u));
  return h;
}

__device__ __forceinline__ bool self_inverse(int k, int n) { return k == 0 || ((n % 2 == 0) && k == -(n / 2)); }
}  // namespace

// ---------------------------------------------------------------------------
// Nested white noise (modes.py:181-220)
// ---------------------------------------------------------------------------
template <class T>
__global__ void white_noise_kernel(uint32_t seed, Mesh3 m, typename Real<T>::T2* __restrict__ out,
                                   uint32_t* __restrict__ hashes) {
  using R = Real<T>;
  const int64_t total = m.half_cells();
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < total; j += (int64_t)gridDim.x * blockDim.x) {
    const Idx3 q = unravel_half(j, m);
    const int kx = fft_mode(q.ix, m.nx), ky = fft_mode(q.iy, m.ny), kz = q.iz;
    const bool plane = kz == 0 || ((m.nz % 2 == 0) && kz == m.nz / 2);
    // canonical member of each Hermitian pair on self-conjugate planes
    const int px = self_inverse(kx, m.nx) ? kx : -kx;
    const int py = self_inverse(ky, m.ny) ? ky : -ky;
    const bool keep = (kx < px) || (kx == px && ky <= py);
    const int hx = plane ? (keep ? kx : px) : kx;
    const int hy = plane ? (keep ? ky : py) : ky;
    const bool self_point = self_inverse(kx, m.nx) && self_inverse(ky, m.ny);
    const uint32_t hr = hash_mode(seed, hx, hy, kz, 0xA24BAED4u);
    const uint32_t hi = hash_mode(seed, hx, hy, kz, 0x9FB21C65u);
    if (hashes != nullptr) {
      hashes[2 * j] = hr;
      hashes[2 * j + 1] = hi;
    }
    // Box-Muller on bin-centred uniforms (modes.py:132-152) in the working precision
    const T scale = (T)2.3283064365386963e-10;
    const T u1 = R::mul(R::add((T)hr, (T)0.5), scale);
    const T u2 = R::mul(R::add((T)hi, (T)0.5), scale);
    const T r = R::sqrt_(R::mul((T)-2.0, R::log_(u1)));
    const T th = R::mul((T)6.2831853071795865, u2);
    const T gr = R::mul(r, R::cos_(th)), gi = R::mul(r, R::sin_(th));
    const T sq = (T)0.7071067811865476;
    typename R::T2 c = R::make2(R::mul(gr, sq), R::mul(gi, sq));
    if (plane) {
      if (self_point) c = R::make2(gr, (T)0);
      if (!keep) c.y = -c.y;
    }
    out[j] = c;
  }
}

int white_noise(uint32_t seed, Mesh3 m, float2* out, uint32_t* hashes, cudaStream_t s) {
  white_noise_kernel<float><<<grid_for(m.half_cells(), 256), 256, 0, s>>>(seed, m, out, hashes);
  PMB_CUDA_CHECK(cudaGetLastError());
  return kOk;
}

int white_noise64(uint32_t seed, Mesh3 m, double2* out, cudaStream_t s) {
  white_noise_kernel<double><<<grid_for(m.half_cells(), 256), 256, 0, s>>>(seed, m, out, nullptr);
  PMB_CUDA_CHECK(cudaGetLastError());
  return kOk;
}

// ---------------------------------------------------------------------------
// Linear modes (modes.py:429-446)
// ---------------------------------------------------------------------------
// k = sqrt(k2) in float (modes.py:314-316); P_lin(k) in FP64 with linear
// interpolation of the transfer table and constant extrapolation
// (boltzmann.py:170, jnp.interp); amplitude sqrt(float(P) * V) in float.
__device__ double interp_table(double x, const double* __restrict__ xp, const double* __restrict__ fp, int n) {
  if (x <= xp[0]) return fp[0];
  if (x >= xp[n - 1]) return fp[n - 1];
  int lo = 0, hi = n - 1;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (xp[mid] <= x) lo = mid; else hi = mid;
  }
  return fp[lo] + (x - xp[lo]) * (fp[hi] - fp[lo]) / (xp[hi] - xp[lo]);
}

template <class T>
__global__ void linear_modes_kernel(const typename Real<T>::T2* __restrict__ in, typename Real<T>::T2* __restrict__ out,
                                    T* __restrict__ amp_out, Mesh3 m, const T* __restrict__ kx,
                                    const T* __restrict__ ky, const T* __restrict__ kz, const double* __restrict__ tk,
                                    const double* __restrict__ tt, int ntab, LinearPowerParams p) {
  using R = Real<T>;
  const int64_t total = m.half_cells();
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < total; j += (int64_t)gridDim.x * blockDim.x) {
    const Idx3 q = unravel_half(j, m);
    const T a = kx[q.ix], b = ky[q.iy], c = kz[q.iz];
    const T k = R::sqrt_(R::add(R::add(R::mul(a, a), R::mul(b, b)), R::mul(c, c)));
    const double kd = (double)k;
    const double Tk = interp_table(kd, tk, tt, ntab);
    const double amp = p.pi_c2_over_om * Tk;
    const double P = kd > 0.0 ? p.coef * pow(kd / p.k_pivot, p.n_s) * amp * amp * p.growth2 : 0.0;
    const T A = R::sqrt_(R::mul((T)P, (T)p.box_vol));
    if (amp_out != nullptr) amp_out[j] = A;
    if (in != nullptr) {
      const typename R::T2 v = in[j];
      out[j] = R::make2(R::mul(v.x, A), R::mul(v.y, A));
    }
  }
}

int linear_modes(const float2* in, float2* out, float* amp, Mesh3 m, const float* ktab, const double* tk,
                 const double* tt, int ntab, LinearPowerParams p, cudaStream_t s) {
  const float* kx = ktab;
  const float* ky = kx + m.nx;
  const float* kz = ky + m.ny;
  linear_modes_kernel<float><<<grid_for(m.half_cells(), 256), 256, 0, s>>>(in, out, amp, m, kx, ky, kz, tk, tt, ntab,
                                                                           p);
  PMB_CUDA_CHECK(cudaGetLastError());
  return kOk;
}

int linear_modes64(const double2* in, double2* out, Mesh3 m, const double* ktab, const double* tk, const double* tt,
                   int ntab, LinearPowerParams p, cudaStream_t s) {
  const double* kx = ktab;
  const double* ky = kx + m.nx;
  const double* kz = ky + m.ny;
  linear_modes_kernel<double><<<grid_for(m.half_cells(), 256), 256, 0, s>>>(in, out, nullptr, m, kx, ky, kz, tk, tt,
                                                                            ntab, p);
  PMB_CUDA_CHECK(cudaGetLastError());
  return kOk;
}

// ---------------------------------------------------------------------------
// 2LPT spectral stages (lpt.py:17-43, 239-301, 379-431)
// ---------------------------------------------------------------------------
// tables: [kx ky kz cx cy cz] of the particle grid (c = Nyquist-zeroed -k).
template <class T>
struct LptTables {
  const T *kx, *ky, *kz, *cx, *cy, *cz;
};
template <class T>
__device__ __forceinline__ LptTables<T> lpt_tables(const T* t, Mesh3 m) {
  LptTables<T> r;
  const int nzh = m.nz / 2 + 1;
  r.kx = t;
  r.ky = r.kx + m.nx;
  r.kz = r.ky + m.ny;
  r.cx = r.kz + nzh;
  r.cy = r.cx + m.nx;
  r.cz = r.cy + m.ny;
  return r;
}

// pot1 = -(modes / cell_vol) / k^2 (lpt.py:379, 390; gravity.py:283-285)
template <class T>
__device__ __forceinline__ typename Real<T>::T2 pot_from(typename Real<T>::T2 v, T k2) {
  using R = Real<T>;
  if (k2 == (T)0) return R::make2((T)0, (T)0);
  return R::make2(R::div(-v.x, k2), R::div(-v.y, k2));
}

template <class T>
__device__ __forceinline__ T k2_at(const LptTables<T>& t, const Idx3& q) {
  using R = Real<T>;
  const T a = t.kx[q.ix], b = t.ky[q.iy], c = t.kz[q.iz];
  return R::add(R::add(R::mul(a, a), R::mul(b, b)), R::mul(c, c));
}

// Six strain spectra -k_i k_j pot1 * inv_n in the order (00, 11, 22, 01, 02,
// 12); off-diagonal factors use the Nyquist-zeroed wavenumbers (lpt.py:31-35).
// Also writes pot1 (times inv_n) for the first-order gradient.
template <class T>
__global__ void lpt_strain_kernel(const typename Real<T>::T2* __restrict__ modes, T inv_cell_vol,
                                  typename Real<T>::T2* __restrict__ pot1, typename Real<T>::T2* __restrict__ strains,
                                  Mesh3 m, const T* __restrict__ tab, T inv_n) {
  using R = Real<T>;
  const LptTables<T> t = lpt_tables(tab, m);
  const int64_t total = m.half_cells();
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < total; j += (int64_t)gridDim.x * blockDim.x) {
    const Idx3 q = unravel_half(j, m);
    typename R::T2 v = modes[j];
    v.x = R::mul(v.x, inv_cell_vol);
    v.y = R::mul(v.y, inv_cell_vol);
    const typename R::T2 p = pot_from<T>(v, k2_at(t, q));
    pot1[j] = p;
    const T k[3] = {t.kx[q.ix], t.ky[q.iy], t.kz[q.iz]};
    // Nyquist-zeroed k is -c
    const T kz0[3] = {-t.cx[q.ix], -t.cy[q.iy], -t.cz[q.iz]};
    const int pi[6] = {0, 1, 2, 0, 0, 1}, pj[6] = {0, 1, 2, 1, 2, 2};
#pragma unroll
    for (int s = 0; s < 6; ++s) {
      const T ki = s < 3 ? k[pi[s]] : kz0[pi[s]];
      const T kj = s < 3 ? k[pj[s]] : kz0[pj[s]];
      const T f = R::mul(R::mul(-ki, kj), inv_n);
      strains[(int64_t)s * total + j] = R::make2(R::mul(p.x, f), R::mul(p.y, f));
    }
  }
}

// 2LPT source sum_{i<j} phi_ii phi_jj - phi_ij^2 (lpt.py:263-299), summation
// order of the reference loops.
template <class T>
__global__ void lpt_source_kernel(const T* __restrict__ s6, T* __restrict__ L, int64_t n) {
  using R = Real<T>;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const T d0 = s6[i], d1 = s6[n + i], d2 = s6[2 * n + i];
    const T s01 = s6[3 * n + i], s02 = s6[4 * n + i], s12 = s6[5 * n + i];
    T l = (T)0;
    l = R::add(l, R::mul(d0, d2));
    l = R::add(l, R::mul(d0, d1));
    l = R::add(l, R::mul(d1, d2));
    l = R::sub(l, R::mul(s01, s01));
    l = R::sub(l, R::mul(s02, s02));
    l = R::sub(l, R::mul(s12, s12));
    L[i] = l;
  }
}

// pot2 = -L_hat / k^2, then the six gradient spectra (i c_d) pot_m * inv_n
// for m = 1 (from pot1) and m = 2 (from pot2), layout [m][d].
template <class T>
__global__ void lpt_gradient_kernel(const typename Real<T>::T2* __restrict__ pot1,
                                    const typename Real<T>::T2* __restrict__ L_hat,
                                    typename Real<T>::T2* __restrict__ grads, Mesh3 m, const T* __restrict__ tab,
                                    T inv_n) {
  using R = Real<T>;
  const LptTables<T> t = lpt_tables(tab, m);
  const int64_t total = m.half_cells();
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < total; j += (int64_t)gridDim.x * blockDim.x) {
    const Idx3 q = unravel_half(j, m);
    const typename R::T2 p1 = pot1[j];
    const typename R::T2 p2 = L_hat != nullptr ? pot_from<T>(L_hat[j], k2_at(t, q)) : R::make2((T)0, (T)0);
    const T c[3] = {t.cx[q.ix], t.cy[q.iy], t.cz[q.iz]};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      grads[(int64_t)d * total + j] = R::make2(R::mul(-R::mul(c[d], p1.y), inv_n), R::mul(R::mul(c[d], p1.x), inv_n));
      grads[(int64_t)(3 + d) * total + j] =
          R::make2(R::mul(-R::mul(c[d], p2.y), inv_n), R::mul(R::mul(c[d], p2.x), inv_n));
    }
  }
}

// Sample the gradient fields at the particles' Lagrangian grid points
// (lpt.py:46-62: rint((pmid*cell + disp)/spacing) mod grid) and apply
// disp += D_m g_m, vel += a^2 H D'_m g_m for m = 1..order (lpt.py:412-431).
template <class T>
__global__ void lpt_displace_kernel(const int16_t* __restrict__ pmid, T* __restrict__ disp, T* __restrict__ vel,
                                    int64_t n, Mesh3 g, T cell, T spacing, const T* __restrict__ fields, int order,
                                    T D1, T V1, T D2, T V2, int64_t* __restrict__ index_out) {
  using R = Real<T>;
  const int64_t ng = g.cells();
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (int64_t)gridDim.x * blockDim.x) {
    int c[3];
    const int dims[3] = {g.nx, g.ny, g.nz};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const T x = R::add(R::mul((T)pmid[3 * p + a], cell), disp[3 * p + a]);
      c[a] = pmod((int)R::rint_(R::div(x, spacing)), dims[a]);
    }
    const int64_t idx = ((int64_t)c[0] * g.ny + c[1]) * g.nz + c[2];
    if (index_out != nullptr) index_out[p] = idx;
    const T Ds[2] = {D1, D2}, Vs[2] = {V1, V2};
    for (int mo = 0; mo < order; ++mo) {
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        const T gv = fields[(int64_t)(3 * mo + d) * ng + idx];
        disp[3 * p + d] = R::add(disp[3 * p + d], R::mul(Ds[mo], gv));
        vel[3 * p + d] = R::add(vel[3 * p + d], R::mul(Vs[mo], gv));
      }
    }
  }
}

int lpt_strains(const float2* modes, float inv_cell_vol, float2* pot1, float2* strains, Mesh3 m, const float* tab,
                float inv_n, cudaStream_t s) {
  lpt_strain_kernel<float><<<grid_for(m.half_cells(), 256), 256, 0, s>>>(modes, inv_cell_vol, pot1, strains, m, tab,
                                                                         inv_n);
  PMB_CUDA_CHECK(cudaGetLastError());
  return kOk;
}

int lpt_source(const float* s6, float* L, int64_t n, cudaStream_t s) {
  lpt_source_kernel<float><<<grid_for(n, 256), 256, 0, s>>>(s6, L, n);
  PMB_CUDA_CHECK(cudaGetLastError());
  return kOk;
}

int lpt_gradients(const float2* pot1, const float2* L_hat, float2* grads, Mesh3 m, const float* tab, float inv_n,
                  cudaStream_t s) {
  lpt_gradient_kernel<float><<<grid_for(m.half_cells(), 256), 256, 0, s>>>(pot1, L_hat, grads, m, tab, inv_n);
  PMB_CUDA_CHECK(cudaGetLastError());
  return kOk;
}

int lpt_displace(const int16_t* pmid, float* disp, float* vel, int64_t n, Mesh3 g, float cell, float spacing,
                 const float* fields, int order, float D1, float V1, float D2, float V2, int64_t* index_out,
                 cudaStream_t s) {
  lpt_displace_kernel<float><<<grid_for(n, 256), 256, 0, s>>>(pmid, disp, vel, n, g, cell, spacing, fields, order, D1,
                                                               V1, D2, V2, index_out);
  PMB_CUDA_CHECK(cudaGetLastError());
  return kOk;
}

int lpt_strains64(const double2* modes, double inv_cell_vol, double2* pot1, double2* strains, Mesh3 m,
                  const double* tab, double inv_n, cudaStream_t s) {
  lpt_strain_kernel<double><<<grid_for(m.half_cells(), 256), 256, 0, s>>>(modes, inv_cell_vol, pot1, strains, m, tab,
                                                                          inv_n);
  PMB_CUDA_CHECK(cudaGetLastError());
  return kOk;
}

int lpt_source64(const double* s6, double* L, int64_t n, cudaStream_t s) {
  lpt_source_kernel<double><<<grid_for(n, 256), 256, 0, s>>>(s6, L, n);
  PMB_CUDA_CHECK(cudaGetLastError());
  return kOk;
}

int lpt_gradients64(const double2* pot1, const double2* L_hat, double2* grads, Mesh3 m, const double* tab,
                    double inv_n, cudaStream_t s) {
  lpt_gradient_kernel<double><<<grid_for(m.half_cells(), 256), 256, 0, s>>>(pot1, L_hat, grads, m, tab, inv_n);
  PMB_CUDA_CHECK(cudaGetLastError());
  return kOk;
}

int lpt_displace64(const int16_t* pmid, double* disp, double* vel, int64_t n, Mesh3 g, double cell, double spacing,
                   const double* fields, int order, double D1, double V1, double D2, double V2, int64_t* index_out,
                   cudaStream_t s) {
  lpt_displace_kernel<double><<<grid_for(n, 256), 256, 0, s>>>(pmid, disp, vel, n, g, cell, spacing, fields, order,
                                                                D1, V1, D2, V2, index_out);
  PMB_CUDA_CHECK(cudaGetLastError());
  return kOk;
}

// ---------------------------------------------------------------------------
// 2LPT adjoint
// ---------------------------------------------------------------------------
// Field cotangents from particle cotangents (transpose of the sampling):
// cot[m][d][idx_p] += D_m disp_cot[p,d] + V_m vel_cot[p,d], plus the FP64 dots
// sum_p g_m[d](idx_p) * disp_cot / vel_cot for the growth-factor cotangents.
template <class T>
__global__ void lpt_field_cot_kernel(const int64_t* __restrict__ index, const T* __restrict__ disp_cot,
                                     const T* __restrict__ vel_cot, int64_t n, int64_t ng,
                                     const T* __restrict__ fields, int order, T D1, T V1, T D2, T V2,
                                     T* __restrict__ cot, double* __restrict__ dots) {
  using R = Real<T>;
  double acc[4] = {0, 0, 0, 0};
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (int64_t)gridDim.x * blockDim.x) {
    const int64_t idx = index[p];
    const T Ds[2] = {D1, D2}, Vs[2] = {V1, V2};
    for (int mo = 0; mo < order; ++mo) {
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        const T dc = disp_cot[3 * p + d], vc = vel_cot[3 * p + d];
        atomicAdd(&cot[(int64_t)(3 * mo + d) * ng + idx], R::add(R::mul(Ds[mo], dc), R::mul(Vs[mo], vc)));
        const T gv = fields[(int64_t)(3 * mo + d) * ng + idx];
        acc[2 * mo] += (double)gv * dc;
        acc[2 * mo + 1] += (double)gv * vc;
      }
    }
  }
  for (int k = 0; k < 4; ++k) {
    double v = acc[k];
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(&dots[k], v);
  }
}

// L_hat_cot = G * sum_d (-i c_d) F2_d  (times post), the transpose of the
// second-order gradient stage; F2 = rFFT of the order-2 field cotangents.
template <class T>
__global__ void lpt_grad2_adjoint_kernel(const typename Real<T>::T2* __restrict__ F2,
                                         typename Real<T>::T2* __restrict__ out, Mesh3 m, const T* __restrict__ tab,
                                         T post) {
  using R = Real<T>;
  const LptTables<T> t = lpt_tables(tab, m);
  const int64_t total = m.half_cells();
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < total; j += (int64_t)gridDim.x * blockDim.x) {
    const Idx3 q = unravel_half(j, m);
    const T c[3] = {t.cx[q.ix], t.cy[q.iy], t.cz[q.iz]};
    T ar = 0, ai = 0;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const typename Real<T>::T2 a = F2[(int64_t)d * total + j];
      ar = R::add(ar, R::mul(c[d], a.y));
      ai = R::sub(ai, R::mul(c[d], a.x));
    }
    const typename Real<T>::T2 p = pot_from<T>(R::make2(ar, ai), k2_at(t, q));
    out[j] = R::make2(R::mul(p.x, post), R::mul(p.y, post));
  }
}

// Cotangents of the six strains given the source cotangent L_cot:
// d_i: L_cot * sum_{j != i} d_j;  s_ij: -2 L_cot s_ij.
template <class T>
__global__ void lpt_source_adjoint_kernel(const T* __restrict__ s6, const T* __restrict__ Lc, T* __restrict__ c6,
                                          int64_t n) {
  using R = Real<T>;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const T d0 = s6[i], d1 = s6[n + i], d2 = s6[2 * n + i];
    const T l = Lc[i];
    c6[i] = R::mul(l, R::add(d1, d2));
    c6[n + i] = R::mul(l, R::add(d0, d2));
    c6[2 * n + i] = R::mul(l, R::add(d0, d1));
#pragma unroll
    for (int s = 3; s < 6; ++s) c6[(int64_t)s * n + i] = R::mul(R::mul((T)-2, l), s6[(int64_t)s * n + i]);
  }
}

// modes_cot = G/V_cell * mult/N * [sum_d (-i c_d) F1_d + sum_s (-k_i k_j)_s FS_s]
// (the packed d/dRe + i d/dIm convention), optionally times the linear-mode
// amplitude; FS = rFFT of the strain cotangents.
template <class T>
__global__ void lpt_modes_adjoint_kernel(const typename Real<T>::T2* __restrict__ F1,
                                         const typename Real<T>::T2* __restrict__ FS, const T* __restrict__ amp,
                                         typename Real<T>::T2* __restrict__ out, Mesh3 m, const T* __restrict__ tab,
                                         T scale) {
  using R = Real<T>;
  const LptTables<T> t = lpt_tables(tab, m);
  const int64_t total = m.half_cells();
  const int nzh = m.nz / 2 + 1;
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < total; j += (int64_t)gridDim.x * blockDim.x) {
    const Idx3 q = unravel_half(j, m);
    const T c[3] = {t.cx[q.ix], t.cy[q.iy], t.cz[q.iz]};
    const T k[3] = {t.kx[q.ix], t.ky[q.iy], t.kz[q.iz]};
    const T kz0[3] = {-c[0], -c[1], -c[2]};
    T ar = 0, ai = 0;
    if (F1 != nullptr) {
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        const typename Real<T>::T2 a = F1[(int64_t)d * total + j];
        ar = R::add(ar, R::mul(c[d], a.y));
        ai = R::sub(ai, R::mul(c[d], a.x));
      }
    }
    if (FS != nullptr) {
      const int pi[6] = {0, 1, 2, 0, 0, 1}, pj[6] = {0, 1, 2, 1, 2, 2};
#pragma unroll
      for (int s = 0; s < 6; ++s) {
        const T ki = s < 3 ? k[pi[s]] : kz0[pi[s]];
        const T kj = s < 3 ? k[pj[s]] : kz0[pj[s]];
        const T f = R::mul(-ki, kj);
        const typename Real<T>::T2 a = FS[(int64_t)s * total + j];
        ar = R::add(ar, R::mul(f, a.x));
        ai = R::add(ai, R::mul(f, a.y));
      }
    }
    const T mult = (q.iz == 0 || ((m.nz % 2 == 0) && q.iz == nzh - 1)) ? (T)1 : (T)2;
    typename Real<T>::T2 p = pot_from<T>(R::make2(ar, ai), k2_at(t, q));
    T f = R::mul(scale, mult);
    if (amp != nullptr) f = R::mul(f, amp[j]);
    out[j] = R::make2(R::mul(p.x, f), R::mul(p.y, f));
  }
}

int lpt_field_cot(const int64_t* index, const float* disp_cot, const float* vel_cot, int64_t n, int64_t ng,
                  const float* fields, int order, float D1, float V1, float D2, float V2, float* cot, double* dots,
                  cudaStream_t s) {
  lpt_field_cot_kernel<float><<<grid_for(n, 256), 256, 0, s>>>(index, disp_cot, vel_cot, n, ng, fields, order, D1, V1, D2,
                                                         V2, cot, dots);
  PMB_CUDA_CHECK(cudaGetLastError());
  return kOk;
}

int lpt_grad2_adjoint(const float2* F2, float2* out, Mesh3 m, const float* tab, float post, cudaStream_t s) {
  lpt_grad2_adjoint_kernel<float><<<grid_for(m.half_cells(), 256), 256, 0, s>>>(F2, out, m, tab, post);
  PMB_CUDA_CHECK(cudaGetLastError());
  return kOk;
}

int lpt_source_adjoint(const float* s6, const float* Lc, float* c6, int64_t n, cudaStream_t s) {
  lpt_source_adjoint_kernel<float><<<grid_for(n, 256), 256, 0, s>>>(s6, Lc, c6, n);
  PMB_CUDA_CHECK(cudaGetLastError());
  return kOk;
}

int lpt_modes_adjoint(const float2* F1, const float2* FS, const float* amp, float2* out, Mesh3 m, const float* tab,
                      float scale, cudaStream_t s) {
  lpt_modes_adjoint_kernel<float><<<grid_for(m.half_cells(), 256), 256, 0, s>>>(F1, FS, amp, out, m, tab, scale);
  PMB_CUDA_CHECK(cudaGetLastError());
  return kOk;
}

int lpt_field_cot64(const int64_t* index, const double* disp_cot, const double* vel_cot, int64_t n, int64_t ng,
                    const double* fields, int order, double D1, double V1, double D2, double V2, double* cot,
                    double* dots, cudaStream_t s) {
  lpt_field_cot_kernel<double><<<grid_for(n, 256), 256, 0, s>>>(index, disp_cot, vel_cot, n, ng, fields, order, D1, V1,
                                                                 D2, V2, cot, dots);
  PMB_CUDA_CHECK(cudaGetLastError());
  return kOk;
}

int lpt_grad2_adjoint64(const double2* F2, double2* out, Mesh3 m, const double* tab, double post, cudaStream_t s) {
  lpt_grad2_adjoint_kernel<double><<<grid_for(m.half_cells(), 256), 256, 0, s>>>(F2, out, m, tab, post);
  PMB_CUDA_CHECK(cudaGetLastError());
  return kOk;
}

int lpt_source_adjoint64(const double* s6, const double* Lc, double* c6, int64_t n, cudaStream_t s) {
  lpt_source_adjoint_kernel<double><<<grid_for(n, 256), 256, 0, s>>>(s6, Lc, c6, n);
  PMB_CUDA_CHECK(cudaGetLastError());
  return kOk;
}

int lpt_modes_adjoint64(const double2* F1, const double2* FS, const double* amp, double2* out, Mesh3 m,
                        const double* tab, double scale, cudaStream_t s) {
  lpt_modes_adjoint_kernel<double><<<grid_for(m.half_cells(), 256), 256, 0, s>>>(F1, FS, amp, out, m, tab, scale);
  PMB_CUDA_CHECK(cudaGetLastError());
  return kOk;
}

// ---------------------------------------------------------------------------
// Power spectrum shells (power_spectrum.py:120-143)
// ---------------------------------------------------------------------------
// shell = floor(sqrt(n^2) + 1e-9) clipped, weight = |d|^2 * W^-2p * mult in
// float (W = product of per-axis sinc(n/M) tables), summed in FP64.
template <class T>
__global__ void pk_shells_kernel(const typename Real<T>::T2* __restrict__ spec, Mesh3 m, const T* __restrict__ sinc_tab,
                                 int mas_power, int num_shells, double* __restrict__ sums,
                                 const typename Real<T>::T2* __restrict__ spec_b, double* __restrict__ sums_b,
                                 double* __restrict__ sums_x) {
  using R = Real<T>;
  extern __shared__ double sh[];
  double* shA = sh;
  double* shB = sh + num_shells;
  double* shX = sh + 2 * num_shells;
  const bool cross = spec_b != nullptr;
  const int nsh = cross ? 3 * num_shells : num_shells;
  for (int t = threadIdx.x; t < nsh; t += blockDim.x) sh[t] = 0.0;
  __syncthreads();
  const T* sx = sinc_tab;
  const T* sy = sx + m.nx;
  const T* sz = sy + m.ny;
  const int64_t total = m.half_cells();
  const int nzh = m.nz / 2 + 1;
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < total; j += (int64_t)gridDim.x * blockDim.x) {
    const Idx3 q = unravel_half(j, m);
    const long long mx = fft_mode(q.ix, m.nx), my = fft_mode(q.iy, m.ny), mz = q.iz;
    const long long n2 = mx * mx + my * my + mz * mz;
    int shell = (int)floor(sqrt((double)n2) + 1e-9);
    if (shell > num_shells - 1) shell = num_shells - 1;
    const T mult = (q.iz == 0 || ((m.nz % 2 == 0) && q.iz == nzh - 1)) ? (T)1 : (T)2;
    T deconv = (T)1;
    if (mas_power > 0) {
      const T w = R::mul(R::mul(sx[q.ix], sy[q.iy]), sz[q.iz]);
      deconv = R::pow_(w, (T)(-2 * mas_power));
    }
    const typename R::T2 a = spec[j];
    const T pa = R::add(R::mul(a.x, a.x), R::mul(a.y, a.y));
    atomicAdd(&shA[shell], (double)R::mul(R::mul(pa, deconv), mult));
    if (cross) {
      const typename R::T2 b = spec_b[j];
      const T pb = R::add(R::mul(b.x, b.x), R::mul(b.y, b.y));
      const T px = R::add(R::mul(a.x, b.x), R::mul(a.y, b.y));
      atomicAdd(&shB[shell], (double)R::mul(R::mul(pb, deconv), mult));
      atomicAdd(&shX[shell], (double)R::mul(R::mul(px, deconv), mult));
    }
  }
  __syncthreads();
  for (int t = threadIdx.x; t < num_shells; t += blockDim.x) {
    if (shA[t] != 0.0) atomicAdd(&sums[t], shA[t]);
    if (cross) {
      if (shB[t] != 0.0) atomicAdd(&sums_b[t], shB[t]);
      if (shX[t] != 0.0) atomicAdd(&sums_x[t], shX[t]);
    }
  }
}

int pk_shells(const float2* spec, Mesh3 m, const float* sinc_tab, int mas_power, int num_shells, double* sums,
              const float2* spec_b, double* sums_b, double* sums_x, cudaStream_t s) {
  const int nsh = spec_b != nullptr ? 3 * num_shells : num_shells;
  const size_t smem = sizeof(double) * nsh;
  if (smem > 200 * 1024) return kUnsupported;
  PMB_CUDA_CHECK(smem_optin((const void*)pk_shells_kernel<float>, 200 * 1024));
  int64_t b = (m.half_cells() + 255) / 256;
  if (b > 148 * 8) b = 148 * 8;
  pk_shells_kernel<float><<<(unsigned)(b > 0 ? b : 1), 256, smem, s>>>(spec, m, sinc_tab, mas_power, num_shells, sums,
                                                                       spec_b, sums_b, sums_x);
  PMB_CUDA_CHECK(cudaGetLastError());
  return kOk;
}

int pk_shells64(const double2* spec, Mesh3 m, const double* sinc_tab, int mas_power, int num_shells, double* sums,
                cudaStream_t s) {
  const size_t smem = sizeof(double) * num_shells;
  if (smem > 200 * 1024) return kUnsupported;
  PMB_CUDA_CHECK(smem_optin((const void*)pk_shells_kernel<double>, 200 * 1024));
  int64_t b = (m.half_cells() + 255) / 256;
  if (b > 148 * 8) b = 148 * 8;
  pk_shells_kernel<double><<<(unsigned)(b > 0 ? b : 1), 256, smem, s>>>(spec, m, sinc_tab, mas_power, num_shells,
                                                                        sums, nullptr, nullptr, nullptr);
  PMB_CUDA_CHECK(cudaGetLastError());
  return kOk;
}

// Adjoint of the shell power: given dL/dP_shell (already divided by nmodes and
// times the normalisation), out = 2 * spec * deconv * w_shell * (1/mult) so
// that M * irfftn(out) is the real-field cotangent (rfftn^T for the
// Hermitian-consistent spectrum).
// T = double: the float64 build's form, with the same operations in double.
template <class T>
__global__ void pk_shells_adjoint_kernel(const typename Real<T>::T2* __restrict__ spec, Mesh3 m,
                                         const T* __restrict__ sinc_tab, int mas_power, int num_shells,
                                         const double* __restrict__ wshell, T post,
                                         typename Real<T>::T2* __restrict__ out) {
  using R = Real<T>;
  const T* sx = sinc_tab;
  const T* sy = sx + m.nx;
  const T* sz = sy + m.ny;
  const int64_t total = m.half_cells();
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < total; j += (int64_t)gridDim.x * blockDim.x) {
    const Idx3 q = unravel_half(j, m);
    const long long mx = fft_mode(q.ix, m.nx), my = fft_mode(q.iy, m.ny), mz = q.iz;
    const long long n2 = mx * mx + my * my + mz * mz;
    int shell = (int)floor(sqrt((double)n2) + 1e-9);
    if (shell > num_shells - 1) shell = num_shells - 1;
    T deconv = (T)1;
    if (mas_power > 0) {
      const T w = R::mul(R::mul(sx[q.ix], sy[q.iy]), sz[q.iz]);
      deconv = R::pow_(w, (T)(-2 * mas_power));
    }
    // the multiplicity cancels against the 1/mult of the rFFT transpose
    const T f = R::mul(R::mul((T)2 * (T)wshell[shell], deconv), post);
    const typename R::T2 a = spec[j];
    out[j] = R::make2(R::mul(a.x, f), R::mul(a.y, f));
  }
}

int pk_shells_adjoint(const float2* spec, Mesh3 m, const float* sinc_tab, int mas_power, int num_shells,
                      const double* wshell, float post, float2* out, cudaStream_t s) {
  pk_shells_adjoint_kernel<float><<<grid_for(m.half_cells(), 256), 256, 0, s>>>(spec, m, sinc_tab, mas_power,
                                                                                num_shells, wshell, post, out);
  PMB_CUDA_CHECK(cudaGetLastError());
  return kOk;
}

int pk_shells_adjoint64(const double2* spec, Mesh3 m, const double* sinc_tab, int mas_power, int num_shells,
                        const double* wshell, double post, double2* out, cudaStream_t s) {
  pk_shells_adjoint_kernel<double><<<grid_for(m.half_cells(), 256), 256, 0, s>>>(spec, m, sinc_tab, mas_power,
                                                                                 num_shells, wshell, post, out);
  PMB_CUDA_CHECK(cudaGetLastError());
  return kOk;
}

// Shell mode counts and mean |n| (power_spectrum.py:46-74), FP64.
__global__ void shell_stats_kernel(Mesh3 m, int num_shells, double* __restrict__ counts, double* __restrict__ ksum) {
  extern __shared__ double sh[];
  for (int t = threadIdx.x; t < 2 * num_shells; t += blockDim.x) sh[t] = 0.0;
  __syncthreads();
  const int64_t total = m.half_cells();
  const int nzh = m.nz / 2 + 1;
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < total; j += (int64_t)gridDim.x * blockDim.x) {
    const Idx3 q = unravel_half(j, m);
    const long long mx = fft_mode(q.ix, m.nx), my = fft_mode(q.iy, m.ny), mz = q.iz;
    const double mag = sqrt((double)(mx * mx + my * my + mz * mz));
    int shell = (int)floor(mag + 1e-6);
    if (shell > num_shells - 1) shell = num_shells - 1;
    const double mult = (q.iz == 0 || ((m.nz % 2 == 0) && q.iz == nzh - 1)) ? 1.0 : 2.0;
    atomicAdd(&sh[shell], mult);
    atomicAdd(&sh[num_shells + shell], mag * mult);
  }
  __syncthreads();
  for (int t = threadIdx.x; t < num_shells; t += blockDim.x) {
    if (sh[t] != 0.0) atomicAdd(&counts[t], sh[t]);
    if (sh[num_shells + t] != 0.0) atomicAdd(&ksum[t], sh[num_shells + t]);
  }
}

int shell_stats(Mesh3 m, int num_shells, double* counts, double* ksum, cudaStream_t s) {
  const size_t smem = sizeof(double) * 2 * num_shells;
  if (smem > 200 * 1024) return kUnsupported;
  PMB_CUDA_CHECK(smem_optin((const void*)shell_stats_kernel, 200 * 1024));
  int64_t b = (m.half_cells() + 255) / 256;
  if (b > 148 * 8) b = 148 * 8;
  shell_stats_kernel<<<(unsigned)(b > 0 ? b : 1), 256, smem, s>>>(m, num_shells, counts, ksum);
  PMB_CUDA_CHECK(cudaGetLastError());
  return kOk;
}

// delta = rho / mean - 1 (power_spectrum.py:371-374), mean from an FP64 sum.
template <class T>
__global__ void overdensity_kernel(const T* __restrict__ rho, T* __restrict__ delta, int64_t n,
                                   const double* __restrict__ total) {
  using R = Real<T>;
  const T mean = (T)(*total / (double)n);
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    delta[i] = R::sub(R::div(rho[i], mean), (T)1);
}

int overdensity(const float* rho, float* delta, int64_t n, const double* total, cudaStream_t s) {
  overdensity_kernel<float><<<grid_for(n, 256), 256, 0, s>>>(rho, delta, n, total);
  PMB_CUDA_CHECK(cudaGetLastError());
  return kOk;
}

int overdensity64(const double* rho, double* delta, int64_t n, const double* total, cudaStream_t s) {
  overdensity_kernel<double><<<grid_for(n, 256), 256, 0, s>>>(rho, delta, n, total);
  PMB_CUDA_CHECK(cudaGetLastError());
  return kOk;
}

}  // namespace pmb
