// Spectral stages of the PM force: cuFFT R2C/C2R plans with caller-provided
// work areas, the fused Green's-function x gradient multiplier and its
// adjoint, and the FP64 power-spectrum shell sums.
//
// Reference semantics: nbody/gravity.py:174-196 (particle-Nyquist masks),
// :283-352 (continuum and discrete-Laplacian Poisson kernels), :355-391 and
// core/configuration.py:365-376 (spectral gradient with the Nyquist
// derivative zeroed), corrections/core.py:333-334 (multiplicative transfer),
// analysis/power_spectrum.py:106-143 (shell sums).
#include <cufft.h>

#include <cmath>
#include <map>
#include <mutex>
#include <tuple>

#include "pmb_common.cuh"
#include "pmb_kernels.cuh"
#include "pmb_spectral_device.cuh"

namespace pmb {

// ---------------------------------------------------------------------------
// cuFFT plan cache.  Plans are created once per (device, shape, batch, kind)
// without auto-allocation; every execution binds the caller's work area, so
// the library never allocates device memory per call.
// ---------------------------------------------------------------------------
namespace {
struct PlanKey {
  int dev, nx, ny, nz, batch, kind;
  bool operator<(const PlanKey& o) const {
    return std::tie(dev, nx, ny, nz, batch, kind) < std::tie(o.dev, o.nx, o.ny, o.nz, o.batch, o.kind);
  }
};
struct PlanVal {
  cufftHandle h;
  size_t work;
};
std::mutex g_plan_mu;
std::map<PlanKey, PlanVal>& plans() {
  static std::map<PlanKey, PlanVal> p;
  return p;
}

int get_plan(Mesh3 m, int batch, int kind, PlanVal* out) {
  int dev = 0;
  PMB_CUDA_CHECK(cudaGetDevice(&dev));
  PlanKey key{dev, m.nx, m.ny, m.nz, batch, kind};
  std::lock_guard<std::mutex> lk(g_plan_mu);
  auto it = plans().find(key);
  if (it != plans().end()) {
    *out = it->second;
    return kOk;
  }
  cufftHandle h;
  if (cufftCreate(&h) != CUFFT_SUCCESS) {
    set_last_error("cufftCreate failed");
    return kCufftError;
  }
  cufftSetAutoAllocation(h, 0);
  long long n[3] = {m.nx, m.ny, m.nz};
  long long rdist = (long long)m.cells();
  long long cdist = (long long)m.half_cells();
  size_t work = 0;
  cufftResult r;
  // kind 0 R2C, 1 C2R (float32); 2 D2Z, 3 Z2D (float64)
  if (kind == 0 || kind == 2) {
    r = cufftMakePlanMany64(h, 3, n, nullptr, 1, rdist, nullptr, 1, cdist, kind == 0 ? CUFFT_R2C : CUFFT_D2Z, batch,
                            &work);
  } else {
    r = cufftMakePlanMany64(h, 3, n, nullptr, 1, cdist, nullptr, 1, rdist, kind == 1 ? CUFFT_C2R : CUFFT_Z2D, batch,
                            &work);
  }
  if (r != CUFFT_SUCCESS) {
    cufftDestroy(h);
    set_last_error("cufftMakePlanMany64 failed");
    return kCufftError;
  }
  PlanVal v{h, work};
  plans()[key] = v;
  *out = v;
  return kOk;
}
}  // namespace

static bool split_batches(Mesh3 m);

int64_t fft_work_bytes(Mesh3 m, int batch) {
  if (batch > 1 && split_batches(m)) batch = 1;
  PlanVal a, b;
  if (get_plan(m, batch, 0, &a) != kOk) return -1;
  if (get_plan(m, batch, 1, &b) != kOk) return -1;
  return (int64_t)(a.work > b.work ? a.work : b.work);
}

int64_t fft_work_bytes64(Mesh3 m, int batch) {
  PlanVal a, b;
  if (get_plan(m, batch, 2, &a) != kOk) return -1;
  if (get_plan(m, batch, 3, &b) != kOk) return -1;
  return (int64_t)(a.work > b.work ? a.work : b.work);
}

int fft_d2z(Mesh3 m, int batch, double* in, double2* out, void* work, cudaStream_t s) {
  PlanVal p;
  int st = get_plan(m, batch, 2, &p);
  if (st != kOk) return st;
  if (cufftSetStream(p.h, s) != CUFFT_SUCCESS || cufftSetWorkArea(p.h, work) != CUFFT_SUCCESS ||
      cufftExecD2Z(p.h, in, (cufftDoubleComplex*)out) != CUFFT_SUCCESS) {
    set_last_error("cufftExecD2Z failed");
    return kCufftError;
  }
  return kOk;
}

int fft_z2d(Mesh3 m, int batch, double2* in, double* out, void* work, cudaStream_t s) {
  PlanVal p;
  int st = get_plan(m, batch, 3, &p);
  if (st != kOk) return st;
  if (cufftSetStream(p.h, s) != CUFFT_SUCCESS || cufftSetWorkArea(p.h, work) != CUFFT_SUCCESS ||
      cufftExecZ2D(p.h, (cufftDoubleComplex*)in, out) != CUFFT_SUCCESS) {
    set_last_error("cufftExecZ2D failed");
    return kCufftError;
  }
  return kOk;
}

// Batched plans of very large meshes measured slower per transform than
// single transforms (1024^3 on B200: 7.0 ms vs 5.8 ms per R2C, 7.2 ms vs
// 6.0 ms per C2R), so batches of such meshes run one transform at a time.
static bool split_batches(Mesh3 m) { return m.cells() > ((int64_t)1 << 27); }

int fft_r2c(Mesh3 m, int batch, float* in, float2* out, void* work, cudaStream_t s) {
  if (batch > 1 && split_batches(m)) {
    for (int b = 0; b < batch; ++b) {
      const int st = fft_r2c(m, 1, in + (int64_t)b * m.cells(), out + (int64_t)b * m.half_cells(), work, s);
      if (st != kOk) return st;
    }
    return kOk;
  }
  PlanVal p;
  int st = get_plan(m, batch, 0, &p);
  if (st != kOk) return st;
  if (cufftSetStream(p.h, s) != CUFFT_SUCCESS || cufftSetWorkArea(p.h, work) != CUFFT_SUCCESS ||
      cufftExecR2C(p.h, in, (cufftComplex*)out) != CUFFT_SUCCESS) {
    set_last_error("cufftExecR2C failed");
    return kCufftError;
  }
  return kOk;
}

int fft_c2r(Mesh3 m, int batch, float2* in, float* out, void* work, cudaStream_t s) {
  if (batch > 1 && split_batches(m)) {
    for (int b = 0; b < batch; ++b) {
      const int st = fft_c2r(m, 1, in + (int64_t)b * m.half_cells(), out + (int64_t)b * m.cells(), work, s);
      if (st != kOk) return st;
    }
    return kOk;
  }
  PlanVal p;
  int st = get_plan(m, batch, 1, &p);
  if (st != kOk) return st;
  if (cufftSetStream(p.h, s) != CUFFT_SUCCESS || cufftSetWorkArea(p.h, work) != CUFFT_SUCCESS ||
      cufftExecC2R(p.h, (cufftComplex*)in, out) != CUFFT_SUCCESS) {
    set_last_error("cufftExecC2R failed");
    return kCufftError;
  }
  return kOk;
}

// ---------------------------------------------------------------------------
// Green's function x gradient
// ---------------------------------------------------------------------------
// Flat grid-stride loops over the half spectrum; the cell coordinates come
// from 32-bit index arithmetic (Index = uint32_t) whenever the spectrum has
// fewer than 2^31 cells (the loop index then cannot wrap), which keeps the
// multipliers memory-bound.
template <class Index>
__global__ void green_gradient_kernel(const float2* __restrict__ src, float2* __restrict__ grad, Mesh3 m,
                                      SpecTables t, GreenParams g) {
  const Index nzh = (Index)(m.nz / 2 + 1), ny = (Index)m.ny;
  const Index total = (Index)m.half_cells();
  for (Index j = (Index)blockIdx.x * blockDim.x + threadIdx.x; j < total; j += (Index)gridDim.x * blockDim.x) {
    const Index r = j / nzh;
    const Index ix = r / ny;
    green_gradient_at(src, grad, (int64_t)j, (int64_t)total, (int)ix, (int)(r - ix * ny), (int)(j - r * nzh), m, t,
                      g);
  }
}

template <class Index>
__global__ void green_gradient_adjoint_kernel(const float2* __restrict__ gc, float2* __restrict__ out, Mesh3 m,
                                              SpecTables t, GreenParams g) {
  const Index nzh = (Index)(m.nz / 2 + 1), ny = (Index)m.ny;
  const Index total = (Index)m.half_cells();
  for (Index j = (Index)blockIdx.x * blockDim.x + threadIdx.x; j < total; j += (Index)gridDim.x * blockDim.x) {
    const Index r = j / nzh;
    const Index ix = r / ny;
    green_gradient_adjoint_at(gc, out, (int64_t)j, (int64_t)total, (int)ix, (int)(r - ix * ny), (int)(j - r * nzh), m,
                              t, g);
  }
}

// Four consecutive cells per thread with 32-byte vector loads and stores;
// the cell coordinates are computed once per group and advanced in place.
// Needs total % 4 == 0 (and 16-byte aligned spectra, as the workspaces are).
__device__ __forceinline__ void advance_cell(int& ix, int& iy, int& iz, int nzh, int ny) {
  if (++iz == nzh) {
    iz = 0;
    if (++iy == ny) {
      iy = 0;
      ++ix;
    }
  }
}

__global__ void green_gradient_kernel4(const float2* __restrict__ src, float2* __restrict__ grad, Mesh3 m,
                                       SpecTables t, GreenParams g) {
  const uint32_t nzh = (uint32_t)(m.nz / 2 + 1), ny = (uint32_t)m.ny;
  const uint32_t total = (uint32_t)m.half_cells(), groups = total / 4;
  const float4* s4 = reinterpret_cast<const float4*>(src);
  for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < groups; q += gridDim.x * blockDim.x) {
    const uint32_t j = 4 * q, r = j / nzh, x = r / ny;
    int ix = (int)x, iy = (int)(r - x * ny), iz = (int)(j - r * nzh);
    const float4 a = s4[2 * q], b = s4[2 * q + 1];
    const float2 v[4] = {make_float2(a.x, a.y), make_float2(a.z, a.w), make_float2(b.x, b.y), make_float2(b.z, b.w)};
    float2 o[4][3];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      green_gradient_value(v[e], (int64_t)j + e, ix, iy, iz, m, t, g, o[e]);
      advance_cell(ix, iy, iz, (int)nzh, (int)ny);
    }
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      float4* g4 = reinterpret_cast<float4*>(grad + (int64_t)d * total);
      g4[2 * q] = make_float4(o[0][d].x, o[0][d].y, o[1][d].x, o[1][d].y);
      g4[2 * q + 1] = make_float4(o[2][d].x, o[2][d].y, o[3][d].x, o[3][d].y);
    }
  }
}

__global__ void green_gradient_adjoint_kernel4(const float2* __restrict__ gc, float2* __restrict__ out, Mesh3 m,
                                               SpecTables t, GreenParams g) {
  const uint32_t nzh = (uint32_t)(m.nz / 2 + 1), ny = (uint32_t)m.ny;
  const uint32_t total = (uint32_t)m.half_cells(), groups = total / 4;
  for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < groups; q += gridDim.x * blockDim.x) {
    const uint32_t j = 4 * q, r = j / nzh, x = r / ny;
    int ix = (int)x, iy = (int)(r - x * ny), iz = (int)(j - r * nzh);
    float2 a[3][4];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const float4* c4 = reinterpret_cast<const float4*>(gc + (int64_t)d * total);
      const float4 u = c4[2 * q], w = c4[2 * q + 1];
      a[d][0] = make_float2(u.x, u.y);
      a[d][1] = make_float2(u.z, u.w);
      a[d][2] = make_float2(w.x, w.y);
      a[d][3] = make_float2(w.z, w.w);
    }
    float2 o[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const float2 ae[3] = {a[0][e], a[1][e], a[2][e]};
      o[e] = green_gradient_adjoint_value(ae, (int64_t)j + e, ix, iy, iz, m, t, g);
      advance_cell(ix, iy, iz, (int)nzh, (int)ny);
    }
    float4* o4 = reinterpret_cast<float4*>(out);
    o4[2 * q] = make_float4(o[0].x, o[0].y, o[1].x, o[1].y);
    o4[2 * q + 1] = make_float4(o[2].x, o[2].y, o[3].x, o[3].y);
  }
}

// One gradient component d of the forward multiplier (the streamed force
// builds the components one at a time into a single spectrum).
__global__ void green_gradient_component_kernel(const float2* __restrict__ src, float2* __restrict__ out, Mesh3 m,
                                                SpecTables t, GreenParams g, int d) {
  const int64_t nzh = m.nz / 2 + 1, ny = m.ny;
  const int64_t total = m.half_cells();
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < total; j += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = j / nzh, ix = r / ny;
    float2 o[3];
    green_gradient_value(src[j], j, (int)ix, (int)(r - ix * ny), (int)(j - r * nzh), m, t, g, o);
    out[j] = o[d];
  }
}

// acc[3 i + d] = planar[d * n + i]
__global__ void interleave3_kernel(const float* __restrict__ planar, float* __restrict__ acc, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    acc[3 * i] = planar[i];
    acc[3 * i + 1] = planar[n + i];
    acc[3 * i + 2] = planar[2 * n + i];
  }
}

static bool vec4_ok(Mesh3 m, const void* a, const void* b) {
  return m.half_cells() % 4 == 0 && m.half_cells() < 2147483648ll && ((uintptr_t)a & 31) == 0 &&
         ((uintptr_t)b & 31) == 0;
}

static unsigned grid_for(int64_t total, int th) {
  int64_t b = (total + th - 1) / th;
  int64_t cap = 148 * 32;
  return (unsigned)(b < cap ? (b > 0 ? b : 1) : cap);
}

int green_gradient(const float2* src_hat, float2* grad_hat, Mesh3 m, SpecTables t, GreenParams g, cudaStream_t s) {
  const unsigned grid = grid_for(m.half_cells(), 256);
  if (vec4_ok(m, src_hat, grad_hat))
    green_gradient_kernel4<<<grid_for(m.half_cells() / 4, 256), 256, 0, s>>>(src_hat, grad_hat, m, t, g);
  else if (m.half_cells() < 2147483648ll)
    green_gradient_kernel<uint32_t><<<grid, 256, 0, s>>>(src_hat, grad_hat, m, t, g);
  else
    green_gradient_kernel<int64_t><<<grid, 256, 0, s>>>(src_hat, grad_hat, m, t, g);
  PMB_CUDA_CHECK(cudaGetLastError());
  return kOk;
}

int green_gradient_component(const float2* src_hat, float2* out, Mesh3 m, SpecTables t, GreenParams g, int d,
                             cudaStream_t s) {
  green_gradient_component_kernel<<<grid_for(m.half_cells(), 256), 256, 0, s>>>(src_hat, out, m, t, g, d);
  PMB_CUDA_CHECK(cudaGetLastError());
  return kOk;
}

int interleave3(const float* planar, float* acc, int64_t n, cudaStream_t s) {
  if (n > 0) interleave3_kernel<<<grid_for(n, 256), 256, 0, s>>>(planar, acc, n);
  PMB_CUDA_CHECK(cudaGetLastError());
  return kOk;
}

int green_gradient_adjoint(const float2* grad_cot_hat, float2* src_cot_hat, Mesh3 m, SpecTables t, GreenParams g,
                           cudaStream_t s) {
  const unsigned grid = grid_for(m.half_cells(), 256);
  if (vec4_ok(m, grad_cot_hat, src_cot_hat))
    green_gradient_adjoint_kernel4<<<grid_for(m.half_cells() / 4, 256), 256, 0, s>>>(grad_cot_hat, src_cot_hat, m, t,
                                                                                    g);
  else if (m.half_cells() < 2147483648ll)
    green_gradient_adjoint_kernel<uint32_t><<<grid, 256, 0, s>>>(grad_cot_hat, src_cot_hat, m, t, g);
  else
    green_gradient_adjoint_kernel<int64_t><<<grid, 256, 0, s>>>(grad_cot_hat, src_cot_hat, m, t, g);
  PMB_CUDA_CHECK(cudaGetLastError());
  return kOk;
}

// Interlaced assignment (nbody/gravity.py:440-463).  The deposit shifted by
// half a cell on every axis has the spectrum of the regular one times
// exp(+i (kx + ky + kz) h / 2); P = exp(-i (kx + ky + kz) h / 2) moves it
// back.  With k_d h / 2 = pi s_d / n_d over the signed frequency s_d (x and y
// as fftfreq, the Nyquist index negative; z >= 0 as rfftfreq) the phase is
// exp(-i pi t), t = sx / nx + sy / ny + sz / nz, taken with sincospif.
//   mode 0 (forward):   s0 = (s0 + P s1) / 2
//   mode 1 (transpose): s1 = conj(P) s0 / 2, then s0 = s0 / 2
__global__ void interlace_kernel(float2* __restrict__ s0, float2* __restrict__ s1, Mesh3 m, int mode) {
  const int64_t nzh = m.nz / 2 + 1, ny = m.ny;
  const int64_t total = m.half_cells();
  const float inx = 1.0f / (float)m.nx, iny = 1.0f / (float)m.ny, inz = 1.0f / (float)m.nz;
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < total; j += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = j / nzh, ix = r / ny;
    const int iy = (int)(r - ix * ny), iz = (int)(j - r * nzh);
    const int sx = (2 * ix >= m.nx) ? (int)ix - m.nx : (int)ix;
    const int sy = (2 * iy >= m.ny) ? iy - m.ny : iy;
    const float t = (float)sx * inx + (float)sy * iny + (float)iz * inz;
    float sn, cs;
    sincospif(t, &sn, &cs);  // P = cs - i sn
    const float2 a = s0[j];
    if (mode == 0) {
      const float2 b = s1[j];
      s0[j] = make_float2(0.5f * (a.x + (cs * b.x + sn * b.y)), 0.5f * (a.y + (cs * b.y - sn * b.x)));
    } else {
      s1[j] = make_float2(0.5f * (cs * a.x - sn * a.y), 0.5f * (cs * a.y + sn * a.x));
      s0[j] = make_float2(0.5f * a.x, 0.5f * a.y);
    }
  }
}

int interlace(float2* s0, float2* s1, Mesh3 m, int mode, cudaStream_t s) {
  interlace_kernel<<<grid_for(m.half_cells(), 256), 256, 0, s>>>(s0, s1, m, mode);
  PMB_CUDA_CHECK(cudaGetLastError());
  return kOk;
}

// Stages of a force with a real-space residual potential (the mesh-CNN
// correction, corrections/core.py:321-331): the potential spectrum alone,
// the gradients of a potential plus a residual spectrum, and the transpose
// of the gradient without the Green's function.
//   P = K(k) S_hat * post                      (pmb_green_potential)
//   grad_d = (i c_d) (P + q_scale Q) * post    (pmb_gradient_spectra)
//   out = sum_d conj(i c_d) A_d * post         (pmb_gradient_adjoint_plain)
__global__ void green_potential_kernel(const float2* __restrict__ src, float2* __restrict__ out, Mesh3 m,
                                       SpecTables t, GreenParams g) {
  const int64_t nzh = m.nz / 2 + 1, ny = m.ny;
  const int64_t total = m.half_cells();
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < total; j += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = j / nzh, ix = r / ny;
    const int iy = (int)(r - ix * ny), iz = (int)(j - r * nzh);
    float2 v = src[j];
    if (t.mx != nullptr) {
      const float mk = __fmul_rn(__fmul_rn(t.mx[ix], t.my[iy]), t.mz[iz]);
      v.x = __fmul_rn(v.x, mk);
      v.y = __fmul_rn(v.y, mk);
    }
    const float k2 = k2_of(t, (int)ix, iy, iz);
    float pr = 0.f, pi = 0.f;
    if (k2 != 0.f) {
      pr = __fdiv_rn(-v.x, k2);
      pi = __fdiv_rn(-v.y, k2);
      if (g.transfer != nullptr || g.radial != nullptr) {
        const float T = transfer_of(g, t, j, (int)ix, iy, iz, m);
        pr = __fmul_rn(pr, T);
        pi = __fmul_rn(pi, T);
      }
    }
    out[j] = make_float2(__fmul_rn(pr, g.post_scale), __fmul_rn(pi, g.post_scale));
  }
}

__global__ void gradient_spectra_kernel(const float2* __restrict__ P, const float2* __restrict__ Q, float q_scale,
                                        float2* __restrict__ grad, Mesh3 m, SpecTables t, float post) {
  const int64_t nzh = m.nz / 2 + 1, ny = m.ny;
  const int64_t total = m.half_cells();
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < total; j += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = j / nzh, ix = r / ny;
    const int iy = (int)(r - ix * ny), iz = (int)(j - r * nzh);
    float2 v = P[j];
    if (Q != nullptr) {
      const float2 q = Q[j];
      v.x = __fadd_rn(v.x, __fmul_rn(q_scale, q.x));
      v.y = __fadd_rn(v.y, __fmul_rn(q_scale, q.y));
    }
    const float c[3] = {t.cx[ix], t.cy[iy], t.cz[iz]};
#pragma unroll
    for (int d = 0; d < 3; ++d)
      grad[(int64_t)d * total + j] = make_float2(__fmul_rn(-__fmul_rn(c[d], v.y), post), __fmul_rn(__fmul_rn(c[d], v.x), post));
  }
}

__global__ void gradient_adjoint_plain_kernel(const float2* __restrict__ A, float2* __restrict__ out, Mesh3 m,
                                              SpecTables t, float post) {
  const int64_t nzh = m.nz / 2 + 1, ny = m.ny;
  const int64_t total = m.half_cells();
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < total; j += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = j / nzh, ix = r / ny;
    const int iy = (int)(r - ix * ny), iz = (int)(j - r * nzh);
    const float c[3] = {t.cx[ix], t.cy[iy], t.cz[iz]};
    float sr = 0.f, si = 0.f;  // sum_d (-i c_d) A_d
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const float2 a = A[(int64_t)d * total + j];
      sr = __fadd_rn(sr, __fmul_rn(c[d], a.y));
      si = __fsub_rn(si, __fmul_rn(c[d], a.x));
    }
    out[j] = make_float2(__fmul_rn(sr, post), __fmul_rn(si, post));
  }
}

int green_potential(const float2* src, float2* out, Mesh3 m, SpecTables t, GreenParams g, cudaStream_t s) {
  green_potential_kernel<<<grid_for(m.half_cells(), 256), 256, 0, s>>>(src, out, m, t, g);
  PMB_CUDA_CHECK(cudaGetLastError());
  return kOk;
}

int gradient_spectra(const float2* P, const float2* Q, float q_scale, float2* grad, Mesh3 m, SpecTables t, float post,
                     cudaStream_t s) {
  gradient_spectra_kernel<<<grid_for(m.half_cells(), 256), 256, 0, s>>>(P, Q, q_scale, grad, m, t, post);
  PMB_CUDA_CHECK(cudaGetLastError());
  return kOk;
}

int gradient_adjoint_plain(const float2* A, float2* out, Mesh3 m, SpecTables t, float post, cudaStream_t s) {
  gradient_adjoint_plain_kernel<<<grid_for(m.half_cells(), 256), 256, 0, s>>>(A, out, m, t, post);
  PMB_CUDA_CHECK(cudaGetLastError());
  return kOk;
}

// x = x * a + b, elementwise in float.
__global__ void scale_real_kernel(float* __restrict__ x, int64_t n, float a, float b) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    x[i] = __fadd_rn(__fmul_rn(x[i], a), b);
}

int scale_real(float* x, int64_t count, float a, float b, cudaStream_t s) {
  scale_real_kernel<<<grid_for(count, 256), 256, 0, s>>>(x, count, a, b);
  PMB_CUDA_CHECK(cudaGetLastError());
  return kOk;
}

}  // namespace pmb
