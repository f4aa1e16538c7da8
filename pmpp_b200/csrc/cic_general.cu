// CIC on a mesh whose cell size differs from the particles' (the explicit
// cell_size argument of cic/scatter.py:235 and cic/gather.py:414).
//
// Reference semantics: the explicit-cell branch of the Pallas coordinate
// helper (cic/pallas.py:192-222) and of enmesh (cic/enmesh.py:108-127).  Per
// axis, in float: position p = mod((pmid * a1 + disp) - offset, L * a1) on
// the particles' periodic box (L cells of size a1); for corner bit b the
// mesh index is i_b = floor(mod(p + b * a2, L * a1) / a2) and the offset
// d_b = p - i_b * a2, folded into (-L a1 / 2, L a1 / 2]; the weight is
// 1 - |d_b / a2| and its gradient sign(-d_b / a2) times the other two axes'
// weights, divided by a2.  Corners outside the target mesh (0 <= i < shape)
// are dropped.  Particles with valid[p] == 0 deposit nothing, gather 0 and
// get zero cotangents (cic/pallas.py:133-141).
//
// This path resamples onto arbitrary grids, so it works per particle without
// the cell sort: the deposit accumulates exact 64-bit fixed-point sums with
// global integer atomics (order-independent, hence deterministic) and a
// second kernel converts them to float.  The PM force never takes it.
#include "pmb_cic_device.cuh"
#include "pmb_common.cuh"
#include "pmb_integrate.cuh"
#include "pmb_kernels.cuh"

namespace pmb {

// floored float modulus, exact (fmod is exact; the sign fix adds y once)
__device__ __forceinline__ float fmod_floor(float x, float y) {
  float r = fmodf(x, y);
  if (r != 0.f && ((r < 0.f) != (y < 0.f))) r = __fadd_rn(r, y);
  return r;
}

struct GeneralCorners {
  int64_t idx[8];  // raveled target index, -1 when the corner is dropped
  float w[8];
  float g[8][3];   // weight gradient before the division by a2
};

__device__ __forceinline__ void general_axis(int pm, float d, float a1, float a2, int L, float o, int shape,
                                             int idx[2], float w[2], float sg[2]) {
  const float period = __fmul_rn((float)L, a1);
  float p = __fsub_rn(__fadd_rn(__fmul_rn((float)pm, a1), d), o);
  p = fmod_floor(p, period);
#pragma unroll
  for (int b = 0; b < 2; ++b) {
    const float np = fmod_floor(__fadd_rn(p, b ? a2 : 0.f), period);
    const int i = (int)floorf(__fdiv_rn(np, a2));
    float delta = __fsub_rn(p, __fmul_rn((float)i, a2));
    const float half = __fmul_rn(0.5f, period);
    if (delta > half) delta = __fsub_rn(delta, period);
    if (delta < -half) delta = __fadd_rn(delta, period);
    const float q = __fdiv_rn(delta, a2);
    w[b] = __fsub_rn(1.0f, fabsf(q));
    sg[b] = q < 0.f ? 1.0f : (q > 0.f ? -1.0f : 0.0f);
    idx[b] = (i >= 0 && i < shape) ? i : -1;
  }
}

__device__ __forceinline__ void general_corners(const int16_t* __restrict__ pmid, const float* __restrict__ disp,
                                                int64_t p, const GeneralGrid& G, GeneralCorners& k) {
  int ix[2], iy[2], iz[2];
  float wx[2], wy[2], wz[2], sx[2], sy[2], sz[2];
  general_axis(pmid[3 * p + 0], disp[3 * p + 0], G.a1, G.a2, G.gx, G.ox, G.t.nx, ix, wx, sx);
  general_axis(pmid[3 * p + 1], disp[3 * p + 1], G.a1, G.a2, G.gy, G.oy, G.t.ny, iy, wy, sy);
  general_axis(pmid[3 * p + 2], disp[3 * p + 2], G.a1, G.a2, G.gz, G.oz, G.t.nz, iz, wz, sz);
#pragma unroll
  for (int c = 0; c < 8; ++c) {
    const int bx = c & 1, by = (c >> 1) & 1, bz = (c >> 2) & 1;
    const bool ok = ix[bx] >= 0 && iy[by] >= 0 && iz[bz] >= 0;
    k.idx[c] = ok ? ((int64_t)ix[bx] * G.t.ny + iy[by]) * G.t.nz + iz[bz] : -1;
    k.w[c] = __fmul_rn(__fmul_rn(wx[bx], wy[by]), wz[bz]);
    k.g[c][0] = __fmul_rn(__fmul_rn(sx[bx], wy[by]), wz[bz]);
    k.g[c][1] = __fmul_rn(__fmul_rn(sy[by], wz[bz]), wx[bx]);
    k.g[c][2] = __fmul_rn(__fmul_rn(sz[bz], wx[bx]), wy[by]);
  }
}

__global__ void general_scatter_kernel(const int16_t* __restrict__ pmid, const float* __restrict__ disp,
                                       const uint8_t* __restrict__ valid, int64_t n, GeneralGrid G, int C,
                                       const float* __restrict__ val, float val_const,
                                       const double* __restrict__ scale_dev, unsigned long long* __restrict__ acc) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n || (valid != nullptr && !valid[p])) return;
  GeneralCorners k;
  general_corners(pmid, disp, p, G, k);
  const double scale = *scale_dev;
  const int64_t cells = G.t.cells();
  for (int c = 0; c < C; ++c) {
    const float v = val ? val[p * C + c] : val_const;
#pragma unroll
    for (int b = 0; b < 8; ++b) {
      if (k.idx[b] < 0) continue;
      const long long q = __double2ll_rn((double)__fmul_rn(v, k.w[b]) * scale);
      atomicAdd(&acc[c * cells + k.idx[b]], (unsigned long long)q);
    }
  }
}

__global__ void fixed_to_float_kernel(const unsigned long long* __restrict__ acc, int64_t count,
                                      const double* __restrict__ scale_dev, float* __restrict__ out) {
  const double inv = 1.0 / *scale_dev;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = (float)((double)(long long)acc[i] * inv);
}

__global__ void general_gather_kernel(const int16_t* __restrict__ pmid, const float* __restrict__ disp,
                                      const uint8_t* __restrict__ valid, int64_t n, GeneralGrid G, int C,
                                      const float* __restrict__ mesh, float* __restrict__ out) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const bool ok = valid == nullptr || valid[p];
  GeneralCorners k;
  general_corners(pmid, disp, p, G, k);
  const int64_t cells = G.t.cells();
  for (int c = 0; c < C; ++c) {
    float a = 0.f;
#pragma unroll
    for (int b = 0; b < 8; ++b)
      if (ok && k.idx[b] >= 0) a = __fadd_rn(a, __fmul_rn(mesh[c * cells + k.idx[b]], k.w[b]));
    out[p * C + c] = a;
  }
}

// disp_cot[p] = sum_b (sum_c u_c mesh_c[i_b]) grad_b / a2 and
// wsum[p, c] = sum_b mesh_c[i_b] w_b (cic/pallas.py:358-409, 327-355).
__global__ void general_interp_grad_kernel(const int16_t* __restrict__ pmid, const float* __restrict__ disp,
                                           const uint8_t* __restrict__ valid, int64_t n, GeneralGrid G, int C,
                                           const float* __restrict__ mesh, const float* __restrict__ u, float u_const,
                                           float* __restrict__ disp_cot, float* __restrict__ wsum) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const bool ok = valid == nullptr || valid[p];
  GeneralCorners k;
  general_corners(pmid, disp, p, G, k);
  const int64_t cells = G.t.cells();
  float g0 = 0.f, g1 = 0.f, g2 = 0.f;
#pragma unroll
  for (int b = 0; b < 8; ++b) {
    float inner = 0.f;
    for (int c = 0; c < C; ++c) {
      const float mv = (ok && k.idx[b] >= 0) ? mesh[c * cells + k.idx[b]] : 0.f;
      inner = __fadd_rn(inner, __fmul_rn(mv, u ? u[p * C + c] : u_const));
    }
    g0 = __fadd_rn(g0, __fmul_rn(inner, k.g[b][0]));
    g1 = __fadd_rn(g1, __fmul_rn(inner, k.g[b][1]));
    g2 = __fadd_rn(g2, __fmul_rn(inner, k.g[b][2]));
  }
  disp_cot[3 * p + 0] = __fdiv_rn(g0, G.a2);
  disp_cot[3 * p + 1] = __fdiv_rn(g1, G.a2);
  disp_cot[3 * p + 2] = __fdiv_rn(g2, G.a2);
  if (wsum != nullptr) {
    for (int c = 0; c < C; ++c) {
      float a = 0.f;
#pragma unroll
      for (int b = 0; b < 8; ++b)
        if (ok && k.idx[b] >= 0) a = __fadd_rn(a, __fmul_rn(mesh[c * cells + k.idx[b]], k.w[b]));
      wsum[p * C + c] = a;
    }
  }
}

int64_t general_scatter_scratch_bytes(Mesh3 t, int C) { return align_up(8 * (int64_t)C * t.cells(), 256) + 256; }

int general_scatter(const int16_t* pmid, const float* disp, const uint8_t* valid, int64_t n, GeneralGrid G, int C,
                    const float* val, float val_const, float* out, void* scratch, cudaStream_t s) {
  const int64_t count = (int64_t)C * G.t.cells();
  unsigned long long* acc = (unsigned long long*)scratch;
  char* tail = (char*)scratch + align_up(8 * count, 256);
  double* scale = (double*)tail;
  unsigned int* tmp = (unsigned int*)(tail + 8);
  if (val != nullptr) {
    int st = compute_scale(val, n * C, n, scale, tmp, s);
    if (st != kOk) return st;
  } else {
    const int st = set_double(scale, fixed_point_scale(fixed_point_pow2(n), fabsf(val_const)), s);
    if (st != kOk) return st;
  }
  PMB_CUDA_CHECK(cudaMemsetAsync(acc, 0, 8 * count, s));
  if (n > 0)
    general_scatter_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(pmid, disp, valid, n, G, C, val, val_const,
                                                                       scale, acc);
  if (count > 0) {
    int64_t blocks = (count + 255) / 256;
    if (blocks > 148 * 64) blocks = 148 * 64;
    fixed_to_float_kernel<<<(unsigned)blocks, 256, 0, s>>>(acc, count, scale, out);
  }
  PMB_CUDA_CHECK(cudaGetLastError());
  return kOk;
}

int general_gather(const int16_t* pmid, const float* disp, const uint8_t* valid, int64_t n, GeneralGrid G, int C,
                   const float* mesh, float* out, cudaStream_t s) {
  if (n > 0)
    general_gather_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(pmid, disp, valid, n, G, C, mesh, out);
  PMB_CUDA_CHECK(cudaGetLastError());
  return kOk;
}

int general_interp_grad(const int16_t* pmid, const float* disp, const uint8_t* valid, int64_t n, GeneralGrid G,
                        int C, const float* mesh, const float* u, float u_const, float* disp_cot, float* wsum,
                        cudaStream_t s) {
  if (n > 0)
    general_interp_grad_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(pmid, disp, valid, n, G, C, mesh, u,
                                                                           u_const, disp_cot, wsum);
  PMB_CUDA_CHECK(cudaGetLastError());
  return kOk;
}

}  // namespace pmb
