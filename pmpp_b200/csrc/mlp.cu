// Learned Green's-function correction: a small MLP
//   T(|k|, a, Omega_m, sigma8) = 1 + W4 sin(W3 sin(W2 sin(W1 x + b1) + b2) + b3) + b4,
//   x = (|k| / k_Nyquist, a, Omega_m, sigma8), width 64,
// that multiplies the Green's function (the hook of corrections/core.py:333-334;
// the reference's radial filter, corrections/radial.py:29-71, ignores the
// cosmology, this one is conditioned on it).  Weights are bf16, every product
// accumulates in FP32.  Because T depends on k only through |k|, it is
// evaluated once per force evaluation on the exact table of integer
// |n|^2 = nx^2 + ny^2 + nz^2 values (|k| / k_Ny = 2 sqrt(n^2) / M for a cubic
// mesh) and the Green x gradient kernel reads that table.  Training: the force
// adjoint emits dL/dT per |n|^2 (transfer_cot_kernel) and mlp_backward_kernel
// turns it into parameter gradients.  The whole network is ~10^8 flops per
// table, so it runs on the SIMT pipes; tensor cores would not change the
// step time.
#include <cuda_bf16.h>

#include "pmb_common.cuh"
#include "pmb_mlp.cuh"

namespace pmb {

namespace {
constexpr int H = kMlpWidth;
constexpr int kIn = 4;

struct MlpW {
  const __nv_bfloat16 *W1, *W2, *W3, *W4;  // [H][4], [H][H], [H][H], [H]
  const float *b1, *b2, *b3, *b4;          // [H], [H], [H], [1]
};

__device__ __forceinline__ MlpW unpack(const __nv_bfloat16* w, const float* b) {
  MlpW p;
  p.W1 = w;
  p.W2 = p.W1 + H * kIn;
  p.W3 = p.W2 + H * H;
  p.W4 = p.W3 + H * H;
  p.b1 = b;
  p.b2 = p.b1 + H;
  p.b3 = p.b2 + H;
  p.b4 = p.b3 + H;
  return p;
}

// Stage the bf16 weights (as float) and biases in shared memory.
struct SmemW {
  float W1[H * kIn], W2[H * H], W3[H * H], W4[H];
  float b1[H], b2[H], b3[H], b4;
};

__device__ void load_weights(SmemW& s, const MlpW& p) {
  for (int i = threadIdx.x; i < H * kIn; i += blockDim.x) s.W1[i] = __bfloat162float(p.W1[i]);
  for (int i = threadIdx.x; i < H * H; i += blockDim.x) {
    s.W2[i] = __bfloat162float(p.W2[i]);
    s.W3[i] = __bfloat162float(p.W3[i]);
  }
  for (int i = threadIdx.x; i < H; i += blockDim.x) {
    s.W4[i] = __bfloat162float(p.W4[i]);
    s.b1[i] = p.b1[i];
    s.b2[i] = p.b2[i];
    s.b3[i] = p.b3[i];
  }
  if (threadIdx.x == 0) s.b4 = p.b4[0];
}

__device__ __forceinline__ void features(int64_t n2, const MlpCond& c, float x[kIn]) {
  x[0] = sqrtf((float)n2) * c.kscale;
  x[1] = c.a;
  x[2] = c.omega_m;
  x[3] = c.sigma8;
}

// forward for one input; keeps the pre-activation states needed by backward
__device__ float forward_one(const SmemW& s, const float x[kIn], float z1[H], float z2[H], float z3[H]) {
  float h1[H], h2[H];
#pragma unroll 4
  for (int j = 0; j < H; ++j) {
    float acc = s.b1[j];
#pragma unroll
    for (int i = 0; i < kIn; ++i) acc = fmaf(s.W1[j * kIn + i], x[i], acc);
    z1[j] = acc;
    h1[j] = sinf(acc);
  }
  for (int j = 0; j < H; ++j) {
    float acc = s.b2[j];
#pragma unroll 8
    for (int i = 0; i < H; ++i) acc = fmaf(s.W2[j * H + i], h1[i], acc);
    z2[j] = acc;
    h2[j] = sinf(acc);
  }
  float y = s.b4;
  for (int j = 0; j < H; ++j) {
    float acc = s.b3[j];
#pragma unroll 8
    for (int i = 0; i < H; ++i) acc = fmaf(s.W3[j * H + i], h2[i], acc);
    z3[j] = acc;
    y = fmaf(s.W4[j], sinf(acc), y);
  }
  return y;
}
}  // namespace

// Table evaluation, tile-parallel: a block evaluates kTE entries; thread
// (group g, unit j) computes hidden unit j for entries g, g+4, ... so every
// layer is a (kTE x 64) x (64 x 64) product from shared memory.  Weights are
// kept transposed ([in][out]) so a warp reads 32 consecutive output units.
constexpr int kTE = 32;

__global__ void __launch_bounds__(256) mlp_table_kernel(const __nv_bfloat16* __restrict__ w,
                                                        const float* __restrict__ b, MlpCond cond, int len,
                                                        float* __restrict__ table) {
  __shared__ __nv_bfloat16 W2t[H * H], W3t[H * H];  // [in][out]
  __shared__ float W1t[kIn * H], W4[H], b1[H], b2[H], b3[H];
  __shared__ float xin[kTE][kIn];
  __shared__ float act[2][kTE][H];
  const MlpW p = unpack(w, b);
  for (int q = threadIdx.x; q < H * H; q += blockDim.x) {
    const int o = q / H, i = q % H;
    W2t[i * H + o] = p.W2[q];
    W3t[i * H + o] = p.W3[q];
  }
  for (int q = threadIdx.x; q < H * kIn; q += blockDim.x) W1t[(q % kIn) * H + q / kIn] = __bfloat162float(p.W1[q]);
  for (int q = threadIdx.x; q < H; q += blockDim.x) {
    W4[q] = __bfloat162float(p.W4[q]);
    b1[q] = p.b1[q];
    b2[q] = p.b2[q];
    b3[q] = p.b3[q];
  }
  const float b4 = p.b4[0];
  const int j = threadIdx.x % H;   // hidden unit
  const int g0 = threadIdx.x / H;  // entry group 0..3
  constexpr int kPer = kTE / 4;    // entries per thread
  for (int tile = blockIdx.x * kTE; tile < len; tile += gridDim.x * kTE) {
    __syncthreads();
    if (threadIdx.x < kTE) {
      float x[kIn];
      features(tile + threadIdx.x, cond, x);
#pragma unroll
      for (int i = 0; i < kIn; ++i) xin[threadIdx.x][i] = x[i];
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < kPer; ++k) {
      const int e = g0 + 4 * k;
      float acc = b1[j];
#pragma unroll
      for (int i = 0; i < kIn; ++i) acc = fmaf(W1t[i * H + j], xin[e][i], acc);
      act[0][e][j] = sinf(acc);
    }
    __syncthreads();
#pragma unroll
    for (int l = 0; l < 2; ++l) {
      const __nv_bfloat16* Wt = l == 0 ? W2t : W3t;
      const float* bl = l == 0 ? b2 : b3;
      float acc[kPer];
#pragma unroll
      for (int k = 0; k < kPer; ++k) acc[k] = bl[j];
      for (int i = 0; i < H; ++i) {
        const float wv = __bfloat162float(Wt[i * H + j]);
#pragma unroll
        for (int k = 0; k < kPer; ++k) acc[k] = fmaf(wv, act[l][g0 + 4 * k][i], acc[k]);
      }
#pragma unroll
      for (int k = 0; k < kPer; ++k) act[l ^ 1][g0 + 4 * k][j] = sinf(acc[k]);
      __syncthreads();
    }
    // output y_e = b4 + sum_j W4[j] h3[e][j]: one warp per entry
    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    for (int e = warp; e < kTE; e += blockDim.x / 32) {
      float v = W4[lane] * act[0][e][lane] + W4[lane + 32] * act[0][e][lane + 32];
      for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
      const int idx = tile + e;
      // T(|k| = 0) = 1 (corrections/radial.py:193-194)
      if (lane == 0 && idx < len) table[idx] = idx == 0 ? 1.0f : 1.0f + (b4 + v);
    }
  }
}

// Backward over the table: given dL/dT per entry (FP64), accumulate
// dL/dparams (FP32, parameter layout of the bf16 weights then the biases).
// Each block handles a tile of entries: per-entry deltas go to shared
// memory, then every thread owns a set of parameters and sums its
// outer-product contributions over the tile before one global atomic each.
constexpr int kTile = 32;

struct BackSmem {
  SmemW s;
  float sx[kTile][kIn];
  float sh1[kTile][H], sh2[kTile][H], sh3[kTile][H];
  float sd1[kTile][H], sd2[kTile][H], sd3[kTile][H];
  float sg[kTile];
};

__global__ void __launch_bounds__(128) mlp_backward_kernel(const __nv_bfloat16* __restrict__ w,
                                                           const float* __restrict__ b, MlpCond cond, int len,
                                                           const double* __restrict__ tcot,
                                                           float* __restrict__ grad) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  BackSmem& B = *reinterpret_cast<BackSmem*>(smem_raw);
  SmemW& s = B.s;
  auto& sx = B.sx;
  auto& sh1 = B.sh1;
  auto& sh2 = B.sh2;
  auto& sh3 = B.sh3;
  auto& sd1 = B.sd1;
  auto& sd2 = B.sd2;
  auto& sd3 = B.sd3;
  auto& sg = B.sg;
  load_weights(s, unpack(w, b));
  __syncthreads();
  for (int tile0 = blockIdx.x * kTile; tile0 < len; tile0 += gridDim.x * kTile) {
    // per-entry forward + backward (threads 0..kTile-1)
    if (threadIdx.x < kTile) {
      const int e = tile0 + threadIdx.x;
      const int t = threadIdx.x;
      float g = 0.f;
      float x[kIn], z1[H], z2[H], z3[H];
      if (e < len && e > 0) {
        g = (float)tcot[e];
        features(e, cond, x);
        forward_one(s, x, z1, z2, z3);
      } else {
        for (int i = 0; i < kIn; ++i) x[i] = 0.f;
        for (int j = 0; j < H; ++j) z1[j] = z2[j] = z3[j] = 0.f;
      }
      sg[t] = g;
      for (int i = 0; i < kIn; ++i) sx[t][i] = x[i];
      float d3[H];
      for (int j = 0; j < H; ++j) {
        sh1[t][j] = sinf(z1[j]);
        sh2[t][j] = sinf(z2[j]);
        sh3[t][j] = sinf(z3[j]);
        d3[j] = g * s.W4[j] * cosf(z3[j]);
        sd3[t][j] = d3[j];
      }
      float d2[H];
      for (int i = 0; i < H; ++i) {
        float acc = 0.f;
        for (int j = 0; j < H; ++j) acc = fmaf(s.W3[j * H + i], d3[j], acc);
        d2[i] = acc * cosf(z2[i]);
        sd2[t][i] = d2[i];
      }
      for (int i = 0; i < H; ++i) {
        float acc = 0.f;
        for (int j = 0; j < H; ++j) acc = fmaf(s.W2[j * H + i], d2[j], acc);
        sd1[t][i] = acc * cosf(z1[i]);
      }
    }
    __syncthreads();
    // parameter gradients: each thread owns parameters p = tid, tid + 128, ...
    const int nW1 = H * kIn, nW2 = H * H, nW3 = H * H, nW4 = H;
    const int total = nW1 + nW2 + nW3 + nW4 + 3 * H + 1;
    for (int p = threadIdx.x; p < total; p += blockDim.x) {
      float acc = 0.f;
      if (p < nW1) {
        const int j = p / kIn, i = p % kIn;
        for (int t = 0; t < kTile; ++t) acc = fmaf(sd1[t][j], sx[t][i], acc);
      } else if (p < nW1 + nW2) {
        const int q = p - nW1, j = q / H, i = q % H;
        for (int t = 0; t < kTile; ++t) acc = fmaf(sd2[t][j], sh1[t][i], acc);
      } else if (p < nW1 + nW2 + nW3) {
        const int q = p - nW1 - nW2, j = q / H, i = q % H;
        for (int t = 0; t < kTile; ++t) acc = fmaf(sd3[t][j], sh2[t][i], acc);
      } else if (p < nW1 + nW2 + nW3 + nW4) {
        const int j = p - nW1 - nW2 - nW3;
        for (int t = 0; t < kTile; ++t) acc = fmaf(sg[t], sh3[t][j], acc);
      } else {
        const int q = p - (nW1 + nW2 + nW3 + nW4);
        if (q < H) {
          for (int t = 0; t < kTile; ++t) acc += sd1[t][q];
        } else if (q < 2 * H) {
          for (int t = 0; t < kTile; ++t) acc += sd2[t][q - H];
        } else if (q < 3 * H) {
          for (int t = 0; t < kTile; ++t) acc += sd3[t][q - 2 * H];
        } else {
          for (int t = 0; t < kTile; ++t) acc += sg[t];
        }
      }
      if (acc != 0.f) atomicAdd(&grad[p], acc);
    }
    __syncthreads();
  }
}

// dL/dT per integer |n|^2 of one force adjoint:
//   sum over half-spectrum cells with that |n|^2 of
//   mult / M * Re(conj(sum_d (-i c_d) R_d) * G * mask * S_hat)
// where R_d = rFFT of the force-mesh cotangents and S_hat = rFFT of the
// Poisson source at the same positions.  (The transfer enters as
// phi = T * G * mask * S_hat and the C2R transpose weights stored cells by
// mult / M in the packed d/dRe + i d/dIm convention.)
__global__ void transfer_cot_kernel(const float2* __restrict__ R3, const float2* __restrict__ S_hat, Mesh3 m,
                                    SpecTables t, double inv_m, int len, double* __restrict__ out) {
  extern __shared__ double sh[];
  for (int i = threadIdx.x; i < len; i += blockDim.x) sh[i] = 0.0;
  __syncthreads();
  const int nzh = m.nz / 2 + 1;
  const int64_t total = m.half_cells();
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < total; j += (int64_t)gridDim.x * blockDim.x) {
    const int iz = (int)(j % nzh);
    const int64_t r = j / nzh;
    const int iy = (int)(r % m.ny);
    const int ix = (int)(r / m.ny);
    const float kx = t.kx[ix], ky = t.ky[iy], kz = t.kz[iz];
    const float k2 = __fadd_rn(__fadd_rn(__fmul_rn(kx, kx), __fmul_rn(ky, ky)), __fmul_rn(kz, kz));
    if (k2 == 0.f) continue;
    const float c[3] = {t.cx[ix], t.cy[iy], t.cz[iz]};
    double ur = 0.0, ui = 0.0;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const float2 a = R3[(int64_t)d * total + j];
      ur += (double)c[d] * a.y;
      ui -= (double)c[d] * a.x;
    }
    float2 sv = S_hat[j];
    double mk = 1.0;
    if (t.mx != nullptr) mk = (double)t.mx[ix] * t.my[iy] * t.mz[iz];
    const double g = -mk / (double)k2;
    const double qr = g * sv.x, qi = g * sv.y;
    const double mult = (iz == 0 || ((m.nz % 2 == 0) && iz == nzh - 1)) ? 1.0 : 2.0;
    const int nx = ix < (m.nx + 1) / 2 ? ix : ix - m.nx;
    const int ny = iy < (m.ny + 1) / 2 ? iy : iy - m.ny;
    const long long n2 = (long long)nx * nx + (long long)ny * ny + (long long)iz * iz;
    if (n2 < len) atomicAdd(&sh[n2], mult * inv_m * (ur * qr + ui * qi));
  }
  __syncthreads();
  for (int i = threadIdx.x; i < len; i += blockDim.x)
    if (sh[i] != 0.0) atomicAdd(&out[i], sh[i]);
}

int mlp_table(const void* w, const float* b, MlpCond c, int len, float* table, cudaStream_t s) {
  int blocks = (len + kTE - 1) / kTE;
  if (blocks > 148 * 8) blocks = 148 * 8;
  mlp_table_kernel<<<blocks > 0 ? blocks : 1, 256, 0, s>>>((const __nv_bfloat16*)w, b, c, len, table);
  PMB_CUDA_CHECK(cudaGetLastError());
  return kOk;
}

int mlp_backward(const void* w, const float* b, MlpCond c, int len, const double* tcot, float* grad, cudaStream_t s) {
  int blocks = (len + kTile - 1) / kTile;
  if (blocks > 148 * 2) blocks = 148 * 2;
  PMB_CUDA_CHECK(smem_optin((const void*)mlp_backward_kernel, (int)sizeof(BackSmem)));
  mlp_backward_kernel<<<blocks > 0 ? blocks : 1, 128, sizeof(BackSmem), s>>>((const __nv_bfloat16*)w, b, c, len, tcot,
                                                                            grad);
  PMB_CUDA_CHECK(cudaGetLastError());
  return kOk;
}

int transfer_cot(const float2* R3, const float2* S_hat, Mesh3 m, SpecTables t, int len, double* out, cudaStream_t s) {
  const size_t smem = sizeof(double) * (size_t)len;
  if (smem > 200 * 1024) return kUnsupported;
  PMB_CUDA_CHECK(smem_optin((const void*)transfer_cot_kernel, 200 * 1024));
  int64_t blocks = (m.half_cells() + 255) / 256;
  if (blocks > 148 * 4) blocks = 148 * 4;
  transfer_cot_kernel<<<(unsigned)(blocks > 0 ? blocks : 1), 256, smem, s>>>(R3, S_hat, m, t, 1.0 / (double)m.cells(),
                                                                           len, out);
  PMB_CUDA_CHECK(cudaGetLastError());
  return kOk;
}

}  // namespace pmb
