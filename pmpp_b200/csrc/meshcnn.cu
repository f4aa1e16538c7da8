// Mesh-CNN residual potential (corrections/mesh_cnn.py:66-110,
// corrections/core.py:321-331): a small periodic 3-D convolutional network
// that maps the normalised Poisson source and potential (plus constant
// conditioning channels a, Omega_m, sigma8) to a real-space potential
// residual.  The host (pmpp_b200/meshcnn.py) composes the network from the
// kernels here; all tensors are channel-planar float32 (C, nx, ny, nz).
//
// Convolutions follow haiku's Conv3D after explicit periodic padding by one
// cell ('VALID'): out[co](p) = bias[co] + sum_tap sum_ci in[ci](p + off(tap))
// W[tap][ci][co], tap = (kd * 3 + kh) * 3 + kw, off = (kd-1, kh-1, kw-1)
// (cross-correlation, weights (3, 3, 3, Cin, Cout) as haiku stores them).
// The transposed form (the input gradient of a layer with weights
// (3, 3, 3, CO, CI)) reads W[tap][co][ci] at p - off(tap).  One thread per
// output cell holds the CO accumulators; weights sit in shared memory; the
// 27 neighbour loads per input channel come through L1.
#include "../../include/pmb200.h"
#include "pmb_common.cuh"
#include "pmb_kernels.cuh"

namespace pmb {
namespace {

constexpr float kGeluC = 0.7978845608028654f;  // sqrt(2 / pi)
constexpr float kGeluA = 0.044715f;

// jax.nn.gelu (approximate=True): 0.5 x (1 + tanh(sqrt(2/pi) (x + 0.044715 x^3)))
__device__ __forceinline__ float gelu(float x) {
  const float u = kGeluC * (x + kGeluA * x * x * x);
  return 0.5f * x * (1.f + tanhf(u));
}
__device__ __forceinline__ float gelu_grad(float x) {
  const float u = kGeluC * (x + kGeluA * x * x * x);
  const float t = tanhf(u);
  return 0.5f * (1.f + t) + 0.5f * x * (1.f - t * t) * kGeluC * (1.f + 3.f * kGeluA * x * x);
}

__device__ __forceinline__ int wrap(int i, int n) { return i < 0 ? i + n : (i >= n ? i - n : i); }

// act: 0 z only; 1 z and h = gelu(z); 2 z * gelu'(zref) (a backward step).
template <int CI, int CO, bool TRANS>
__global__ void __launch_bounds__(256) cnn_conv_kernel(const float* __restrict__ in, const float* __restrict__ W,
                                                       const float* __restrict__ bias, const float* __restrict__ res,
                                                       const float* __restrict__ zref, int act,
                                                       float* __restrict__ out_z, float* __restrict__ out_h, Mesh3 m) {
  __shared__ float sw[27 * CI * CO];
  for (int i = threadIdx.x; i < 27 * CI * CO; i += blockDim.x) sw[i] = W[i];
  __syncthreads();
  const int64_t cells = m.cells();
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < cells; p += (int64_t)gridDim.x * blockDim.x) {
    const int z = (int)(p % m.nz);
    const int64_t r = p / m.nz;
    const int y = (int)(r % m.ny), x = (int)(r / m.ny);
    float acc[CO];
#pragma unroll
    for (int co = 0; co < CO; ++co) acc[co] = bias != nullptr ? bias[co] : 0.f;
    for (int kd = 0; kd < 3; ++kd) {
      const int xx = wrap(TRANS ? x - (kd - 1) : x + (kd - 1), m.nx);
      for (int kh = 0; kh < 3; ++kh) {
        const int yy = wrap(TRANS ? y - (kh - 1) : y + (kh - 1), m.ny);
        const int64_t rowp = ((int64_t)xx * m.ny + yy) * m.nz;
#pragma unroll
        for (int kw = 0; kw < 3; ++kw) {
          const int zz = wrap(TRANS ? z - (kw - 1) : z + (kw - 1), m.nz);
          const int tap = (kd * 3 + kh) * 3 + kw;
          const float* wt = sw + tap * CI * CO;
#pragma unroll
          for (int ci = 0; ci < CI; ++ci) {
            const float v = __ldg(in + (int64_t)ci * cells + rowp + zz);
#pragma unroll
            for (int co = 0; co < CO; ++co) acc[co] = fmaf(v, TRANS ? wt[co * CI + ci] : wt[ci * CO + co], acc[co]);
          }
        }
      }
    }
#pragma unroll
    for (int co = 0; co < CO; ++co) {
      float v = acc[co];
      if (res != nullptr) v += res[(int64_t)co * cells + p];
      if (act == 2) v *= gelu_grad(zref[(int64_t)co * cells + p]);
      out_z[(int64_t)co * cells + p] = v;
      if (act == 1) out_h[(int64_t)co * cells + p] = gelu(v);
    }
  }
}

// dW[tap][ci][co] += sum_p in[ci](p + off(tap)) dout[co](p), db[co] += sum_p
// dout[co](p).  Persistent blocks take whole z-rows: the nine (x, y)
// neighbour rows of the input and the output row go to shared memory, each
// thread keeps its weights' partial sums in registers across rows, and adds
// them to the FP64 totals once at the end.
template <int CI, int CO>
__global__ void __launch_bounds__(256) cnn_wgrad_kernel(const float* __restrict__ in, const float* __restrict__ dout,
                                                        Mesh3 m, double* __restrict__ dW, double* __restrict__ db) {
  constexpr int NWT = 27 * CI * CO;
  constexpr int PER = (NWT + 255) / 256;
  extern __shared__ float sm[];
  float* s_in = sm;                      // [9][CI][nz]
  float* sd = sm + 9 * CI * m.nz;        // [CO][nz]
  const int64_t cells = m.cells();
  const int nz = m.nz;
  float acc[PER];
#pragma unroll
  for (int k = 0; k < PER; ++k) acc[k] = 0.f;
  float bacc = 0.f;
  const int64_t rows = (int64_t)m.nx * m.ny;
  for (int64_t r = blockIdx.x; r < rows; r += gridDim.x) {
    const int y = (int)(r % m.ny), x = (int)(r / m.ny);
    __syncthreads();
    for (int i = threadIdx.x; i < 9 * CI * nz; i += blockDim.x) {
      const int zz = i % nz, rest = i / nz;
      const int ci = rest % CI, nb = rest / CI;
      const int xx = wrap(x + nb / 3 - 1, m.nx), yy = wrap(y + nb % 3 - 1, m.ny);
      s_in[i] = in[(int64_t)ci * cells + ((int64_t)xx * m.ny + yy) * nz + zz];
    }
    for (int i = threadIdx.x; i < CO * nz; i += blockDim.x) {
      const int zz = i % nz, co = i / nz;
      sd[i] = dout[(int64_t)co * cells + r * nz + zz];
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < PER; ++k) {
      const int w = threadIdx.x + 256 * k;
      if (w < NWT) {
        const int co = w % CO, ci = (w / CO) % CI, tap = w / (CI * CO);
        const int kd = tap / 9, kh = (tap / 3) % 3, kw = tap % 3;
        const float* src = s_in + ((kd * 3 + kh) * CI + ci) * nz;
        const float* d = sd + co * nz;
        float s = 0.f;
        for (int zz = 0; zz < nz; ++zz) s = fmaf(src[wrap(zz + kw - 1, nz)], d[zz], s);
        acc[k] += s;
      }
    }
    if (db != nullptr && threadIdx.x < CO) {
      float s = 0.f;
      for (int zz = 0; zz < nz; ++zz) s += sd[threadIdx.x * nz + zz];
      bacc += s;
    }
  }
#pragma unroll
  for (int k = 0; k < PER; ++k) {
    const int w = threadIdx.x + 256 * k;
    if (w < NWT) atomicAdd(&dW[w], (double)acc[k]);
  }
  if (db != nullptr && threadIdx.x < CO) atomicAdd(&db[threadIdx.x], (double)bacc);
}

// x0 = [S * inv_s, phi * inv_p] (the normalised source and potential)
__global__ void cnn_stem_input_kernel(const float* __restrict__ S, const float* __restrict__ phi, int64_t n,
                                      float inv_s, float inv_p, float* __restrict__ x0) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    x0[i] = S[i] * inv_s;
    x0[n + i] = phi[i] * inv_p;
  }
}

// R = g phi + c tanh(o)  with c = max_residual * potential scale
__global__ void cnn_residual_kernel(const float* __restrict__ phi, const float* __restrict__ o, int64_t n, float g,
                                    float c, float* __restrict__ R) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    R[i] = g * phi[i] + c * tanhf(o[i]);
}

// Transpose of cnn_residual_kernel: dphi = g Rc, do = Rc c (1 - tanh(o)^2),
// dots[0] += sum Rc phi (for g), dots[1] += sum Rc tanh(o) (for c).
__global__ void cnn_residual_adjoint_kernel(const float* __restrict__ Rc, const float* __restrict__ phi,
                                            const float* __restrict__ o, int64_t n, float g, float c,
                                            float* __restrict__ dphi, float* __restrict__ dout,
                                            double* __restrict__ dots) {
  double s0 = 0.0, s1 = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float rc = Rc[i], t = tanhf(o[i]);
    dphi[i] = g * rc;
    dout[i] = rc * c * (1.f - t * t);
    s0 += (double)rc * phi[i];
    s1 += (double)rc * t;
  }
  for (int k = 16; k; k >>= 1) {
    s0 += __shfl_xor_sync(0xFFFFFFFFu, s0, k);
    s1 += __shfl_xor_sync(0xFFFFFFFFu, s1, k);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(&dots[0], s0);
    atomicAdd(&dots[1], s1);
  }
}

// Through the normalisations x = v / s(v), s = sqrt(mean(v^2) + eps):
// dv = dx / s - v * (sum dx v) / (M s^3), given per input cS = sum(dx v) /
// (M s^3); plus a direct term kP * phi for the potential scale's own use.
__global__ void cnn_norm_adjoint_kernel(const float* __restrict__ dx0, const float* __restrict__ S,
                                        const float* __restrict__ phi, int64_t n, float inv_s, float cS, float inv_p,
                                        float cP, float* __restrict__ dS, float* __restrict__ dphi) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    dS[i] = dx0[i] * inv_s - S[i] * cS;
    dphi[i] += dx0[n + i] * inv_p - phi[i] * cP;
  }
}

unsigned grid_of(int64_t n) {
  int64_t b = (n + 255) / 256;
  const int64_t cap = 148 * 16;
  return (unsigned)(b < 1 ? 1 : (b > cap ? cap : b));
}

template <int CI, int CO>
int launch_conv(const float* in, const float* W, const float* bias, const float* res, const float* zref, int act,
                float* out_z, float* out_h, Mesh3 m, bool trans, cudaStream_t s) {
  if (trans)
    cnn_conv_kernel<CI, CO, true><<<grid_of(m.cells()), 256, 0, s>>>(in, W, bias, res, zref, act, out_z, out_h, m);
  else
    cnn_conv_kernel<CI, CO, false><<<grid_of(m.cells()), 256, 0, s>>>(in, W, bias, res, zref, act, out_z, out_h, m);
  PMB_CUDA_CHECK(cudaGetLastError());
  return kOk;
}

template <int CI, int CO>
int launch_wgrad(const float* in, const float* dout, Mesh3 m, double* dW, double* db, cudaStream_t s) {
  const size_t smem = sizeof(float) * (size_t)(9 * CI + CO) * m.nz;
  if (smem > 200 * 1024) {
    set_last_error("pmb_cnn_conv3d_wgrad: mesh rows too long for the shared-memory row tile");
    return kUnsupported;
  }
  PMB_CUDA_CHECK(smem_optin((const void*)cnn_wgrad_kernel<CI, CO>, 200 * 1024));
  const int64_t rows = (int64_t)m.nx * m.ny;
  const unsigned grid = (unsigned)(rows < 148 * 2 ? rows : 148 * 2);
  cnn_wgrad_kernel<CI, CO><<<grid, 256, smem, s>>>(in, dout, m, dW, db);
  PMB_CUDA_CHECK(cudaGetLastError());
  return kOk;
}

// (ci, co) pairs of the network: stem 2 -> C, blocks C -> C, head C -> 1, for C in {4, 8, 16}
#define PMB_CNN_PAIRS(X) X(2, 4) X(4, 4) X(4, 1) X(2, 8) X(8, 8) X(8, 1) X(2, 16) X(16, 16) X(16, 1)

}  // namespace
}  // namespace pmb

using namespace pmb;

#define CNN_REQUIRE(cond, msg) \
  do {                         \
    if (!(cond)) {             \
      set_last_error(msg);     \
      return kInvalidArgument; \
    }                          \
  } while (0)

extern "C" {

int pmb_cnn_conv3d(const float* in, int ci, const float* W, const float* bias, const float* res, const float* zref,
                   int act, float* out_z, float* out_h, int co, int nx, int ny, int nz, int transposed,
                   void* stream) {
  CNN_REQUIRE(nx > 0 && ny > 0 && nz > 0, "pmb_cnn_conv3d: bad mesh");
  CNN_REQUIRE(in && W && out_z, "pmb_cnn_conv3d: null buffer");
  CNN_REQUIRE(act >= 0 && act <= 2, "pmb_cnn_conv3d: act must be 0, 1 or 2");
  CNN_REQUIRE(act != 1 || out_h != nullptr, "pmb_cnn_conv3d: act 1 needs out_h");
  CNN_REQUIRE(act != 2 || zref != nullptr, "pmb_cnn_conv3d: act 2 needs zref");
  Mesh3 m{nx, ny, nz};
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  // transposed: the forward layer's (CI, CO) are (co, ci) of this call
  const int fi = transposed ? co : ci, fo = transposed ? ci : co;
#define PMB_CNN_CONV_CASE(A, B)                                                                          \
  if (fi == A && fo == B)                                                                                \
    return transposed ? launch_conv<B, A>(in, W, bias, res, zref, act, out_z, out_h, m, true, s)         \
                      : launch_conv<A, B>(in, W, bias, res, zref, act, out_z, out_h, m, false, s);
  PMB_CNN_PAIRS(PMB_CNN_CONV_CASE)
#undef PMB_CNN_CONV_CASE
  set_last_error("pmb_cnn_conv3d: unsupported channel pair (stem 2->C, C->C, C->1 with C in {4, 8, 16})");
  return kUnsupported;
}

int pmb_cnn_conv3d_wgrad(const float* in, int ci, const float* dout, int co, int nx, int ny, int nz, double* dW,
                         double* db, void* stream) {
  CNN_REQUIRE(nx > 0 && ny > 0 && nz > 0, "pmb_cnn_conv3d_wgrad: bad mesh");
  CNN_REQUIRE(in && dout && dW, "pmb_cnn_conv3d_wgrad: null buffer");
  Mesh3 m{nx, ny, nz};
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
#define PMB_CNN_WGRAD_CASE(A, B) \
  if (ci == A && co == B) return launch_wgrad<A, B>(in, dout, m, dW, db, s);
  PMB_CNN_PAIRS(PMB_CNN_WGRAD_CASE)
#undef PMB_CNN_WGRAD_CASE
  set_last_error("pmb_cnn_conv3d_wgrad: unsupported channel pair");
  return kUnsupported;
}

int pmb_cnn_stem_input(const float* S, const float* phi, int64_t n, float inv_s, float inv_p, float* x0,
                       void* stream) {
  CNN_REQUIRE(n > 0 && S && phi && x0, "pmb_cnn_stem_input: bad arguments");
  cnn_stem_input_kernel<<<grid_of(n), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(S, phi, n, inv_s, inv_p, x0);
  PMB_CUDA_CHECK(cudaGetLastError());
  return kOk;
}

int pmb_cnn_residual(const float* phi, const float* o, int64_t n, float g, float c, float* R, void* stream) {
  CNN_REQUIRE(n > 0 && phi && o && R, "pmb_cnn_residual: bad arguments");
  cnn_residual_kernel<<<grid_of(n), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(phi, o, n, g, c, R);
  PMB_CUDA_CHECK(cudaGetLastError());
  return kOk;
}

int pmb_cnn_residual_adjoint(const float* Rc, const float* phi, const float* o, int64_t n, float g, float c,
                             float* dphi, float* dout, double* dots, void* stream) {
  CNN_REQUIRE(n > 0 && Rc && phi && o && dphi && dout && dots, "pmb_cnn_residual_adjoint: bad arguments");
  cnn_residual_adjoint_kernel<<<grid_of(n), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(Rc, phi, o, n, g, c,
                                                                                               dphi, dout, dots);
  PMB_CUDA_CHECK(cudaGetLastError());
  return kOk;
}

int pmb_cnn_norm_adjoint(const float* dx0, const float* S, const float* phi, int64_t n, float inv_s, float cS,
                         float inv_p, float cP, float* dS, float* dphi, void* stream) {
  CNN_REQUIRE(n > 0 && dx0 && S && phi && dS && dphi, "pmb_cnn_norm_adjoint: bad arguments");
  cnn_norm_adjoint_kernel<<<grid_of(n), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(dx0, S, phi, n, inv_s, cS,
                                                                                           inv_p, cP, dS, dphi);
  PMB_CUDA_CHECK(cudaGetLastError());
  return kOk;
}

}  // extern "C"
