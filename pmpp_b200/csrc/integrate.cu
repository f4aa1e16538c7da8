// Kick, drift and their adjoints, plus FP64 reductions for the cosmology
// cotangents.  Float updates use two roundings (multiply, then add) exactly as
// the reference's XLA elementwise ops: integrator.py:225 (drift), :536
// (kick), :570-580 (kick adjoint), :465-473 (drift adjoint).
#include "pmb_common.cuh"
#include "pmb_integrate.cuh"

namespace pmb {

namespace {
unsigned grid_n(int64_t n, int th) {
  int64_t b = (n + th - 1) / th;
  int64_t cap = 148 * 32;
  return (unsigned)(b < cap ? (b > 0 ? b : 1) : cap);
}

__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
  return v;
}

__device__ __forceinline__ void block_add(double v, double* out) {
  __shared__ double sh[32];
  v = warp_sum(v);
  int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) sh[w] = v;
  __syncthreads();
  if (w == 0) {
    v = lane < (int)(blockDim.x >> 5) ? sh[lane] : 0.0;
    v = warp_sum(v);
    if (lane == 0) atomicAdd(out, v);
  }
}
}  // namespace

// y += x * f
__global__ void axpy_kernel(float* __restrict__ y, const float* __restrict__ x, int64_t n, float f) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    y[i] = __fadd_rn(y[i], __fmul_rn(x[i], f));
}

// Kick adjoint (integrator.py:566-580): vel -= acc*K; acc_cot += vel_cot*K;
// dot += sum(vel_cot * acc).
__global__ void kick_adj_kernel(float* __restrict__ vel, const float* __restrict__ acc, const float* __restrict__ vel_cot,
                                float* __restrict__ acc_cot, int64_t n, float k, double* __restrict__ dot) {
  double s = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float a = acc[i], vc = vel_cot[i];
    vel[i] = __fsub_rn(vel[i], __fmul_rn(a, k));
    acc_cot[i] = __fadd_rn(acc_cot[i], __fmul_rn(vc, k));
    s += (double)vc * (double)a;
  }
  block_add(s, dot);
}

// Drift adjoint (integrator.py:459-474): disp -= vel*D; vel_cot += disp_cot*D;
// dot += sum(disp_cot * vel).
// One or two consecutive kick adjoints with the same acceleration (the closing
// half-kick of one step and the opening one of the next), in the order the
// separate kernels would apply them, plus the force-slot dot sum(acc_cot * acc)
// of the force adjoint that follows.  zero_cot: acc_cot is taken as zero
// (the force adjoint before consumed it).
// With disp_cot, the cotangent half of the drift adjoint that precedes the
// kicks in the reverse sweep runs first, as drift_cot_adj_kernel would:
// vel_cot += disp_cot * dd, dot_d += sum disp_cot * vel (vel before the kicks).
__global__ void kick_adj2_kernel(float* __restrict__ vel, const float* __restrict__ acc,
                                 float* __restrict__ vel_cot, float* __restrict__ acc_cot, int64_t n, float ka,
                                 float kb, int two, int zero_cot, double* __restrict__ dot_a,
                                 double* __restrict__ dot_b, double* __restrict__ dot_f,
                                 const float* __restrict__ disp_cot, float dd, double* __restrict__ dot_d) {
  double s = 0.0, sf = 0.0, sd = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float a = acc[i];
    float vc = vel_cot[i];
    float v = vel[i];
    if (disp_cot != nullptr) {
      const float dc = disp_cot[i];
      vc = __fadd_rn(vc, __fmul_rn(dc, dd));
      vel_cot[i] = vc;
      sd += (double)dc * (double)v;
    }
    v = __fsub_rn(v, __fmul_rn(a, ka));
    float c = __fadd_rn(zero_cot ? 0.f : acc_cot[i], __fmul_rn(vc, ka));
    if (two) {
      v = __fsub_rn(v, __fmul_rn(a, kb));
      c = __fadd_rn(c, __fmul_rn(vc, kb));
    }
    vel[i] = v;
    acc_cot[i] = c;
    s += (double)vc * (double)a;
    sf += (double)c * (double)a;
  }
  block_add(s, dot_a);
  if (two) block_add(s, dot_b);
  if (dot_f != nullptr) block_add(sf, dot_f);
  if (disp_cot != nullptr) block_add(sd, dot_d);
}

// Cotangent half of the drift adjoint: vel_cot += disp_cot * d, dot += sum
// disp_cot * vel.  The position half (disp -= vel * d) runs fused into the
// next force evaluation's sort as a drift by -d (the same float operations).
__global__ void drift_cot_adj_kernel(const float* __restrict__ vel, const float* __restrict__ disp_cot,
                                     float* __restrict__ vel_cot, int64_t n, float d, double* __restrict__ dot) {
  double s = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float dc = disp_cot[i];
    vel_cot[i] = __fadd_rn(vel_cot[i], __fmul_rn(dc, d));
    s += (double)dc * (double)vel[i];
  }
  block_add(s, dot);
}

__global__ void drift_adj_kernel(float* __restrict__ disp, const float* __restrict__ vel,
                                 const float* __restrict__ disp_cot, float* __restrict__ vel_cot, int64_t n, float d,
                                 double* __restrict__ dot) {
  double s = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float v = vel[i], dc = disp_cot[i];
    disp[i] = __fsub_rn(disp[i], __fmul_rn(v, d));
    vel_cot[i] = __fadd_rn(vel_cot[i], __fmul_rn(dc, d));
    s += (double)dc * (double)v;
  }
  block_add(s, dot);
}

__global__ void dot_kernel(const float* __restrict__ a, const float* __restrict__ b, int64_t n, double* __restrict__ out) {
  double s = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    s += (double)a[i] * (double)b[i];
  block_add(s, out);
}

__global__ void sum_kernel(const float* __restrict__ a, int64_t n, double* __restrict__ out) {
  double s = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    s += (double)a[i];
  block_add(s, out);
}

__global__ void set_double_kernel(double* p, double v) { *p = v; }

int axpy(float* y, const float* x, int64_t n, float f, cudaStream_t s) {
  if (n > 0) axpy_kernel<<<grid_n(n, 256), 256, 0, s>>>(y, x, n, f);
  PMB_CUDA_CHECK(cudaGetLastError());
  return kOk;
}

int kick_adj(float* vel, const float* acc, const float* vel_cot, float* acc_cot, int64_t n, float k, double* dot,
             cudaStream_t s) {
  if (n > 0) kick_adj_kernel<<<grid_n(n, 256), 256, 0, s>>>(vel, acc, vel_cot, acc_cot, n, k, dot);
  PMB_CUDA_CHECK(cudaGetLastError());
  return kOk;
}

int kick_adj2(float* vel, const float* acc, float* vel_cot, float* acc_cot, int64_t n, float ka, float kb,
              int two, int zero_cot, double* dot_a, double* dot_b, double* dot_f, const float* disp_cot, float dd,
              double* dot_d, cudaStream_t s) {
  if (n > 0)
    kick_adj2_kernel<<<grid_n(n, 256), 256, 0, s>>>(vel, acc, vel_cot, acc_cot, n, ka, kb, two, zero_cot, dot_a, dot_b,
                                                    dot_f, disp_cot, dd, dot_d);
  PMB_CUDA_CHECK(cudaGetLastError());
  return kOk;
}

int drift_cot_adj(const float* vel, const float* disp_cot, float* vel_cot, int64_t n, float d, double* dot,
                  cudaStream_t s) {
  if (n > 0) drift_cot_adj_kernel<<<grid_n(n, 256), 256, 0, s>>>(vel, disp_cot, vel_cot, n, d, dot);
  PMB_CUDA_CHECK(cudaGetLastError());
  return kOk;
}

int drift_adj(float* disp, const float* vel, const float* disp_cot, float* vel_cot, int64_t n, float d, double* dot,
              cudaStream_t s) {
  if (n > 0) drift_adj_kernel<<<grid_n(n, 256), 256, 0, s>>>(disp, vel, disp_cot, vel_cot, n, d, dot);
  PMB_CUDA_CHECK(cudaGetLastError());
  return kOk;
}

int dot(const float* a, const float* b, int64_t n, double* out, cudaStream_t s) {
  if (n > 0) dot_kernel<<<grid_n(n, 256), 256, 0, s>>>(a, b, n, out);
  PMB_CUDA_CHECK(cudaGetLastError());
  return kOk;
}

int sum(const float* a, int64_t n, double* out, cudaStream_t s) {
  if (n > 0) sum_kernel<<<grid_n(n, 256), 256, 0, s>>>(a, n, out);
  PMB_CUDA_CHECK(cudaGetLastError());
  return kOk;
}

int set_double(double* p, double v, cudaStream_t s) {
  set_double_kernel<<<1, 1, 0, s>>>(p, v);
  PMB_CUDA_CHECK(cudaGetLastError());
  return kOk;
}

}  // namespace pmb
