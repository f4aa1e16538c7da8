// Shared definitions for the PM++ B200 kernels.
//
// Layout conventions (all C order, row-major):
//   pmid   int16  (N, 3)       anchor mesh cell of each particle
//   disp   float  (N, 3)       comoving displacement from pmid * cell
//   vel/acc float (N, 3)
//   mesh   float  (C, Mx, My, Mz)          planar channels
//   spec   float2 (C, Mx, My, Mz/2 + 1)    rFFT half spectra
// A "row" is the z-line (x, y) of the mesh; the cell sort bins particles by
// the row of their lower CIC corner, so bin order equals raveled-cell order.
#pragma once

#include <cmath>
#include <cstdint>
#include <cuda_runtime.h>
#include <map>
#include <mutex>
#include <utility>

namespace pmb {

// Status codes returned by every C-ABI entry point.
enum Status : int {
  kOk = 0,
  kInvalidArgument = -1,
  kCudaError = -2,
  kCufftError = -3,
  kUnsupported = -4,
  kScratchTooSmall = -5,
  kDeviceFlagged = -6,
};

// Conditions the kernels report through the status word of a sorted buffer
// and the device-wide flags (pmb_sorted_status, pmb_device_status).
enum DeviceFlag : unsigned int {
  kFlagWaitTimeout = 1u,     // a bounded wait on bulk / TMA copies gave up
  kFlagNonFiniteDisp = 2u,   // a displacement reaching the cell sort was NaN or infinite
  kFlagNonFiniteValue = 4u,  // a deposited value was NaN or infinite
};

struct Mesh3 {
  int nx, ny, nz;
  __host__ __device__ int64_t rows() const { return (int64_t)nx * ny; }
  __host__ __device__ int64_t cells() const { return (int64_t)nx * ny * nz; }
  __host__ __device__ int64_t half_cells() const { return (int64_t)nx * ny * (nz / 2 + 1); }
};

__host__ __device__ inline int pmod(int a, int m) {
  int r = a % m;
  return r < 0 ? r + m : r;
}

__host__ __device__ inline int64_t align_up(int64_t v, int64_t a) { return (v + a - 1) / a * a; }

// Particle binning shared by every CIC kernel.  Restates the float32
// arithmetic of the reference enmesh (cic/enmesh.py:139-149) and the Pallas
// coordinate helper (cic/pallas.py:225-256): d = disp / cell in IEEE float
// (no fast-math), lower corner i = pmid + floor(d), fraction f = d - floor(d)
// (exact in float).  The per-axis corner weight is 1 - |f - b| evaluated in
// float, which reproduces 1 - |d - (floor(d) + b)| bit for bit.
__device__ __forceinline__ float axis_weight(float f, int b) {
  return __fsub_rn(1.0f, fabsf(b ? __fsub_rn(f, 1.0f) : f));
}
// sign(-(f - b)) as in enmesh.py:155 (0 exactly at f == b).
__device__ __forceinline__ float axis_sign(float f, int b) {
  float d = b ? __fsub_rn(f, 1.0f) : f;
  return d < 0.0f ? 1.0f : (d > 0.0f ? -1.0f : 0.0f);
}

// Correctly rounded arithmetic and math of the float32 kernels and of their
// float64 instantiations (the reference's x64 build), so one kernel source
// serves both precisions with the float path unchanged.
template <class T>
struct Real;
template <>
struct Real<float> {
  using T2 = float2;
  __device__ static __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
  __device__ static __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
  __device__ static __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
  __device__ static __forceinline__ float div(float a, float b) { return __fdiv_rn(a, b); }
  __device__ static __forceinline__ float sqrt_(float a) { return sqrtf(a); }
  __device__ static __forceinline__ float log_(float a) { return logf(a); }
  __device__ static __forceinline__ float cos_(float a) { return cosf(a); }
  __device__ static __forceinline__ float sin_(float a) { return sinf(a); }
  __device__ static __forceinline__ float floor_(float a) { return floorf(a); }
  __device__ static __forceinline__ float fabs_(float a) { return fabsf(a); }
  __device__ static __forceinline__ float rint_(float a) { return rintf(a); }
  __device__ static __forceinline__ float pow_(float a, float b) { return powf(a, b); }
  __device__ static __forceinline__ float2 make2(float a, float b) { return make_float2(a, b); }
};
template <>
struct Real<double> {
  using T2 = double2;
  __device__ static __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
  __device__ static __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
  __device__ static __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
  __device__ static __forceinline__ double div(double a, double b) { return __ddiv_rn(a, b); }
  __device__ static __forceinline__ double sqrt_(double a) { return sqrt(a); }
  __device__ static __forceinline__ double log_(double a) { return log(a); }
  __device__ static __forceinline__ double cos_(double a) { return cos(a); }
  __device__ static __forceinline__ double sin_(double a) { return sin(a); }
  __device__ static __forceinline__ double floor_(double a) { return floor(a); }
  __device__ static __forceinline__ double fabs_(double a) { return fabs(a); }
  __device__ static __forceinline__ double rint_(double a) { return rint(a); }
  __device__ static __forceinline__ double pow_(double a, double b) { return pow(a, b); }
  __device__ static __forceinline__ double2 make2(double a, double b) { return make_double2(a, b); }
};

// Sorted particle record: fractions along x, y, z and the raveled lower cell.
struct __align__(16) Rec {
  float fx, fy, fz;
  uint32_t key;
};

// Spectral description of one mesh: per-axis wavenumbers, the derivative
// factors c (neg_ik = i c, Nyquist zeroed) and the optional particle-Nyquist
// masks, all in float precision, built on the host with the reference
// formulas (numerics/fft.py:4-44, core/configuration.py:365-376,
// core/utils.py:15-37).
struct SpecTables {
  const float* kx;
  const float* ky;
  const float* kz;
  const float* cx;
  const float* cy;
  const float* cz;
  const float* mx;  // may be null (mesh == particle grid)
  const float* my;
  const float* mz;
};

// Table layout [kx ky kz cx cy cz (mx my mz)] (kz, cz, mz of length nz/2+1)
// as built by the host configuration.
inline SpecTables spec_tables_from(const float* t, Mesh3 m, int has_masks) {
  const int nzh = m.nz / 2 + 1;
  SpecTables s;
  s.kx = t;
  s.ky = s.kx + m.nx;
  s.kz = s.ky + m.ny;
  s.cx = s.kz + nzh;
  s.cy = s.cx + m.nx;
  s.cz = s.cy + m.ny;
  if (has_masks) {
    s.mx = s.cz + nzh;
    s.my = s.mx + m.nx;
    s.mz = s.my + m.ny;
  } else {
    s.mx = s.my = s.mz = nullptr;
  }
  return s;
}

// Scale of the fixed-point deposit: pow2e / 2^ceil(log2 amax), the largest
// power of two with scale * amax <= pow2e, so val * w * scale is exact in
// float and rounding it to an integer is the only rounding (1.0 for a zero or
// negative amax).
__host__ __device__ inline double fixed_point_scale(double pow2e, float amax) {
  if (!(amax > 0.f)) return 1.0;
  int x = 0;
  const double m = frexp((double)amax, &x);  // amax = m 2^x, m in [0.5, 1)
  return ldexp(pow2e, m == 0.5 ? 1 - x : -x);
}

// Floats in one spectral table of mesh m.
inline int64_t spec_table_len(Mesh3 m, int has_masks) {
  const int64_t nzh = m.nz / 2 + 1;
  return (has_masks ? 3 : 2) * ((int64_t)m.nx + m.ny + nzh);
}

}  // namespace pmb

#define PMB_CUDA_CHECK(expr)                         \
  do {                                               \
    cudaError_t _e = (expr);                         \
    if (_e != cudaSuccess) {                         \
      pmb::set_last_error(cudaGetErrorString(_e));   \
      return pmb::kCudaError;                        \
    }                                                \
  } while (0)

namespace pmb {
void set_last_error(const char* msg);

// Raises kernel fn's dynamic shared-memory limit to at least `bytes` on the
// current device.  The attribute belongs to the device's context, so it is
// tracked per (device, kernel): a process may drive several GPUs.  Thread-safe.
inline cudaError_t smem_optin(const void* fn, int bytes) {
  static std::mutex mu;
  static std::map<std::pair<int, const void*>, int> done;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lock(mu);
  int& have = done[std::make_pair(dev, fn)];
  if (have >= bytes) return cudaSuccess;
  e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e == cudaSuccess) have = bytes;
  return e;
}
}
