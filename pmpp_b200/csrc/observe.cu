// Forward observers: windowed periodic projections of a density mesh
// (nbody/observers.py:18-56 density_projection_observer, :82-126 the saved
// maps of nbody_kappa; core/utils.py:420-463 wraparound_slice).
//
// out = sum over the window t = 0 .. count-1 of mesh[(start + t) mod n_axis]
// along one axis, count = min(stop - start, max_width) (0 when stop <= start),
// for every cell of the other two axes.  Each output cell is summed by one
// thread (axes 0 and 1, coalesced over the contiguous z axis) or one warp
// (axis 2, lanes striding z, then a fixed shuffle tree), in FP64 and in a
// fixed order: the projections are deterministic.  One read of the window's
// planes, one write of the map: HBM-bound.
#include "pmb_kernels.cuh"

namespace pmb {

__global__ void project_outer_kernel(const float* __restrict__ mesh, float* __restrict__ out, int64_t plane,
                                     int n_axis, int start, int count, int64_t n_out) {
  // axis 0: plane = ny nz -> out (ny, nz); axis 1: plane = nz, the outer
  // stride ny nz = plane * n_axis -> out (nx, nz)
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n_out; j += (int64_t)gridDim.x * blockDim.x) {
    const int64_t hi = j / plane, lo = j - hi * plane;
    const float* base = mesh + hi * plane * n_axis + lo;
    double acc = 0.0;
    int i = start % n_axis;
    if (i < 0) i += n_axis;
    for (int t = 0; t < count; ++t) {
      acc += (double)base[(int64_t)i * plane];
      if (++i == n_axis) i = 0;
    }
    out[j] = (float)acc;
  }
}

__global__ void project_z_kernel(const float* __restrict__ mesh, float* __restrict__ out, int nz, int start,
                                 int count, int64_t rows) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  int s0 = start % nz;
  if (s0 < 0) s0 += nz;
  for (int64_t r = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < rows; r += warps) {
    const float* row = mesh + r * nz;
    double acc = 0.0;
    for (int t = lane; t < count; t += 32) {
      int i = s0 + t;
      i -= (i / nz) * nz;
      acc += (double)row[i];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) out[r] = (float)acc;
  }
}

int project_window(const float* mesh, Mesh3 m, int axis, int start, int stop, int max_width, float* out,
                   cudaStream_t s) {
  int count = stop - start;
  if (max_width >= 0 && count > max_width) count = max_width;
  if (count < 0) count = 0;
  const int th = 256;
  if (axis == 0 || axis == 1) {
    const int64_t plane = axis == 0 ? (int64_t)m.ny * m.nz : (int64_t)m.nz;
    const int n_axis = axis == 0 ? m.nx : m.ny;
    const int64_t n_out = axis == 0 ? (int64_t)m.ny * m.nz : (int64_t)m.nx * m.nz;
    int64_t b = (n_out + th - 1) / th;
    if (b > 148 * 16) b = 148 * 16;
    project_outer_kernel<<<(unsigned)(b > 0 ? b : 1), th, 0, s>>>(mesh, out, plane, n_axis, start, count, n_out);
  } else {
    const int64_t rows = (int64_t)m.nx * m.ny;
    int64_t b = (rows * 32 + th - 1) / th;
    if (b > 148 * 16) b = 148 * 16;
    project_z_kernel<<<(unsigned)(b > 0 ? b : 1), th, 0, s>>>(mesh, out, m.nz, start, count, rows);
  }
  PMB_CUDA_CHECK(cudaGetLastError());
  return kOk;
}

}  // namespace pmb
