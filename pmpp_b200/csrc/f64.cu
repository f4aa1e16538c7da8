// float64 build of the PM path (the reference's x64 configuration): nested
// white noise, linear modes, 2LPT, the PM force with drift / kick, and P(k),
// all in double precision with cuFFT D2Z / Z2D.
//
// Reference semantics are those of the float32 kernels (cic/enmesh.py:139-162,
// cic/scatter.py:315-338, cic/gather.py:452-472, nbody/gravity.py:283-399,
// 626-633, initial_conditions/lpt.py:337-449, analysis/power_spectrum.py:
// 106-143) evaluated in float64.  This build is for parity at float64
// precision, not for speed: the deposit adds the eight corner weights with
// double-precision atomics straight into the density (no sort), and the
// gather reads the corners directly; the float32 kernels are the optimised
// hot path.
#include <cmath>

#include "../../include/pmb200.h"
#include "pmb_common.cuh"
#include "pmb_ic.cuh"
#include "pmb_kernels.cuh"

namespace pmb {
namespace {

using RD = Real<double>;

unsigned grid_for(int64_t total, int th) {
  int64_t b = (total + th - 1) / th;
  const int64_t cap = 148 * 32;
  return (unsigned)(b < cap ? (b > 0 ? b : 1) : cap);
}

struct Cell64 {
  int c[3];
  double f[3];
};

// Lower corner and fractions in float64 (enmesh.py:139-147); org is the mesh
// origin's offset within a cell (the interlaced deposit's cell / 2,
// cic/enmesh.py:128-147), subtracted before the division.
__device__ __forceinline__ Cell64 bin64(const int16_t* __restrict__ pmid, const double* __restrict__ disp, int64_t i,
                                       Mesh3 m, double cell, double org = 0.0) {
  Cell64 r;
  const int dims[3] = {m.nx, m.ny, m.nz};
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const double q = RD::div(org != 0.0 ? RD::sub(disp[3 * i + a], org) : disp[3 * i + a], cell);
    const double l = floor(q);
    r.f[a] = RD::sub(q, l);
    r.c[a] = pmod((int)pmid[3 * i + a] + (int)l, dims[a]);
  }
  return r;
}

__device__ __forceinline__ double w64(double f, int b) { return RD::sub(1.0, fabs(b ? RD::sub(f, 1.0) : f)); }

// Optional drift disp += vel * D, then the CIC deposit of val per particle.
__global__ void deposit64_kernel(const int16_t* __restrict__ pmid, double* __restrict__ disp,
                                 const double* __restrict__ vel, double drift, int64_t n, Mesh3 m, double cell,
                                 double val, double* __restrict__ rho, double org = 0.0) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    if (vel != nullptr) {
#pragma unroll
      for (int a = 0; a < 3; ++a) disp[3 * i + a] = RD::add(disp[3 * i + a], RD::mul(vel[3 * i + a], drift));
    }
    const Cell64 b = bin64(pmid, disp, i, m, cell, org);
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const int bx = k & 1, by = (k >> 1) & 1, bz = (k >> 2) & 1;
      const int x = bx ? (b.c[0] + 1 == m.nx ? 0 : b.c[0] + 1) : b.c[0];
      const int y = by ? (b.c[1] + 1 == m.ny ? 0 : b.c[1] + 1) : b.c[1];
      const int z = bz ? (b.c[2] + 1 == m.nz ? 0 : b.c[2] + 1) : b.c[2];
      const double w = RD::mul(RD::mul(w64(b.f[0], bx), w64(b.f[1], by)), w64(b.f[2], bz));
      atomicAdd(&rho[((int64_t)x * m.ny + y) * m.nz + z], RD::mul(val, w));
    }
  }
}

// rho -> (rho - 1) * src_mul (gravity.py:628-630)
__global__ void source64_kernel(double* __restrict__ rho, int64_t n, double src_mul) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    rho[i] = RD::mul(RD::sub(rho[i], 1.0), src_mul);
}

struct Tables64 {
  const double *kx, *ky, *kz, *cx, *cy, *cz, *mx, *my, *mz;
};

// Green x gradient in float64: phi = -(S mask) / k^2 * T, grad_d = (i c_d) phi,
// 1/M folded in; T the correction's transfer per half-spectrum cell
// (corrections/core.py:333-334), none when transfer is null.
__global__ void green64_kernel(const double2* __restrict__ src, double2* __restrict__ grad, Mesh3 m, Tables64 t,
                               double post, const double* __restrict__ transfer) {
  const int nzh = m.nz / 2 + 1;
  const int64_t total = m.half_cells();
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < total; j += (int64_t)gridDim.x * blockDim.x) {
    const int iz = (int)(j % nzh);
    const int64_t r = j / nzh;
    const int iy = (int)(r % m.ny), ix = (int)(r / m.ny);
    double2 v = src[j];
    if (t.mx != nullptr) {
      const double mk = RD::mul(RD::mul(t.mx[ix], t.my[iy]), t.mz[iz]);
      v.x = RD::mul(v.x, mk);
      v.y = RD::mul(v.y, mk);
    }
    const double k2 = RD::add(RD::add(RD::mul(t.kx[ix], t.kx[ix]), RD::mul(t.ky[iy], t.ky[iy])),
                              RD::mul(t.kz[iz], t.kz[iz]));
    double pr = 0.0, pi = 0.0;
    if (k2 != 0.0) {
      pr = RD::div(-v.x, k2);
      pi = RD::div(-v.y, k2);
      if (transfer != nullptr) {
        pr = RD::mul(pr, transfer[j]);
        pi = RD::mul(pi, transfer[j]);
      }
    }
    const double c[3] = {t.cx[ix], t.cy[iy], t.cz[iz]};
#pragma unroll
    for (int d = 0; d < 3; ++d)
      grad[(int64_t)d * total + j] = make_double2(RD::mul(-RD::mul(c[d], pi), post), RD::mul(RD::mul(c[d], pr), post));
  }
}

// acc = CIC gather of the three force meshes; optional vel += acc * kick.
__global__ void gather64_kernel(const int16_t* __restrict__ pmid, const double* __restrict__ disp, int64_t n, Mesh3 m,
                                double cell, const double* __restrict__ mesh, double* __restrict__ acc,
                                double* __restrict__ vel, double kick) {
  const int64_t cells = m.cells();
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const Cell64 b = bin64(pmid, disp, i, m, cell);
    double a[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const int bx = k & 1, by = (k >> 1) & 1, bz = (k >> 2) & 1;
      const int x = bx ? (b.c[0] + 1 == m.nx ? 0 : b.c[0] + 1) : b.c[0];
      const int y = by ? (b.c[1] + 1 == m.ny ? 0 : b.c[1] + 1) : b.c[1];
      const int z = bz ? (b.c[2] + 1 == m.nz ? 0 : b.c[2] + 1) : b.c[2];
      const double w = RD::mul(RD::mul(w64(b.f[0], bx), w64(b.f[1], by)), w64(b.f[2], bz));
      const int64_t idx = ((int64_t)x * m.ny + y) * m.nz + z;
#pragma unroll
      for (int d = 0; d < 3; ++d) a[d] = RD::add(a[d], RD::mul(mesh[(int64_t)d * cells + idx], w));
    }
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      acc[3 * i + d] = a[d];
      if (vel != nullptr) vel[3 * i + d] = RD::add(vel[3 * i + d], RD::mul(a[d], kick));
    }
  }
}

// sign(-(f - b)) as in enmesh.py:155 (0 exactly at f == b).
__device__ __forceinline__ double sign64(double f, int b) {
  const double d = b ? RD::sub(f, 1.0) : f;
  return d < 0.0 ? 1.0 : (d > 0.0 ? -1.0 : 0.0);
}

// Position term of the CIC adjoints in float64 (gather.py:495-502 with u the
// value cotangent, scatter.py:366-370 with u the deposited value):
//   disp_cot += sum_b (sum_c u_c mesh_c[i_b]) grad w_b / cell,
//   grad_i w_b = sign(-(f_i - b_i)) w_{i+1} w_{i+2} (enmesh.py:155-160).
// u: (N, C) per particle, or u_const when null.
template <int C>
__global__ void interp_grad64_kernel(const int16_t* __restrict__ pmid, const double* __restrict__ disp, int64_t n,
                                     Mesh3 m, double cell, const double* __restrict__ mesh,
                                     const double* __restrict__ u, double u_const, double* __restrict__ disp_cot,
                                     double org = 0.0) {
  const int64_t cells = m.cells();
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const Cell64 b = bin64(pmid, disp, i, m, cell, org);
    double uu[C];
#pragma unroll
    for (int c = 0; c < C; ++c) uu[c] = u ? u[i * C + c] : u_const;
    double w[3][2], sg[3][2];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      w[a][0] = w64(b.f[a], 0);
      w[a][1] = w64(b.f[a], 1);
      sg[a][0] = sign64(b.f[a], 0);
      sg[a][1] = sign64(b.f[a], 1);
    }
    double g[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const int bx = k & 1, by = (k >> 1) & 1, bz = (k >> 2) & 1;
      const int x = bx ? (b.c[0] + 1 == m.nx ? 0 : b.c[0] + 1) : b.c[0];
      const int y = by ? (b.c[1] + 1 == m.ny ? 0 : b.c[1] + 1) : b.c[1];
      const int z = bz ? (b.c[2] + 1 == m.nz ? 0 : b.c[2] + 1) : b.c[2];
      const int64_t idx = ((int64_t)x * m.ny + y) * m.nz + z;
      double inner = 0.0;
#pragma unroll
      for (int c = 0; c < C; ++c) inner = RD::add(inner, RD::mul(uu[c], mesh[(int64_t)c * cells + idx]));
      g[0] = RD::add(g[0], RD::mul(inner, RD::mul(RD::mul(sg[0][bx], w[1][by]), w[2][bz])));
      g[1] = RD::add(g[1], RD::mul(inner, RD::mul(RD::mul(sg[1][by], w[2][bz]), w[0][bx])));
      g[2] = RD::add(g[2], RD::mul(inner, RD::mul(RD::mul(sg[2][bz], w[0][bx]), w[1][by])));
    }
#pragma unroll
    for (int a = 0; a < 3; ++a) disp_cot[3 * i + a] = RD::add(disp_cot[3 * i + a], RD::div(g[a], cell));
  }
}

// CIC deposit of per-particle C-vectors (the acceleration cotangents) into C
// planar float64 meshes (cic/scatter.py:275-281), double atomics.
template <int C>
__global__ void deposit64v_kernel(const int16_t* __restrict__ pmid, const double* __restrict__ disp, int64_t n, Mesh3 m,
                                  double cell, const double* __restrict__ val, double* __restrict__ out) {
  const int64_t cells = m.cells();
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const Cell64 b = bin64(pmid, disp, i, m, cell);
    double v[C];
#pragma unroll
    for (int c = 0; c < C; ++c) v[c] = val[i * C + c];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const int bx = k & 1, by = (k >> 1) & 1, bz = (k >> 2) & 1;
      const int x = bx ? (b.c[0] + 1 == m.nx ? 0 : b.c[0] + 1) : b.c[0];
      const int y = by ? (b.c[1] + 1 == m.ny ? 0 : b.c[1] + 1) : b.c[1];
      const int z = bz ? (b.c[2] + 1 == m.nz ? 0 : b.c[2] + 1) : b.c[2];
      const double w = RD::mul(RD::mul(w64(b.f[0], bx), w64(b.f[1], by)), w64(b.f[2], bz));
      const int64_t idx = ((int64_t)x * m.ny + y) * m.nz + z;
#pragma unroll
      for (int c = 0; c < C; ++c) atomicAdd(&out[(int64_t)c * cells + idx], RD::mul(v[c], w));
    }
  }
}

// Transpose of green64_kernel (gravity.py:226-260, 290-321):
// src_cot = post * mask * (-1/k^2) * T * sum_d conj(i c_d) A_d, zero at k = 0.
__global__ void green64_adjoint_kernel(const double2* __restrict__ gc, double2* __restrict__ out, Mesh3 m, Tables64 t,
                                       double post, const double* __restrict__ transfer) {
  const int nzh = m.nz / 2 + 1;
  const int64_t total = m.half_cells();
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < total; j += (int64_t)gridDim.x * blockDim.x) {
    const int iz = (int)(j % nzh);
    const int64_t r = j / nzh;
    const int iy = (int)(r % m.ny), ix = (int)(r / m.ny);
    const double c[3] = {t.cx[ix], t.cy[iy], t.cz[iz]};
    double sr = 0.0, si = 0.0;  // sum_d (-i c_d) A_d
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const double2 a = gc[(int64_t)d * total + j];
      sr = RD::add(sr, RD::mul(c[d], a.y));
      si = RD::sub(si, RD::mul(c[d], a.x));
    }
    const double k2 = RD::add(RD::add(RD::mul(t.kx[ix], t.kx[ix]), RD::mul(t.ky[iy], t.ky[iy])),
                              RD::mul(t.kz[iz], t.kz[iz]));
    double pr = 0.0, pi = 0.0;
    if (k2 != 0.0) {
      if (transfer != nullptr) {
        sr = RD::mul(sr, transfer[j]);
        si = RD::mul(si, transfer[j]);
      }
      pr = RD::div(-sr, k2);
      pi = RD::div(-si, k2);
    }
    if (t.mx != nullptr) {
      const double mk = RD::mul(RD::mul(t.mx[ix], t.my[iy]), t.mz[iz]);
      pr = RD::mul(pr, mk);
      pi = RD::mul(pi, mk);
    }
    out[j] = make_double2(RD::mul(pr, post), RD::mul(pi, post));
  }
}

// Interlaced source spectrum (gravity.py:440-463): mode 0 s0 = (s0 + s1 P) / 2
// with P = exp(-i (kx + ky + kz) cell / 2) = exp(-i pi (nx/Nx + ny/Ny + nz/Nz))
// over the signed mode numbers of the half spectrum; mode 1 its transpose from
// the cotangent c held in s0: s1 = conj(P) c / 2, s0 = c / 2.
__global__ void interlace64_kernel(double2* __restrict__ s0, double2* __restrict__ s1, Mesh3 m, int mode) {
  const int nzh = m.nz / 2 + 1;
  const int64_t total = m.half_cells();
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < total; j += (int64_t)gridDim.x * blockDim.x) {
    const int iz = (int)(j % nzh);
    const int64_t r = j / nzh;
    const int iy = (int)(r % m.ny), ix = (int)(r / m.ny);
    const int kx = ix < (m.nx + 1) / 2 ? ix : ix - m.nx, ky = iy < (m.ny + 1) / 2 ? iy : iy - m.ny;
    const double t = RD::add(RD::add(RD::div((double)kx, (double)m.nx), RD::div((double)ky, (double)m.ny)),
                             RD::div((double)iz, (double)m.nz));
    double sn, cs;
    sincospi(t, &sn, &cs);
    if (mode == 0) {
      const double2 a = s0[j], b = s1[j];
      const double pr = RD::add(RD::mul(b.x, cs), RD::mul(b.y, sn)), pim = RD::sub(RD::mul(b.y, cs), RD::mul(b.x, sn));
      s0[j] = make_double2(RD::mul(0.5, RD::add(a.x, pr)), RD::mul(0.5, RD::add(a.y, pim)));
    } else {
      const double2 c = s0[j];
      s1[j] = make_double2(RD::mul(0.5, RD::sub(RD::mul(c.x, cs), RD::mul(c.y, sn))),
                           RD::mul(0.5, RD::add(RD::mul(c.y, cs), RD::mul(c.x, sn))));
      s0[j] = make_double2(RD::mul(0.5, c.x), RD::mul(0.5, c.y));
    }
  }
}

__global__ void dot64_kernel(const double* __restrict__ a, const double* __restrict__ b, int64_t n,
                             double* __restrict__ out) {
  double s = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    s = fma(a[i], b[i], s);
  for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xFFFFFFFFu, s, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(out, s);
}

__global__ void axpy64_kernel(double* __restrict__ y, const double* __restrict__ x, int64_t n, double f) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    y[i] = RD::add(y[i], RD::mul(x[i], f));
}

__global__ void sum64_kernel(const double* __restrict__ a, int64_t n, double* __restrict__ out) {
  double s = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    s += a[i];
  for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xFFFFFFFFu, s, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(out, s);
}

struct Carve64 {
  char* base;
  int64_t off = 0;
  explicit Carve64(void* b) : base((char*)b) {}
  void* take(int64_t bytes) {
    void* p = base ? base + off : nullptr;
    off += align_up(bytes, 256);
    return p;
  }
};

// Interlaced forms (il) hold two source meshes and spectra: the regular and
// the half-cell-shifted deposit's.
int64_t force64_layout(Mesh3 m, void* ws, double** rho, double2** rho_hat, double2** grad_hat, void** work,
                       bool il = false) {
  Carve64 c(ws);
  const int ns = il ? 2 : 1;
  *rho = (double*)c.take(8 * ns * m.cells());
  *rho_hat = (double2*)c.take(16 * ns * m.half_cells());
  *grad_hat = (double2*)c.take(48 * m.half_cells());
  const int64_t w3 = fft_work_bytes64(m, 3), ws_ = fft_work_bytes64(m, ns);
  if (w3 < 0 || ws_ < 0) return -1;
  *work = c.take(w3 > ws_ ? w3 : ws_);
  return c.off;
}

int64_t force_vjp64_layout(Mesh3 m, void* ws, double** mesh3, double2** spec3, double2** spec1, void** work,
                           bool il = false) {
  Carve64 c(ws);
  const int ns = il ? 2 : 1;
  *mesh3 = (double*)c.take(24 * m.cells());
  *spec3 = (double2*)c.take(48 * m.half_cells());
  *spec1 = (double2*)c.take(16 * ns * m.half_cells());
  const int64_t w3 = fft_work_bytes64(m, 3), ws_ = fft_work_bytes64(m, ns);
  if (w3 < 0 || ws_ < 0) return -1;
  *work = c.take(w3 > ws_ ? w3 : ws_);
  return c.off;
}

int64_t lpt64_layout(Mesh3 g, void* ws, double2** pot1, double2** spec6, double** real6, double** L, double2** Lhat,
                     void** work) {
  Carve64 c(ws);
  const int64_t ng = g.cells(), mc = g.half_cells();
  *pot1 = (double2*)c.take(16 * mc);
  *spec6 = (double2*)c.take(96 * mc);
  *real6 = (double*)c.take(48 * ng);
  *L = (double*)c.take(8 * ng);
  *Lhat = (double2*)c.take(16 * mc);
  const int64_t w6 = fft_work_bytes64(g, 6), w1 = fft_work_bytes64(g, 1);
  if (w6 < 0 || w1 < 0) return -1;
  *work = c.take(w6 > w1 ? w6 : w1);
  return c.off;
}

int64_t lpt_vjp64_layout(Mesh3 g, void* ws, double** cot6, double2** F6, double2** Lhat, double** L, double2** pot1,
                         double2** spec6, double** real6, void** work) {
  Carve64 c(ws);
  const int64_t ng = g.cells(), mc = g.half_cells();
  *cot6 = (double*)c.take(48 * ng);
  *F6 = (double2*)c.take(96 * mc);
  *Lhat = (double2*)c.take(16 * mc);
  *L = (double*)c.take(8 * ng);
  *pot1 = (double2*)c.take(16 * mc);
  *spec6 = (double2*)c.take(96 * mc);
  *real6 = (double*)c.take(48 * ng);
  const int64_t w6 = fft_work_bytes64(g, 6), w1 = fft_work_bytes64(g, 1);
  if (w6 < 0 || w1 < 0) return -1;
  *work = c.take(w6 > w1 ? w6 : w1);
  return c.off;
}

Tables64 tables64(const double* t, Mesh3 m, int has_masks) {
  const int nzh = m.nz / 2 + 1;
  Tables64 s;
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

#define F64_REQUIRE(cond, msg) \
  do {                         \
    if (!(cond)) {             \
      set_last_error(msg);     \
      return kInvalidArgument; \
    }                          \
  } while (0)

#define F64_TRY(expr)            \
  do {                           \
    int _st = (expr);            \
    if (_st != kOk) return _st;  \
  } while (0)

inline cudaStream_t S(void* s) { return reinterpret_cast<cudaStream_t>(s); }

bool valid64(int nx, int ny, int nz) { return nx > 0 && ny > 0 && nz > 0 && (double)nx * ny * nz < 4294967296.0; }

}  // namespace
}  // namespace pmb

using namespace pmb;

extern "C" {

int64_t pmb_force64_workspace_bytes(int nx, int ny, int nz) {
  double* r;
  double2 *rh, *gh;
  void* w;
  return force64_layout(Mesh3{nx, ny, nz}, nullptr, &r, &rh, &gh, &w);
}

static int force64_impl(const int16_t* pmid, double* disp, const double* drift_vel, double drift, int64_t n, int nx,
                        int ny, int nz, double cell, double val, double src_mul, const double* tables, int has_masks,
                        const double* transfer, double* force_meshes, double* acc, double* vel_kick, double kick,
                        void* workspace, int64_t workspace_bytes, void* stream, bool il) {
  Mesh3 m{nx, ny, nz};
  F64_REQUIRE(valid64(nx, ny, nz), "pmb_force64: unsupported mesh shape");
  F64_REQUIRE(n >= 0 && cell > 0.0, "pmb_force64: bad particle count or cell size");
  double* rho;
  double2 *rho_hat, *grad_hat;
  void* work;
  const int64_t need = force64_layout(m, workspace, &rho, &rho_hat, &grad_hat, &work, il);
  F64_REQUIRE(need >= 0, "pmb_force64: cuFFT plan creation failed");
  if (need > workspace_bytes) {
    set_last_error("pmb_force64: workspace too small");
    return kScratchTooSmall;
  }
  cudaStream_t s = S(stream);
  const int ns = il ? 2 : 1;
  PMB_CUDA_CHECK(cudaMemsetAsync(rho, 0, 8 * ns * m.cells(), s));
  if (n > 0) deposit64_kernel<<<grid_for(n, 256), 256, 0, s>>>(pmid, disp, drift_vel, drift, n, m, cell, val, rho);
  if (n > 0 && il)  // the deposit on the mesh shifted by half a cell (gravity.py:446-463), drifted positions
    deposit64_kernel<<<grid_for(n, 256), 256, 0, s>>>(pmid, disp, nullptr, 0.0, n, m, cell, val, rho + m.cells(),
                                                      0.5 * cell);
  source64_kernel<<<grid_for(ns * m.cells(), 256), 256, 0, s>>>(rho, ns * m.cells(), src_mul);
  PMB_CUDA_CHECK(cudaGetLastError());
  F64_TRY(fft_d2z(m, ns, rho, rho_hat, work, s));
  if (il) interlace64_kernel<<<grid_for(m.half_cells(), 256), 256, 0, s>>>(rho_hat, rho_hat + m.half_cells(), m, 0);
  green64_kernel<<<grid_for(m.half_cells(), 256), 256, 0, s>>>(rho_hat, grad_hat, m, tables64(tables, m, has_masks),
                                                               1.0 / (double)m.cells(), transfer);
  PMB_CUDA_CHECK(cudaGetLastError());
  F64_TRY(fft_z2d(m, 3, grad_hat, force_meshes, work, s));
  if (n > 0) gather64_kernel<<<grid_for(n, 256), 256, 0, s>>>(pmid, disp, n, m, cell, force_meshes, acc, vel_kick, kick);
  PMB_CUDA_CHECK(cudaGetLastError());
  return kOk;
}

int pmb_force64(const int16_t* pmid, double* disp, const double* drift_vel, double drift, int64_t n, int nx, int ny,
                int nz, double cell, double val, double src_mul, const double* tables, int has_masks,
                const double* transfer, double* force_meshes, double* acc, double* vel_kick, double kick,
                void* workspace, int64_t workspace_bytes, void* stream) {
  return force64_impl(pmid, disp, drift_vel, drift, n, nx, ny, nz, cell, val, src_mul, tables, has_masks, transfer,
                      force_meshes, acc, vel_kick, kick, workspace, workspace_bytes, stream, false);
}

int64_t pmb_force64_interlaced_workspace_bytes(int nx, int ny, int nz) {
  double* r;
  double2 *rh, *gh;
  void* w;
  return force64_layout(Mesh3{nx, ny, nz}, nullptr, &r, &rh, &gh, &w, true);
}

int pmb_force64_interlaced(const int16_t* pmid, double* disp, const double* drift_vel, double drift, int64_t n, int nx,
                           int ny, int nz, double cell, double val, double src_mul, const double* tables,
                           int has_masks, const double* transfer, double* force_meshes, double* acc, double* vel_kick,
                           double kick, void* workspace, int64_t workspace_bytes, void* stream) {
  return force64_impl(pmid, disp, drift_vel, drift, n, nx, ny, nz, cell, val, src_mul, tables, has_masks, transfer,
                      force_meshes, acc, vel_kick, kick, workspace, workspace_bytes, stream, true);
}

int64_t pmb_force_vjp64_workspace_bytes(int nx, int ny, int nz) {
  double* m3;
  double2 *s3, *s1;
  void* w;
  return force_vjp64_layout(Mesh3{nx, ny, nz}, nullptr, &m3, &s3, &s1, &w);
}

static int force_vjp64_impl(const int16_t* pmid, const double* disp, int64_t n, int nx, int ny, int nz, double cell,
                            double val, double src_mul, const double* tables, int has_masks, const double* transfer,
                            const double* force_meshes, const double* acc_cot, double* disp_cot, void* workspace,
                            int64_t workspace_bytes, void* stream, bool il) {
  Mesh3 m{nx, ny, nz};
  F64_REQUIRE(valid64(nx, ny, nz), "pmb_force_vjp64: unsupported mesh shape");
  F64_REQUIRE(n >= 0 && n < 4294967296ll && cell > 0.0, "pmb_force_vjp64: bad particle count or cell size");
  F64_REQUIRE(n == 0 || (pmid && disp && force_meshes && acc_cot && disp_cot), "pmb_force_vjp64: null buffer");
  double* mesh3;
  double2 *spec3, *spec1;
  void* work;
  const int64_t need = force_vjp64_layout(m, workspace, &mesh3, &spec3, &spec1, &work, il);
  F64_REQUIRE(need >= 0, "pmb_force_vjp64: cuFFT plan creation failed");
  if (need > workspace_bytes) {
    set_last_error("pmb_force_vjp64: workspace too small");
    return kScratchTooSmall;
  }
  cudaStream_t s = S(stream);
  if (n > 0)  // gather adjoint, position term (gather.py:495-502)
    interp_grad64_kernel<3><<<grid_for(n, 256), 256, 0, s>>>(pmid, disp, n, m, cell, force_meshes, acc_cot, 0.0,
                                                             disp_cot);
  PMB_CUDA_CHECK(cudaMemsetAsync(mesh3, 0, 24 * m.cells(), s));
  if (n > 0)  // gather adjoint, mesh term: deposit of the cotangents
    deposit64v_kernel<3><<<grid_for(n, 256), 256, 0, s>>>(pmid, disp, n, m, cell, acc_cot, mesh3);
  PMB_CUDA_CHECK(cudaGetLastError());
  F64_TRY(fft_d2z(m, 3, mesh3, spec3, work, s));
  green64_adjoint_kernel<<<grid_for(m.half_cells(), 256), 256, 0, s>>>(spec3, spec1, m, tables64(tables, m, has_masks),
                                                                       src_mul / (double)m.cells(), transfer);
  // interlaced: split the source cotangent between the two deposits
  if (il) interlace64_kernel<<<grid_for(m.half_cells(), 256), 256, 0, s>>>(spec1, spec1 + m.half_cells(), m, 1);
  PMB_CUDA_CHECK(cudaGetLastError());
  F64_TRY(fft_z2d(m, il ? 2 : 1, spec1, mesh3, work, s));
  if (n > 0)  // scatter adjoint, position term (scatter.py:366-370)
    interp_grad64_kernel<1><<<grid_for(n, 256), 256, 0, s>>>(pmid, disp, n, m, cell, mesh3, nullptr, val, disp_cot);
  if (n > 0 && il)  // the shifted deposit's adjoint on its own mesh
    interp_grad64_kernel<1><<<grid_for(n, 256), 256, 0, s>>>(pmid, disp, n, m, cell, mesh3 + m.cells(), nullptr, val,
                                                             disp_cot, 0.5 * cell);
  PMB_CUDA_CHECK(cudaGetLastError());
  return kOk;
}

int pmb_force_vjp64(const int16_t* pmid, const double* disp, int64_t n, int nx, int ny, int nz, double cell,
                    double val, double src_mul, const double* tables, int has_masks, const double* transfer,
                    const double* force_meshes, const double* acc_cot, double* disp_cot, void* workspace,
                    int64_t workspace_bytes, void* stream) {
  return force_vjp64_impl(pmid, disp, n, nx, ny, nz, cell, val, src_mul, tables, has_masks, transfer, force_meshes,
                          acc_cot, disp_cot, workspace, workspace_bytes, stream, false);
}

int64_t pmb_force_vjp64_interlaced_workspace_bytes(int nx, int ny, int nz) {
  double* m3;
  double2 *s3, *s1;
  void* w;
  return force_vjp64_layout(Mesh3{nx, ny, nz}, nullptr, &m3, &s3, &s1, &w, true);
}

int pmb_force_vjp64_interlaced(const int16_t* pmid, const double* disp, int64_t n, int nx, int ny, int nz,
                               double cell, double val, double src_mul, const double* tables, int has_masks,
                               const double* transfer, const double* force_meshes, const double* acc_cot,
                               double* disp_cot, void* workspace, int64_t workspace_bytes, void* stream) {
  return force_vjp64_impl(pmid, disp, n, nx, ny, nz, cell, val, src_mul, tables, has_masks, transfer, force_meshes,
                          acc_cot, disp_cot, workspace, workspace_bytes, stream, true);
}

int pmb_dot64(const double* a, const double* b, int64_t n, double* out, void* stream) {
  F64_REQUIRE(out != nullptr && n >= 0, "pmb_dot64: bad arguments");
  if (n > 0) dot64_kernel<<<grid_for(n, 256), 256, 0, S(stream)>>>(a, b, n, out);
  PMB_CUDA_CHECK(cudaGetLastError());
  return kOk;
}

int pmb_deposit64(const int16_t* pmid, const double* disp, int64_t n, int nx, int ny, int nz, double cell, double val,
                  double* rho, void* stream) {
  F64_REQUIRE(valid64(nx, ny, nz), "pmb_deposit64: unsupported mesh shape");
  cudaStream_t s = S(stream);
  const Mesh3 m{nx, ny, nz};
  PMB_CUDA_CHECK(cudaMemsetAsync(rho, 0, 8 * m.cells(), s));
  if (n > 0)
    deposit64_kernel<<<grid_for(n, 256), 256, 0, s>>>(pmid, const_cast<double*>(disp), nullptr, 0.0, n, m, cell, val,
                                                      rho);
  PMB_CUDA_CHECK(cudaGetLastError());
  return kOk;
}

int pmb_axpy64(double* y, const double* x, int64_t n, double f, void* stream) {
  if (n > 0) axpy64_kernel<<<grid_for(n, 256), 256, 0, S(stream)>>>(y, x, n, f);
  PMB_CUDA_CHECK(cudaGetLastError());
  return kOk;
}

int pmb_sum64(const double* a, int64_t n, double* out, void* stream) {
  cudaStream_t s = S(stream);
  PMB_CUDA_CHECK(cudaMemsetAsync(out, 0, sizeof(double), s));
  if (n > 0) sum64_kernel<<<grid_for(n, 256), 256, 0, s>>>(a, n, out);
  PMB_CUDA_CHECK(cudaGetLastError());
  return kOk;
}

int64_t pmb_fft64_work_bytes(int nx, int ny, int nz, int batch) { return fft_work_bytes64(Mesh3{nx, ny, nz}, batch); }

int pmb_rfft3_64(int nx, int ny, int nz, int batch, double* in, void* out, void* work, void* stream) {
  F64_REQUIRE(valid64(nx, ny, nz) && batch > 0, "pmb_rfft3_64: bad shape");
  return fft_d2z(Mesh3{nx, ny, nz}, batch, in, (double2*)out, work, S(stream));
}

int pmb_irfft3_64(int nx, int ny, int nz, int batch, void* in, double* out, void* work, void* stream) {
  F64_REQUIRE(valid64(nx, ny, nz) && batch > 0, "pmb_irfft3_64: bad shape");
  return fft_z2d(Mesh3{nx, ny, nz}, batch, (double2*)in, out, work, S(stream));
}

int pmb_white_noise_nested64(uint32_t seed, int gx, int gy, int gz, void* out, void* stream) {
  F64_REQUIRE(valid64(gx, gy, gz), "pmb_white_noise_nested64: bad grid");
  return white_noise64(seed, Mesh3{gx, gy, gz}, (double2*)out, S(stream));
}

int pmb_linear_modes64(const void* modes_in, void* modes_out, int gx, int gy, int gz, const double* kvec,
                       const double* tk, const double* tt, int ntab, double A_s, double n_s, double omega_m,
                       double k_pivot, double growth2, double box_vol, void* stream) {
  F64_REQUIRE(valid64(gx, gy, gz) && ntab >= 2, "pmb_linear_modes64: bad arguments");
  LinearPowerParams p;  // as pmb_linear_modes (boltzmann.py:428-484)
  const double c_light = 299792458.0 / 1e5;
  p.coef = 0.32 * A_s * k_pivot;
  p.k_pivot = k_pivot;
  p.n_s = n_s;
  p.pi_c2_over_om = M_PI * c_light * c_light / omega_m;
  p.growth2 = growth2;
  p.box_vol = box_vol;
  return linear_modes64((const double2*)modes_in, (double2*)modes_out, Mesh3{gx, gy, gz}, kvec, tk, tt, ntab, p,
                        S(stream));
}

int64_t pmb_lpt64_workspace_bytes(int gx, int gy, int gz) {
  double2 *a, *b, *e;
  double *c, *d;
  void* w;
  return lpt64_layout(Mesh3{gx, gy, gz}, nullptr, &a, &b, &c, &d, &e, &w);
}

int pmb_lpt64(const void* modes, int gx, int gy, int gz, double spacing, double cell_vol, const double* tables,
              int order, double D1, double V1, double D2, double V2, const int16_t* pmid, double* disp, double* vel,
              int64_t n, double cell, double* fields, void* workspace, int64_t workspace_bytes, void* stream) {
  return pmb_lpt64_ex(modes, gx, gy, gz, spacing, cell_vol, tables, order, D1, V1, D2, V2, pmid, disp, vel, n, cell,
                      fields, nullptr, workspace, workspace_bytes, stream);
}

int pmb_lpt64_ex(const void* modes, int gx, int gy, int gz, double spacing, double cell_vol, const double* tables,
                 int order, double D1, double V1, double D2, double V2, const int16_t* pmid, double* disp,
                 double* vel, int64_t n, double cell, double* fields, int64_t* index_out, void* workspace,
                 int64_t workspace_bytes, void* stream) {
  Mesh3 g{gx, gy, gz};
  F64_REQUIRE(valid64(gx, gy, gz), "pmb_lpt64: bad grid");
  F64_REQUIRE(order >= 0 && order <= 2, "pmb_lpt64: order must be 0, 1 or 2");
  double2 *pot1, *spec6, *Lhat;
  double *real6, *L;
  void* work;
  const int64_t need = lpt64_layout(g, workspace, &pot1, &spec6, &real6, &L, &Lhat, &work);
  F64_REQUIRE(need >= 0, "pmb_lpt64: cuFFT plan creation failed");
  if (need > workspace_bytes) {
    set_last_error("pmb_lpt64: workspace too small");
    return kScratchTooSmall;
  }
  cudaStream_t s = S(stream);
  const double inv_n = 1.0 / (double)g.cells();
  F64_TRY(lpt_strains64((const double2*)modes, 1.0 / cell_vol, pot1, spec6, g, tables, inv_n, s));
  const double2* Lh = nullptr;
  if (order >= 2) {
    F64_TRY(fft_z2d(g, 6, spec6, real6, work, s));
    F64_TRY(lpt_source64(real6, L, g.cells(), s));
    F64_TRY(fft_d2z(g, 1, L, Lhat, work, s));
    Lh = Lhat;
  }
  F64_TRY(lpt_gradients64(pot1, Lh, spec6, g, tables, inv_n, s));
  F64_TRY(fft_z2d(g, 6, spec6, fields, work, s));
  return lpt_displace64(pmid, disp, vel, n, g, cell, spacing, fields, order, D1, V1, D2, V2, index_out, s);
}

int64_t pmb_lpt_vjp64_workspace_bytes(int gx, int gy, int gz) {
  double *a, *l, *r;
  double2 *f, *lh, *p, *sp;
  void* w;
  return lpt_vjp64_layout(Mesh3{gx, gy, gz}, nullptr, &a, &f, &lh, &l, &p, &sp, &r, &w);
}

int pmb_lpt_vjp64(const void* modes, int gx, int gy, int gz, double cell_vol, const double* tables, int order,
                  double D1, double V1, double D2, double V2, const int64_t* index, const double* fields,
                  const double* disp_cot, const double* vel_cot, int64_t n, const double* amp, void* modes_cot,
                  double* dots, void* workspace, int64_t workspace_bytes, void* stream) {
  Mesh3 g{gx, gy, gz};
  F64_REQUIRE(valid64(gx, gy, gz), "pmb_lpt_vjp64: bad grid");
  F64_REQUIRE(order >= 1 && order <= 2, "pmb_lpt_vjp64: order must be 1 or 2");
  F64_REQUIRE(dots != nullptr && index != nullptr, "pmb_lpt_vjp64: dots and index required");
  double *cot6, *L, *real6;
  double2 *F6, *Lhat, *pot1, *spec6;
  void* work;
  const int64_t need = lpt_vjp64_layout(g, workspace, &cot6, &F6, &Lhat, &L, &pot1, &spec6, &real6, &work);
  F64_REQUIRE(need >= 0, "pmb_lpt_vjp64: cuFFT plan creation failed");
  if (need > workspace_bytes) {
    set_last_error("pmb_lpt_vjp64: workspace too small");
    return kScratchTooSmall;
  }
  cudaStream_t s = S(stream);
  const int64_t ng = g.cells();
  const double inv_n = 1.0 / (double)ng;
  PMB_CUDA_CHECK(cudaMemsetAsync(cot6, 0, 48 * ng, s));
  F64_TRY(lpt_field_cot64(index, disp_cot, vel_cot, n, ng, fields, order, D1, V1, D2, V2, cot6, dots, s));
  F64_TRY(fft_d2z(g, 6, cot6, F6, work, s));
  const double2* FS = nullptr;
  if (order >= 2) {
    F64_TRY(lpt_grad2_adjoint64(F6 + 3 * g.half_cells(), Lhat, g, tables, inv_n, s));
    F64_TRY(fft_z2d(g, 1, Lhat, L, work, s));
    F64_TRY(lpt_strains64((const double2*)modes, 1.0 / cell_vol, pot1, spec6, g, tables, inv_n, s));
    F64_TRY(fft_z2d(g, 6, spec6, real6, work, s));
    F64_TRY(lpt_source_adjoint64(real6, L, cot6, ng, s));
    F64_TRY(fft_d2z(g, 6, cot6, spec6, work, s));
    FS = spec6;
  }
  return lpt_modes_adjoint64(F6, FS, amp, (double2*)modes_cot, g, tables, 1.0 / (cell_vol * (double)ng), s);
}

int pmb_scatter_vjp64(const int16_t* pmid, const double* disp, int64_t n, int nx, int ny, int nz, double cell,
                      double val, const double* mesh_cot, double* disp_cot, void* stream) {
  Mesh3 m{nx, ny, nz};
  F64_REQUIRE(valid64(nx, ny, nz), "pmb_scatter_vjp64: unsupported mesh shape");
  F64_REQUIRE(n >= 0 && n < 4294967296ll && cell > 0.0, "pmb_scatter_vjp64: bad particle count or cell size");
  F64_REQUIRE(n == 0 || (pmid && disp && mesh_cot && disp_cot), "pmb_scatter_vjp64: null buffer");
  if (n > 0)
    interp_grad64_kernel<1><<<grid_for(n, 256), 256, 0, S(stream)>>>(pmid, disp, n, m, cell, mesh_cot, nullptr, val,
                                                                     disp_cot);
  PMB_CUDA_CHECK(cudaGetLastError());
  return kOk;
}

int pmb_pk_shells64(const void* spec, int nx, int ny, int nz, const double* sinc_tab, int mas_power, int num_shells,
                    double* sums, void* stream) {
  F64_REQUIRE(valid64(nx, ny, nz) && num_shells > 0, "pmb_pk_shells64: bad arguments");
  cudaStream_t s = S(stream);
  PMB_CUDA_CHECK(cudaMemsetAsync(sums, 0, sizeof(double) * num_shells, s));
  return pk_shells64((const double2*)spec, Mesh3{nx, ny, nz}, sinc_tab, mas_power, num_shells, sums, s);
}

int pmb_pk_shells_adjoint64(const void* spec, int nx, int ny, int nz, const double* sinc_tab, int mas_power,
                            int num_shells, const double* wshell, double post, void* out, void* stream) {
  F64_REQUIRE(valid64(nx, ny, nz) && num_shells > 0, "pmb_pk_shells_adjoint64: bad arguments");
  F64_REQUIRE(spec && sinc_tab && wshell && out, "pmb_pk_shells_adjoint64: null buffer");
  return pk_shells_adjoint64((const double2*)spec, Mesh3{nx, ny, nz}, sinc_tab, mas_power, num_shells, wshell, post,
                             (double2*)out, S(stream));
}

int pmb_overdensity64(const double* rho, double* delta, int64_t n, const double* total, void* stream) {
  return overdensity64(rho, delta, n, total, S(stream));
}

}  // extern "C"
