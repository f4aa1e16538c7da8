// extern "C" entry points of libpmb200.so (declared in include/pmb200.h).
#include <cstdio>
#include <cstring>
#include <string>

#include "../../include/pmb200.h"
#include "pmb_common.cuh"
#include "pmb_integrate.cuh"
#include "pmb_kernels.cuh"
#include "pmb_sort.cuh"

namespace pmb {
namespace {
thread_local std::string g_last_error = "no error";
}
void set_last_error(const char* msg) { g_last_error = msg ? msg : "unknown error"; }
}  // namespace pmb

using namespace pmb;

namespace {

inline cudaStream_t S(void* s) { return reinterpret_cast<cudaStream_t>(s); }

bool valid_mesh(int nx, int ny, int nz) {
  if (nx < 1 || ny < 1 || nz < 1 || nz > 4096) return false;
  // the sorted record stores the raveled cell key in 32 bits
  return (double)nx * ny * nz < 4294967296.0;
}

#define PMB_REQUIRE(cond, msg)          \
  do {                                  \
    if (!(cond)) {                      \
      set_last_error(msg);              \
      return kInvalidArgument;          \
    }                                   \
  } while (0)

#define PMB_TRY(expr)            \
  do {                           \
    int _st = (expr);            \
    if (_st != kOk) return _st;  \
  } while (0)

struct SortedView {
  Rec* rec;
  uint32_t* perm;
  uint32_t* offs;
};

SortedView sorted_view(void* sorted, int64_t n) {
  char* p = (char*)sorted;
  SortedView v;
  v.rec = (Rec*)p;
  p += align_up(16 * n, 256);
  v.perm = (uint32_t*)p;
  p += align_up(4 * n, 256);
  v.offs = (uint32_t*)p;
  return v;
}

int64_t sorted_bytes(int64_t n, Mesh3 m) { return align_up(16 * n, 256) + align_up(4 * n, 256) + align_up(4 * (m.rows() + 1), 256); }

SpecTables make_tables(const float* t, Mesh3 m, int has_masks) {
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

GreenParams make_green(int green_kernel, const float* transfer, const float* radial, int radial_len, float post_scale) {
  GreenParams g;
  g.green_kernel = green_kernel;
  g.cell = 0.f;
  g.transfer = transfer;
  g.radial = radial;
  g.radial_len = radial_len;
  g.post_scale = post_scale;
  return g;
}

// Carves consecutive 256-byte aligned regions out of a caller workspace.
struct Carve {
  char* base;
  int64_t off = 0;
  int64_t cap;
  Carve(void* b, int64_t c) : base((char*)b), cap(c) {}
  void* take(int64_t bytes) {
    void* p = base ? base + off : nullptr;
    off += align_up(bytes, 256);
    return p;
  }
  bool ok() const { return off <= cap; }
};

}  // namespace

extern "C" {

int pmb_abi_version(void) { return 1; }

const char* pmb_last_error(void) { return g_last_error.c_str(); }

int64_t pmb_sorted_bytes(int64_t n, int nx, int ny, int nz) { return sorted_bytes(n, Mesh3{nx, ny, nz}); }

int64_t pmb_sort_scratch_bytes(int64_t n, int nx, int ny, int nz) { return bin_scratch_bytes(n, Mesh3{nx, ny, nz}); }

int pmb_sort_rows(const int16_t* pmid, float* disp, const float* vel, float drift, int64_t n, int nx, int ny, int nz,
                  float cell, void* sorted, void* scratch, int64_t scratch_bytes, void* stream) {
  Mesh3 m{nx, ny, nz};
  PMB_REQUIRE(valid_mesh(nx, ny, nz), "pmb_sort_rows: unsupported mesh shape");
  PMB_REQUIRE(n >= 0 && n < 4294967295ll, "pmb_sort_rows: particle count out of range");
  PMB_REQUIRE(cell > 0.f, "pmb_sort_rows: cell size must be positive");
  PMB_REQUIRE(scratch_bytes >= bin_scratch_bytes(n, m), "pmb_sort_rows: scratch too small");
  SortedView v = sorted_view(sorted, n);
  return bin_particles(pmid, disp, vel, drift, n, m, cell, v.rec, v.perm, v.offs, scratch, S(stream));
}

int pmb_scatter_rows(const void* sorted, int64_t n, int nx, int ny, int nz, int C, const float* val, float val_const,
                     int mode, float src_mul, float* out, void* scratch16, void* stream) {
  Mesh3 m{nx, ny, nz};
  PMB_REQUIRE(valid_mesh(nx, ny, nz), "pmb_scatter_rows: unsupported mesh shape");
  PMB_REQUIRE(C >= 1 && C <= 4, "pmb_scatter_rows: 1..4 channels supported");
  PMB_REQUIRE(mode == 0 || mode == 1, "pmb_scatter_rows: mode must be 0 or 1");
  SortedView v = sorted_view((void*)sorted, n);
  double* scale = (double*)scratch16;
  unsigned int* tmp = (unsigned int*)((char*)scratch16 + 8);
  if (val != nullptr) {
    PMB_TRY(compute_scale(val, n * C, n, scale, tmp, S(stream)));
  } else {
    float a = fabsf(val_const);
    PMB_REQUIRE(a < INFINITY, "pmb_scatter_rows: non-finite value");
    PMB_TRY(set_double(scale, a > 0.f ? fixed_point_pow2(n) / (double)a : 1.0, S(stream)));
  }
  return scatter_sorted(v.rec, v.perm, v.offs, m, C, val, val_const, scale, mode, src_mul, out, S(stream));
}

int pmb_gather_rows(const void* sorted, int64_t n, int nx, int ny, int nz, int C, const float* mesh, float* out,
                    float* vel, float kick, void* stream) {
  Mesh3 m{nx, ny, nz};
  PMB_REQUIRE(valid_mesh(nx, ny, nz), "pmb_gather_rows: unsupported mesh shape");
  PMB_REQUIRE(C >= 1 && C <= 4, "pmb_gather_rows: 1..4 channels supported");
  SortedView v = sorted_view((void*)sorted, n);
  return gather_sorted(v.rec, v.perm, n, m, C, mesh, out, vel, kick, S(stream));
}

int pmb_interp_grad_rows(const void* sorted, int64_t n, int nx, int ny, int nz, int C, const float* mesh,
                         const float* u, float u_const, float cell, int accumulate, float* disp_cot, float* wsum,
                         void* stream) {
  Mesh3 m{nx, ny, nz};
  PMB_REQUIRE(valid_mesh(nx, ny, nz), "pmb_interp_grad_rows: unsupported mesh shape");
  PMB_REQUIRE(C >= 1 && C <= 4, "pmb_interp_grad_rows: 1..4 channels supported");
  SortedView v = sorted_view((void*)sorted, n);
  return interp_grad_sorted(v.rec, v.perm, n, m, C, mesh, u, u_const, cell, accumulate, disp_cot, wsum, S(stream));
}

int64_t pmb_fft_work_bytes(int nx, int ny, int nz, int batch) { return fft_work_bytes(Mesh3{nx, ny, nz}, batch); }

int pmb_rfft3(int nx, int ny, int nz, int batch, float* in, void* out, void* work, void* stream) {
  PMB_REQUIRE(nx > 0 && ny > 0 && nz > 0 && batch > 0, "pmb_rfft3: bad shape");
  return fft_r2c(Mesh3{nx, ny, nz}, batch, in, (float2*)out, work, S(stream));
}

int pmb_irfft3(int nx, int ny, int nz, int batch, void* in, float* out, void* work, void* stream) {
  PMB_REQUIRE(nx > 0 && ny > 0 && nz > 0 && batch > 0, "pmb_irfft3: bad shape");
  return fft_c2r(Mesh3{nx, ny, nz}, batch, (float2*)in, out, work, S(stream));
}

int pmb_green_gradient(const void* src_hat, void* grad_hat, int nx, int ny, int nz, const float* tables, int has_masks,
                       int green_kernel, const float* transfer, const float* radial, int radial_len, float post_scale,
                       void* stream) {
  Mesh3 m{nx, ny, nz};
  PMB_REQUIRE(nx > 0 && ny > 0 && nz > 0, "pmb_green_gradient: bad shape");
  PMB_REQUIRE(green_kernel == 0 || green_kernel == 1, "pmb_green_gradient: unknown Green's function");
  return green_gradient((const float2*)src_hat, (float2*)grad_hat, m, make_tables(tables, m, has_masks),
                        make_green(green_kernel, transfer, radial, radial_len, post_scale), S(stream));
}

int pmb_green_gradient_adjoint(const void* grad_cot_hat, void* src_cot_hat, int nx, int ny, int nz,
                               const float* tables, int has_masks, int green_kernel, const float* transfer,
                               const float* radial, int radial_len, float post_scale, void* stream) {
  Mesh3 m{nx, ny, nz};
  PMB_REQUIRE(nx > 0 && ny > 0 && nz > 0, "pmb_green_gradient_adjoint: bad shape");
  PMB_REQUIRE(green_kernel == 0 || green_kernel == 1, "pmb_green_gradient_adjoint: unknown Green's function");
  return green_gradient_adjoint((const float2*)grad_cot_hat, (float2*)src_cot_hat, m,
                                make_tables(tables, m, has_masks),
                                make_green(green_kernel, transfer, radial, radial_len, post_scale), S(stream));
}

// ---------------------------------------------------------------------------
// Fused force
// ---------------------------------------------------------------------------
static int64_t force_layout(int64_t n, Mesh3 m, void* ws, int64_t cap, void** sorted, void** bin_scratch,
                            void** scale16, float** src, float2** src_hat, float2** grad_hat, void** fft_work) {
  Carve c(ws, cap);
  *sorted = c.take(sorted_bytes(n, m));
  *bin_scratch = c.take(bin_scratch_bytes(n, m));
  *scale16 = c.take(16);
  *src = (float*)c.take(4 * m.cells());
  *src_hat = (float2*)c.take(8 * m.half_cells());
  *grad_hat = (float2*)c.take(24 * m.half_cells());
  int64_t w = fft_work_bytes(m, 3);
  int64_t w1 = fft_work_bytes(m, 1);
  if (w < 0 || w1 < 0) return -1;
  *fft_work = c.take(w > w1 ? w : w1);
  return c.off;
}

int64_t pmb_force_workspace_bytes(int64_t n, int nx, int ny, int nz) {
  void *a, *b, *c, *f;
  float* s;
  float2 *sh, *gh;
  return force_layout(n, Mesh3{nx, ny, nz}, nullptr, 0, &a, &b, &c, &s, &sh, &gh, &f);
}

int pmb_force(const int16_t* pmid, float* disp, const float* drift_vel, float drift, int64_t n, int nx, int ny, int nz,
              float cell, float val_const, float src_mul, const float* tables, int has_masks, int green_kernel,
              const float* transfer, const float* radial, int radial_len, float* force_meshes, float* acc,
              float* vel_kick, float kick, void* workspace, int64_t workspace_bytes, void* stream) {
  Mesh3 m{nx, ny, nz};
  PMB_REQUIRE(valid_mesh(nx, ny, nz), "pmb_force: unsupported mesh shape");
  PMB_REQUIRE(n >= 0 && n < 4294967295ll, "pmb_force: particle count out of range");
  PMB_REQUIRE(cell > 0.f, "pmb_force: cell size must be positive");
  void *sorted, *bins, *scale16, *work;
  float* src;
  float2 *src_hat, *grad_hat;
  int64_t need = force_layout(n, m, workspace, workspace_bytes, &sorted, &bins, &scale16, &src, &src_hat, &grad_hat, &work);
  PMB_REQUIRE(need >= 0, "pmb_force: cuFFT plan creation failed");
  if (need > workspace_bytes) {
    set_last_error("pmb_force: workspace too small");
    return kScratchTooSmall;
  }
  cudaStream_t s = S(stream);
  PMB_TRY(pmb_sort_rows(pmid, disp, drift_vel, drift, n, nx, ny, nz, cell, sorted, bins, bin_scratch_bytes(n, m), stream));
  PMB_TRY(pmb_scatter_rows(sorted, n, nx, ny, nz, 1, nullptr, val_const, 1, src_mul, src, scale16, stream));
  PMB_TRY(fft_r2c(m, 1, src, src_hat, work, s));
  const float inv_m = (float)(1.0 / (double)m.cells());
  PMB_TRY(green_gradient(src_hat, grad_hat, m, make_tables(tables, m, has_masks),
                         make_green(green_kernel, transfer, radial, radial_len, inv_m), s));
  PMB_TRY(fft_c2r(m, 3, grad_hat, force_meshes, work, s));
  SortedView v = sorted_view(sorted, n);
  return gather_sorted(v.rec, v.perm, n, m, 3, force_meshes, acc, vel_kick, kick, s);
}

static int64_t force_vjp_layout(int64_t n, Mesh3 m, void* ws, int64_t cap, void** sorted, void** bins, void** scale16,
                                float** mesh_cot, float2** spec3, float2** src_hat, float** src_cot, void** work) {
  Carve c(ws, cap);
  *sorted = c.take(sorted_bytes(n, m));
  *bins = c.take(bin_scratch_bytes(n, m));
  *scale16 = c.take(16);
  *mesh_cot = (float*)c.take(12 * m.cells());
  *spec3 = (float2*)c.take(24 * m.half_cells());
  *src_hat = (float2*)c.take(8 * m.half_cells());
  *src_cot = (float*)c.take(4 * m.cells());
  int64_t w = fft_work_bytes(m, 3);
  int64_t w1 = fft_work_bytes(m, 1);
  if (w < 0 || w1 < 0) return -1;
  *work = c.take(w > w1 ? w : w1);
  return c.off;
}

int64_t pmb_force_vjp_workspace_bytes(int64_t n, int nx, int ny, int nz) {
  void *a, *b, *c, *w;
  float *mc, *sc;
  float2 *s3, *sh;
  return force_vjp_layout(n, Mesh3{nx, ny, nz}, nullptr, 0, &a, &b, &c, &mc, &s3, &sh, &sc, &w);
}

int pmb_force_vjp(const int16_t* pmid, const float* disp, int64_t n, int nx, int ny, int nz, float cell,
                  float val_const, float src_mul, const float* tables, int has_masks, int green_kernel,
                  const float* transfer, const float* radial, int radial_len, const float* force_meshes,
                  const float* acc_cot, float* disp_cot, void* workspace, int64_t workspace_bytes, void* stream) {
  Mesh3 m{nx, ny, nz};
  PMB_REQUIRE(valid_mesh(nx, ny, nz), "pmb_force_vjp: unsupported mesh shape");
  PMB_REQUIRE(n >= 0 && n < 4294967295ll, "pmb_force_vjp: particle count out of range");
  PMB_REQUIRE(cell > 0.f, "pmb_force_vjp: cell size must be positive");
  void *sorted, *bins, *scale16, *work;
  float *mesh_cot, *src_cot;
  float2 *spec3, *src_hat;
  int64_t need = force_vjp_layout(n, m, workspace, workspace_bytes, &sorted, &bins, &scale16, &mesh_cot, &spec3,
                                  &src_hat, &src_cot, &work);
  PMB_REQUIRE(need >= 0, "pmb_force_vjp: cuFFT plan creation failed");
  if (need > workspace_bytes) {
    set_last_error("pmb_force_vjp: workspace too small");
    return kScratchTooSmall;
  }
  cudaStream_t s = S(stream);
  PMB_TRY(pmb_sort_rows(pmid, (float*)disp, nullptr, 0.f, n, nx, ny, nz, cell, sorted, bins, bin_scratch_bytes(n, m),
                        stream));
  SortedView v = sorted_view(sorted, n);
  // gather adjoint: position term and the 3-channel scatter of acc_cot
  PMB_TRY(interp_grad_sorted(v.rec, v.perm, n, m, 3, force_meshes, acc_cot, 0.f, cell, 1, disp_cot, nullptr, s));
  PMB_TRY(pmb_scatter_rows(sorted, n, nx, ny, nz, 3, acc_cot, 0.f, 0, 1.f, mesh_cot, scale16, stream));
  // transposes of the C2R, gradient, Green and R2C stages
  PMB_TRY(fft_r2c(m, 3, mesh_cot, spec3, work, s));
  const float post = (float)((double)src_mul / (double)m.cells());
  PMB_TRY(green_gradient_adjoint(spec3, src_hat, m, make_tables(tables, m, has_masks),
                                 make_green(green_kernel, transfer, radial, radial_len, post), s));
  PMB_TRY(fft_c2r(m, 1, src_hat, src_cot, work, s));
  // scatter adjoint of the density (constant particle value)
  return interp_grad_sorted(v.rec, v.perm, n, m, 1, src_cot, nullptr, val_const, cell, 1, disp_cot, nullptr, s);
}

// ---------------------------------------------------------------------------
// Integration
// ---------------------------------------------------------------------------
int pmb_axpy(float* y, const float* x, int64_t n, float f, void* stream) { return axpy(y, x, n, f, S(stream)); }

int pmb_kick_adj(float* vel, const float* acc, const float* vel_cot, float* acc_cot, int64_t n, float kick,
                 double* dot, void* stream) {
  PMB_REQUIRE(dot != nullptr, "pmb_kick_adj: dot accumulator required");
  return kick_adj(vel, acc, vel_cot, acc_cot, n, kick, dot, S(stream));
}

int pmb_drift_adj(float* disp, const float* vel, const float* disp_cot, float* vel_cot, int64_t n, float drift,
                  double* dot, void* stream) {
  PMB_REQUIRE(dot != nullptr, "pmb_drift_adj: dot accumulator required");
  return drift_adj(disp, vel, disp_cot, vel_cot, n, drift, dot, S(stream));
}

int pmb_dot(const float* a, const float* b, int64_t n, double* out, void* stream) {
  PMB_REQUIRE(out != nullptr, "pmb_dot: output required");
  return dot(a, b, n, out, S(stream));
}

// ---------------------------------------------------------------------------
// Stable per-cell sort
// ---------------------------------------------------------------------------
int64_t pmb_sort_by_cell_scratch_bytes(int64_t n, int nx, int ny, int nz) {
  return radix_scratch_bytes(n);
}

int pmb_sort_by_cell(const int16_t* pmid, const float* disp, int64_t n, int nx, int ny, int nz, float cell,
                     uint32_t* keys_out, uint32_t* perm_out, void* scratch, int64_t scratch_bytes, void* stream) {
  Mesh3 m{nx, ny, nz};
  PMB_REQUIRE(valid_mesh(nx, ny, nz), "pmb_sort_by_cell: unsupported mesh shape");
  PMB_REQUIRE(n >= 0 && n < 4294967295ll, "pmb_sort_by_cell: particle count out of range");
  PMB_REQUIRE(cell > 0.f, "pmb_sort_by_cell: cell size must be positive");
  PMB_REQUIRE(scratch_bytes >= radix_scratch_bytes(n), "pmb_sort_by_cell: scratch too small");
  return sort_by_cell(pmid, disp, n, m, cell, keys_out, perm_out, scratch, S(stream));
}

}  // extern "C"
