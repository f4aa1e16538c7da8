// extern "C" entry points of libpmb200.so (declared in include/pmb200.h).
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>

#include "../../include/pmb200.h"
#include "pmb_cic_device.cuh"
#include "pmb_common.cuh"
#include "pmb_ic.cuh"
#include "pmb_integrate.cuh"
#include "pmb_kernels.cuh"
#include "pmb_mlp.cuh"
#include "pmb_sort.cuh"
#include "pmb_tma.cuh"

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

// Sorted buffer: records, permutation, row offsets and a status word (the
// DeviceFlag bits the sort raised).
struct SortedView {
  Rec* rec;
  uint32_t* perm;
  uint32_t* offs;
  uint32_t* status;
};

SortedView sorted_view(void* sorted, int64_t n, Mesh3 m) {
  char* p = (char*)sorted;
  SortedView v;
  v.rec = (Rec*)p;
  p += align_up(16 * n, 256);
  v.perm = (uint32_t*)p;
  p += align_up(4 * n, 256);
  v.offs = (uint32_t*)p;
  p += align_up(4 * (m.rows() + 1), 256);
  v.status = (uint32_t*)p;
  return v;
}

int64_t sorted_bytes(int64_t n, Mesh3 m) {
  return align_up(16 * n, 256) + align_up(4 * n, 256) + align_up(4 * (m.rows() + 1), 256) + 256;
}

SpecTables make_tables(const float* t, Mesh3 m, int has_masks) { return spec_tables_from(t, m, has_masks); }

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

int pmb_abi_version(void) { return 3; }

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
  SortedView v = sorted_view(sorted, n, m);
  return bin_particles(pmid, disp, vel, drift, n, m, cell, v.rec, v.perm, v.offs, scratch, S(stream), nullptr,
                       nullptr, v.status);
}

int pmb_sort_rows_ex(const int16_t* pmid, float* disp, const float* vel, float drift, int64_t n, int nx, int ny,
                     int nz, float cell, float ox, float oy, float oz, const uint8_t* valid, void* sorted,
                     void* scratch, int64_t scratch_bytes, void* stream) {
  Mesh3 m{nx, ny, nz};
  PMB_REQUIRE(valid_mesh(nx, ny, nz), "pmb_sort_rows_ex: unsupported mesh shape");
  PMB_REQUIRE(n >= 0 && n < 4294967295ll, "pmb_sort_rows_ex: particle count out of range");
  PMB_REQUIRE(cell > 0.f, "pmb_sort_rows_ex: cell size must be positive");
  PMB_REQUIRE(std::isfinite(ox) && std::isfinite(oy) && std::isfinite(oz), "pmb_sort_rows_ex: non-finite offset");
  PMB_REQUIRE(scratch_bytes >= bin_scratch_bytes(n, m), "pmb_sort_rows_ex: scratch too small");
  // whole cells and remainder of the offset, the remainder rounded once to float
  BinShift sh;
  const float o[3] = {ox, oy, oz};
  int q[3];
  float r[3];
  for (int a = 0; a < 3; ++a) {
    const double qd = std::floor((double)o[a] / (double)cell);
    PMB_REQUIRE(std::fabs(qd) < 1e9, "pmb_sort_rows_ex: offset too large");
    q[a] = (int)qd;
    r[a] = (float)((double)o[a] - qd * (double)cell);
  }
  sh.qx = q[0];
  sh.qy = q[1];
  sh.qz = q[2];
  sh.rx = r[0];
  sh.ry = r[1];
  sh.rz = r[2];
  SortedView v = sorted_view(sorted, n, m);
  return bin_particles(pmid, disp, vel, drift, n, m, cell, v.rec, v.perm, v.offs, scratch, S(stream), &sh, valid,
                       v.status);
}

int pmb_scatter_rows(const void* sorted, int64_t n, int nx, int ny, int nz, int C, const float* val, int val_sorted,
                     float val_const, int mode, float src_mul, float* out, void* scratch16, void* stream) {
  Mesh3 m{nx, ny, nz};
  PMB_REQUIRE(valid_mesh(nx, ny, nz), "pmb_scatter_rows: unsupported mesh shape");
  PMB_REQUIRE(n >= 0 && n < 4294967295ll, "pmb_scatter_rows: particle count out of range");
  PMB_REQUIRE(C >= 1 && C <= 4, "pmb_scatter_rows: 1..4 channels supported");
  PMB_REQUIRE(mode == 0 || mode == 1, "pmb_scatter_rows: mode must be 0 or 1");
  SortedView v = sorted_view((void*)sorted, n, m);
  double* scale = (double*)scratch16;
  unsigned int* tmp = (unsigned int*)((char*)scratch16 + 8);
  if (val != nullptr) {
    PMB_TRY(compute_scale(val, n * C, n, scale, tmp, S(stream)));
  } else {
    float a = fabsf(val_const);
    PMB_REQUIRE(a < INFINITY, "pmb_scatter_rows: non-finite value");
    PMB_TRY(set_double(scale, fixed_point_scale(fixed_point_pow2(n), a), S(stream)));
  }
  return scatter_sorted(v.rec, v.perm, v.offs, m, C, val, val_sorted, val_const, scale, mode, src_mul, out,
                        S(stream), n, v.status);
}

int pmb_gather_rows2(const void* sorted, int64_t n, int nx, int ny, int nz, int C, const float* mesh, float* out,
                     float* vel, float kick, float kick2, void* stream) {
  Mesh3 m{nx, ny, nz};
  PMB_REQUIRE(valid_mesh(nx, ny, nz), "pmb_gather_rows: unsupported mesh shape");
  PMB_REQUIRE(n >= 0 && n < 4294967295ll, "pmb_gather_rows: particle count out of range");
  PMB_REQUIRE(C >= 1 && C <= 4, "pmb_gather_rows: 1..4 channels supported");
  PMB_REQUIRE(out != nullptr || vel != nullptr, "pmb_gather_rows: out may be null only with vel");
  SortedView v = sorted_view((void*)sorted, n, m);
  return gather_sorted(v.rec, v.perm, v.offs, n, m, C, mesh, out, vel, kick, kick2, S(stream), v.status);
}

int pmb_gather_rows(const void* sorted, int64_t n, int nx, int ny, int nz, int C, const float* mesh, float* out,
                    float* vel, float kick, void* stream) {
  return pmb_gather_rows2(sorted, n, nx, ny, nz, C, mesh, out, vel, kick, 0.f, stream);
}

int pmb_interp_grad_rows(const void* sorted, int64_t n, int nx, int ny, int nz, int C, const float* mesh,
                         const float* u, float u_const, float cell, int accumulate, float* disp_cot, float* wsum,
                         float* u_sorted, void* stream) {
  Mesh3 m{nx, ny, nz};
  PMB_REQUIRE(valid_mesh(nx, ny, nz), "pmb_interp_grad_rows: unsupported mesh shape");
  PMB_REQUIRE(n >= 0 && n < 4294967295ll, "pmb_interp_grad_rows: particle count out of range");
  PMB_REQUIRE(C >= 1 && C <= 4, "pmb_interp_grad_rows: 1..4 channels supported");
  SortedView v = sorted_view((void*)sorted, n, m);
  return interp_grad_sorted(v.rec, v.perm, v.offs, n, m, C, mesh, u, u_const, cell, accumulate, disp_cot, wsum,
                            u_sorted, S(stream), v.status);
}

// ---------------------------------------------------------------------------
// CIC onto a mesh of another cell size
// ---------------------------------------------------------------------------
static int general_grid(int gx, int gy, int gz, float cell, float ox, float oy, float oz, float cell2, int nx, int ny,
                        int nz, GeneralGrid* G) {
  PMB_REQUIRE(gx > 0 && gy > 0 && gz > 0 && cell > 0.f && cell2 > 0.f, "pmb_cic_general: bad particle grid");
  PMB_REQUIRE(valid_mesh(nx, ny, nz), "pmb_cic_general: unsupported mesh shape");
  PMB_REQUIRE(std::isfinite(ox) && std::isfinite(oy) && std::isfinite(oz), "pmb_cic_general: non-finite offset");
  G->gx = gx;
  G->gy = gy;
  G->gz = gz;
  G->a1 = cell;
  G->a2 = cell2;
  G->ox = ox;
  G->oy = oy;
  G->oz = oz;
  G->t = Mesh3{nx, ny, nz};
  return kOk;
}

int64_t pmb_cic_general_scratch_bytes(int nx, int ny, int nz, int C) {
  return general_scatter_scratch_bytes(Mesh3{nx, ny, nz}, C);
}

int pmb_cic_general_scatter(const int16_t* pmid, const float* disp, const uint8_t* valid, int64_t n, int gx, int gy,
                            int gz, float cell, float ox, float oy, float oz, float cell2, int nx, int ny, int nz,
                            int C, const float* val, float val_const, float* out, void* scratch,
                            int64_t scratch_bytes, void* stream) {
  GeneralGrid G;
  PMB_TRY(general_grid(gx, gy, gz, cell, ox, oy, oz, cell2, nx, ny, nz, &G));
  PMB_REQUIRE(n >= 0 && C >= 1 && C <= 4, "pmb_cic_general_scatter: bad particle count or channels");
  PMB_REQUIRE(val != nullptr || std::isfinite(val_const), "pmb_cic_general_scatter: non-finite value");
  if (scratch_bytes < general_scatter_scratch_bytes(G.t, C)) {
    set_last_error("pmb_cic_general_scatter: scratch too small");
    return kScratchTooSmall;
  }
  return general_scatter(pmid, disp, valid, n, G, C, val, val_const, out, scratch, S(stream));
}

int pmb_cic_general_gather(const int16_t* pmid, const float* disp, const uint8_t* valid, int64_t n, int gx, int gy,
                           int gz, float cell, float ox, float oy, float oz, float cell2, int nx, int ny, int nz,
                           int C, const float* mesh, float* out, void* stream) {
  GeneralGrid G;
  PMB_TRY(general_grid(gx, gy, gz, cell, ox, oy, oz, cell2, nx, ny, nz, &G));
  PMB_REQUIRE(n >= 0 && C >= 1 && C <= 4, "pmb_cic_general_gather: bad particle count or channels");
  return general_gather(pmid, disp, valid, n, G, C, mesh, out, S(stream));
}

int pmb_cic_general_interp_grad(const int16_t* pmid, const float* disp, const uint8_t* valid, int64_t n, int gx,
                                int gy, int gz, float cell, float ox, float oy, float oz, float cell2, int nx, int ny,
                                int nz, int C, const float* mesh, const float* u, float u_const, float* disp_cot,
                                float* wsum, void* stream) {
  GeneralGrid G;
  PMB_TRY(general_grid(gx, gy, gz, cell, ox, oy, oz, cell2, nx, ny, nz, &G));
  PMB_REQUIRE(n >= 0 && C >= 1 && C <= 4, "pmb_cic_general_interp_grad: bad particle count or channels");
  return general_interp_grad(pmid, disp, valid, n, G, C, mesh, u, u_const, disp_cot, wsum, S(stream));
}

int pmb_set_gather_staging(int mode) {
  PMB_REQUIRE(mode >= 0 && mode <= 2, "pmb_set_gather_staging: mode must be 0, 1 or 2");
  set_gather_staging(mode);
  return kOk;
}

int pmb_set_wait_limit(int64_t polls) {
  set_wait_polls(polls < 0 ? kWaitPolls : (polls > 0xFFFFFFFFll ? 0xFFFFFFFFu : (uint32_t)polls));
  return kOk;
}

int pmb_sorted_status(const void* sorted, int64_t n, int nx, int ny, int nz, uint32_t* flags, void* stream) {
  PMB_REQUIRE(flags != nullptr && sorted != nullptr, "pmb_sorted_status: null argument");
  PMB_REQUIRE(valid_mesh(nx, ny, nz) && n >= 0, "pmb_sorted_status: bad shape");
  SortedView v = sorted_view(const_cast<void*>(sorted), n, Mesh3{nx, ny, nz});
  PMB_CUDA_CHECK(cudaMemcpyAsync(flags, v.status, 4, cudaMemcpyDeviceToHost, S(stream)));
  PMB_CUDA_CHECK(cudaStreamSynchronize(S(stream)));
  return kOk;
}

int pmb_device_status(uint32_t* flags) {
  PMB_REQUIRE(flags != nullptr, "pmb_device_status: null output");
  PMB_CUDA_CHECK(cudaDeviceSynchronize());
  unsigned int f = 0, fft = 0;
  PMB_TRY(device_flags_take(&f));
  PMB_TRY(pmfft_timeouts(&fft));
  PMB_TRY(pmfft_timeouts_clear());
  if (fft) f |= kFlagWaitTimeout;
  *flags = f;
  if (f == 0) return kOk;
  std::string msg = "pmb_device_status:";
  if (f & kFlagWaitTimeout) msg += " a bounded wait on bulk/TMA copies gave up (results of that launch are invalid);";
  if (f & kFlagNonFiniteDisp) msg += " a non-finite displacement reached the cell sort (its outputs were not written);";
  if (f & kFlagNonFiniteValue) msg += " a non-finite value reached a deposit (its output was not written);";
  set_last_error(msg.c_str());
  return kDeviceFlagged;
}

int pmb_wait_timeouts(uint32_t* count) {
  PMB_REQUIRE(count != nullptr, "pmb_wait_timeouts: null output");
  return wait_timeouts(count);
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

int pmb_interlace_spectra(void* spec0, void* spec1, int nx, int ny, int nz, int mode, void* stream) {
  Mesh3 m{nx, ny, nz};
  PMB_REQUIRE(nx > 0 && ny > 0 && nz > 0, "pmb_interlace_spectra: bad shape");
  PMB_REQUIRE(mode == 0 || mode == 1, "pmb_interlace_spectra: mode must be 0 (combine) or 1 (transpose)");
  PMB_REQUIRE(spec0 != nullptr && spec1 != nullptr && spec0 != spec1, "pmb_interlace_spectra: two distinct spectra");
  return interlace((float2*)spec0, (float2*)spec1, m, mode, S(stream));
}

int pmb_green_potential(const void* src_hat, void* pot_hat, int nx, int ny, int nz, const float* tables, int has_masks,
                        int green_kernel, const float* transfer, const float* radial, int radial_len, float post_scale,
                        void* stream) {
  Mesh3 m{nx, ny, nz};
  PMB_REQUIRE(nx > 0 && ny > 0 && nz > 0, "pmb_green_potential: bad shape");
  PMB_REQUIRE(green_kernel == 0 || green_kernel == 1, "pmb_green_potential: unknown Green's function");
  return green_potential((const float2*)src_hat, (float2*)pot_hat, m, make_tables(tables, m, has_masks),
                         make_green(green_kernel, transfer, radial, radial_len, post_scale), S(stream));
}

int pmb_gradient_spectra(const void* pot_hat, const void* res_hat, float res_scale, void* grad_hat, int nx, int ny,
                         int nz, const float* tables, float post_scale, void* stream) {
  Mesh3 m{nx, ny, nz};
  PMB_REQUIRE(nx > 0 && ny > 0 && nz > 0 && pot_hat && grad_hat, "pmb_gradient_spectra: bad arguments");
  return gradient_spectra((const float2*)pot_hat, (const float2*)res_hat, res_scale, (float2*)grad_hat, m,
                          make_tables(tables, m, 0), post_scale, S(stream));
}

int pmb_gradient_adjoint_plain(const void* grad_cot_hat, void* out_hat, int nx, int ny, int nz, const float* tables,
                               float post_scale, void* stream) {
  Mesh3 m{nx, ny, nz};
  PMB_REQUIRE(nx > 0 && ny > 0 && nz > 0 && grad_cot_hat && out_hat, "pmb_gradient_adjoint_plain: bad arguments");
  return gradient_adjoint_plain((const float2*)grad_cot_hat, (float2*)out_hat, m, make_tables(tables, m, 0),
                                post_scale, S(stream));
}

int pmb_project_density(const float* mesh, int nx, int ny, int nz, int axis, int start, int stop, int max_width,
                        float* out, void* stream) {
  PMB_REQUIRE(nx > 0 && ny > 0 && nz > 0, "pmb_project_density: bad shape");
  PMB_REQUIRE(axis >= 0 && axis <= 2, "pmb_project_density: axis must be 0, 1 or 2");
  PMB_REQUIRE(mesh != nullptr && out != nullptr, "pmb_project_density: null buffer");
  return project_window(mesh, Mesh3{nx, ny, nz}, axis, start, stop, max_width, out, S(stream));
}

// ---------------------------------------------------------------------------
// Fused force
// ---------------------------------------------------------------------------
// Spectral path of the fused force: the hand-written pass chain over the
// y-blocked layout (pmfft.cu) for power-of-two meshes, cuFFT otherwise.
static bool g_use_pmfft = true;

static bool use_pmfft(Mesh3 m) { return g_use_pmfft && pmfft_supported(m); }

}  // extern "C"

namespace pmb {
bool pmfft_enabled() { return g_use_pmfft; }
}  // namespace pmb

extern "C" {

int pmb_set_pmfft(int enabled) {
  g_use_pmfft = enabled != 0;
  return kOk;
}

int pmb_pmfft_supported(int nx, int ny, int nz) { return pmfft_supported(Mesh3{nx, ny, nz}) ? 1 : 0; }

int64_t pmb_pmfft_channel_elems(int nx, int ny, int nz) {
  Mesh3 m{nx, ny, nz};
  return pmfft_supported(m) ? pmfft_channel_elems(m) : -1;
}

int pmb_pmfft_z(int nx, int ny, int nz, int inverse, int batch, const void* in, void* out, void* stream) {
  Mesh3 m{nx, ny, nz};
  PMB_REQUIRE(pmfft_supported(m), "pmb_pmfft_z: mesh not supported (powers of two, 64..1024, nz >= 128)");
  PMB_REQUIRE(batch >= 1, "pmb_pmfft_z: batch must be positive");
  if (inverse) return pmfft_z(m, 1, batch, nullptr, (const float2*)in, (float*)out, nullptr, S(stream));
  return pmfft_z(m, 0, batch, (const float*)in, nullptr, nullptr, (float2*)out, S(stream));
}

int pmb_pmfft_col(int nx, int ny, int nz, int mode, int nbatch, int ch_off, const void* in, void* out,
                  const float* tables, int has_masks, const float* transfer, const float* radial, int radial_len,
                  float post_scale, void* stream) {
  Mesh3 m{nx, ny, nz};
  PMB_REQUIRE(pmfft_supported(m), "pmb_pmfft_col: mesh not supported (powers of two, 64..1024, nz >= 128)");
  PMB_REQUIRE(mode >= 0 && mode <= 8, "pmb_pmfft_col: mode must be 0..8");
  PMB_REQUIRE(nbatch >= 1 && ch_off >= 0, "pmb_pmfft_col: bad batch");
  PMB_REQUIRE(tables != nullptr || mode == 0 || mode == 1 || mode == 4 || mode == 5,
              "pmb_pmfft_col: spectral tables required for the multiplier modes");
  SpecTables t{};
  if (tables != nullptr) t = make_tables(tables, m, has_masks);
  return pmfft_col(m, mode, nbatch, ch_off, (const float2*)in, (float2*)out, t,
                   make_green(0, transfer, radial, radial_len, post_scale), S(stream));
}

int pmb_pmfft_z2(int nx, int ny, int nz, int inverse, int batch, const void* in, void* out, const float* tables,
                 int has_masks, int prune, void* stream) {
  Mesh3 m{nx, ny, nz};
  PMB_REQUIRE(pmfft_supported(m), "pmb_pmfft_z2: mesh not supported (powers of two, 64..1024, nz >= 128)");
  PMB_REQUIRE(batch >= 1, "pmb_pmfft_z2: batch must be positive");
  PMB_REQUIRE(!prune || (tables != nullptr && has_masks), "pmb_pmfft_z2: pruning needs tables with masks");
  SpecTables t{};
  if (prune) t = make_tables(tables, m, 1);
  if (inverse) return pmfft_z_pruned(m, 1, batch, nullptr, (const float2*)in, (float*)out, nullptr, t, S(stream));
  return pmfft_z_pruned(m, 0, batch, (const float*)in, nullptr, nullptr, (float2*)out, t, S(stream));
}

int pmb_pmfft_col2(int nx, int ny, int nz, int mode, int nbatch, int ch_off, const void* in, void* out,
                   const float* tables, int has_masks, const float* transfer, const float* radial, int radial_len,
                   float post_scale, int prune, void* stream) {
  Mesh3 m{nx, ny, nz};
  PMB_REQUIRE(pmfft_supported(m), "pmb_pmfft_col2: mesh not supported (powers of two, 64..1024, nz >= 128)");
  PMB_REQUIRE(mode >= 0 && mode <= 8, "pmb_pmfft_col2: mode must be 0..8");
  PMB_REQUIRE(nbatch >= 1 && ch_off >= 0, "pmb_pmfft_col2: bad batch");
  PMB_REQUIRE(tables != nullptr || mode == 0 || mode == 1 || mode == 4 || mode == 5,
              "pmb_pmfft_col2: spectral tables required for the multiplier modes");
  PMB_REQUIRE(!prune || (tables != nullptr && has_masks), "pmb_pmfft_col2: pruning needs tables with masks");
  PMB_REQUIRE(!prune || (mode != 4 && mode != 5 && mode != 8), "pmb_pmfft_col2: modes 4, 5, 8 have no pruned form");
  SpecTables t{};
  if (tables != nullptr) t = make_tables(tables, m, has_masks);
  return pmfft_col_pruned(m, mode, nbatch, ch_off, (const float2*)in, (float2*)out, t,
                          make_green(0, transfer, radial, radial_len, post_scale), prune != 0, S(stream));
}

int pmb_pmfft_set_col_ctas(int ctas) { return pmfft_set_col_ctas(ctas); }

int pmb_pmfft_timeouts(uint32_t* count) {
  PMB_REQUIRE(count != nullptr, "pmb_pmfft_timeouts: null output");
  return pmfft_timeouts(count);
}

static int64_t force_layout(int64_t n, Mesh3 m, void* ws, int64_t cap, void** sorted, void** bin_scratch,
                            void** scale16, float** src, float2** src_hat, float2** grad_hat, void** fft_work) {
  Carve c(ws, cap);
  *sorted = c.take(sorted_bytes(n, m));
  *bin_scratch = c.take(bin_scratch_bytes(n, m));
  *scale16 = c.take(16);
  *src = (float*)c.take(4 * m.cells());
  if (use_pmfft(m)) {
    // five spectral channels for the pass chain
    *src_hat = (float2*)c.take(5 * 8 * pmfft_channel_elems(m));
    *grad_hat = nullptr;
    *fft_work = nullptr;
    return c.off;
  }
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

int pmb_force2(const int16_t* pmid, float* disp, const float* drift_vel, float drift, int64_t n, int nx, int ny, int nz,
               float cell, float val_const, float src_mul, const float* tables, int has_masks, int green_kernel,
               const float* transfer, const float* radial, int radial_len, float* force_meshes, float* acc,
               float* vel_kick, float kick, float kick2, void* workspace, int64_t workspace_bytes, void* stream) {
  Mesh3 m{nx, ny, nz};
  PMB_REQUIRE(valid_mesh(nx, ny, nz), "pmb_force: unsupported mesh shape");
  PMB_REQUIRE(n >= 0 && n < 4294967295ll, "pmb_force: particle count out of range");
  PMB_REQUIRE(cell > 0.f, "pmb_force: cell size must be positive");
  PMB_REQUIRE(acc != nullptr || vel_kick != nullptr, "pmb_force: acc may be null only with vel_kick");
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
  PMB_TRY(pmb_scatter_rows(sorted, n, nx, ny, nz, 1, nullptr, 0, val_const, 1, src_mul, src, scale16, stream));
  const float inv_m = (float)(1.0 / (double)m.cells());
  if (use_pmfft(m)) {
    PMB_TRY(pmfft_force(m, src, force_meshes, src_hat, make_tables(tables, m, has_masks),
                        make_green(green_kernel, transfer, radial, radial_len, inv_m), s));
  } else {
    PMB_TRY(fft_r2c(m, 1, src, src_hat, work, s));
    PMB_TRY(green_gradient(src_hat, grad_hat, m, make_tables(tables, m, has_masks),
                           make_green(green_kernel, transfer, radial, radial_len, inv_m), s));
    PMB_TRY(fft_c2r(m, 3, grad_hat, force_meshes, work, s));
  }
  SortedView v = sorted_view(sorted, n, m);
  return gather_sorted(v.rec, v.perm, v.offs, n, m, 3, force_meshes, acc, vel_kick, kick, kick2, s, v.status);
}

int pmb_force(const int16_t* pmid, float* disp, const float* drift_vel, float drift, int64_t n, int nx, int ny, int nz,
              float cell, float val_const, float src_mul, const float* tables, int has_masks, int green_kernel,
              const float* transfer, const float* radial, int radial_len, float* force_meshes, float* acc,
              float* vel_kick, float kick, void* workspace, int64_t workspace_bytes, void* stream) {
  return pmb_force2(pmid, disp, drift_vel, drift, n, nx, ny, nz, cell, val_const, src_mul, tables, has_masks,
                    green_kernel, transfer, radial, radial_len, force_meshes, acc, vel_kick, kick, 0.f, workspace,
                    workspace_bytes, stream);
}

// ---------------------------------------------------------------------------
// Low-memory forward force
// ---------------------------------------------------------------------------
static int64_t force_streamed_layout(int64_t n, Mesh3 m, void* ws, int64_t cap, void** sorted, void** bins,
                                     void** scale16, float** real, float2** src_hat, float2** comp_hat,
                                     float** planar, void** work) {
  Carve c(ws, cap);
  *sorted = c.take(sorted_bytes(n, m));
  *bins = c.take(bin_scratch_bytes(n, m));
  *scale16 = c.take(16);
  *real = (float*)c.take(4 * m.cells());
  *src_hat = (float2*)c.take(8 * m.half_cells());
  *comp_hat = (float2*)c.take(8 * m.half_cells());
  *planar = (float*)c.take(12 * n);
  const int64_t w = fft_work_bytes(m, 1);
  if (w < 0) return -1;
  *work = c.take(w);
  return c.off;
}

int64_t pmb_force_streamed_workspace_bytes(int64_t n, int nx, int ny, int nz) {
  void *a, *b, *c, *w;
  float *r, *p;
  float2 *sh, *ch;
  return force_streamed_layout(n, Mesh3{nx, ny, nz}, nullptr, 0, &a, &b, &c, &r, &sh, &ch, &p, &w);
}

int pmb_force_streamed(const int16_t* pmid, float* disp, const float* drift_vel, float drift, int64_t n, int nx,
                       int ny, int nz, float cell, float val_const, float src_mul, const float* tables, int has_masks,
                       int green_kernel, const float* transfer, const float* radial, int radial_len, float* acc,
                       void* workspace, int64_t workspace_bytes, void* stream) {
  Mesh3 m{nx, ny, nz};
  PMB_REQUIRE(valid_mesh(nx, ny, nz), "pmb_force_streamed: unsupported mesh shape");
  PMB_REQUIRE(n >= 0 && n < 4294967295ll, "pmb_force_streamed: particle count out of range");
  PMB_REQUIRE(cell > 0.f, "pmb_force_streamed: cell size must be positive");
  void *sorted, *bins, *scale16, *work;
  float *real, *planar;
  float2 *src_hat, *comp_hat;
  const int64_t need = force_streamed_layout(n, m, workspace, workspace_bytes, &sorted, &bins, &scale16, &real,
                                             &src_hat, &comp_hat, &planar, &work);
  PMB_REQUIRE(need >= 0, "pmb_force_streamed: cuFFT plan creation failed");
  if (need > workspace_bytes) {
    set_last_error("pmb_force_streamed: workspace too small");
    return kScratchTooSmall;
  }
  cudaStream_t s = S(stream);
  PMB_TRY(pmb_sort_rows(pmid, disp, drift_vel, drift, n, nx, ny, nz, cell, sorted, bins, bin_scratch_bytes(n, m),
                        stream));
  PMB_TRY(pmb_scatter_rows(sorted, n, nx, ny, nz, 1, nullptr, 0, val_const, 1, src_mul, real, scale16, stream));
  PMB_TRY(fft_r2c(m, 1, real, src_hat, work, s));
  SortedView v = sorted_view(sorted, n, m);
  const SpecTables t = make_tables(tables, m, has_masks);
  const GreenParams g = make_green(green_kernel, transfer, radial, radial_len, (float)(1.0 / (double)m.cells()));
  for (int d = 0; d < 3; ++d) {
    PMB_TRY(green_gradient_component(src_hat, comp_hat, m, t, g, d, s));
    PMB_TRY(fft_c2r(m, 1, comp_hat, real, work, s));
    PMB_TRY(gather_sorted(v.rec, v.perm, v.offs, n, m, 1, real, planar + (int64_t)d * n, nullptr, 0.f, 0.f, s,
                          v.status));
  }
  return interleave3(planar, acc, n, s);
}

static int64_t force_vjp_layout(int64_t n, Mesh3 m, void* ws, int64_t cap, void** sorted, void** bins, void** scale16,
                                float** cot_sorted, float** mesh_cot, float2** spec3, float2** src_hat, float** src_cot,
                                void** work) {
  Carve c(ws, cap);
  *sorted = c.take(sorted_bytes(n, m));
  *bins = c.take(bin_scratch_bytes(n, m));
  *scale16 = c.take(16);
  *cot_sorted = (float*)c.take(12 * n);
  *mesh_cot = (float*)c.take(12 * m.cells());
  if (use_pmfft(m)) {
    *spec3 = (float2*)c.take(5 * 8 * pmfft_channel_elems(m));
    *src_hat = nullptr;
    *src_cot = (float*)c.take(4 * m.cells());
    *work = nullptr;
    return c.off;
  }
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
  float *cs, *mc, *sc;
  float2 *s3, *sh;
  return force_vjp_layout(n, Mesh3{nx, ny, nz}, nullptr, 0, &a, &b, &c, &cs, &mc, &s3, &sh, &sc, &w);
}

// presorted (may be null): records of exactly these positions left by an
// earlier pmb_force / pmb_sort_rows; the sort is skipped.
static int force_vjp_impl(const int16_t* pmid, const float* disp, int64_t n, int nx, int ny, int nz, float cell,
                          float val_const, float src_mul, const float* tables, int has_masks, int green_kernel,
                          const float* transfer, const float* radial, int radial_len, const float* force_meshes,
                          const float* acc_cot, float* disp_cot, const void* presorted, void* workspace,
                          int64_t workspace_bytes, void* stream) {
  Mesh3 m{nx, ny, nz};
  PMB_REQUIRE(valid_mesh(nx, ny, nz), "pmb_force_vjp: unsupported mesh shape");
  PMB_REQUIRE(n >= 0 && n < 4294967295ll, "pmb_force_vjp: particle count out of range");
  PMB_REQUIRE(cell > 0.f, "pmb_force_vjp: cell size must be positive");
  void *sorted, *bins, *scale16, *work;
  float *cot_sorted, *mesh_cot, *src_cot;
  float2 *spec3, *src_hat;
  int64_t need = force_vjp_layout(n, m, workspace, workspace_bytes, &sorted, &bins, &scale16, &cot_sorted, &mesh_cot,
                                  &spec3, &src_hat, &src_cot, &work);
  PMB_REQUIRE(need >= 0, "pmb_force_vjp: cuFFT plan creation failed");
  if (need > workspace_bytes) {
    set_last_error("pmb_force_vjp: workspace too small");
    return kScratchTooSmall;
  }
  cudaStream_t s = S(stream);
  if (presorted != nullptr)
    sorted = const_cast<void*>(presorted);
  else
    PMB_TRY(pmb_sort_rows(pmid, (float*)disp, nullptr, 0.f, n, nx, ny, nz, cell, sorted, bins,
                          bin_scratch_bytes(n, m), stream));
  SortedView v = sorted_view(sorted, n, m);
  // gather adjoint: position term and the 3-channel scatter of acc_cot
  PMB_TRY(interp_grad_sorted(v.rec, v.perm, v.offs, n, m, 3, force_meshes, acc_cot, 0.f, cell, 1, disp_cot, nullptr,
                             cot_sorted, s, v.status));
  PMB_TRY(pmb_scatter_rows(sorted, n, nx, ny, nz, 3, cot_sorted, 1, 0.f, 0, 1.f, mesh_cot, scale16, stream));
  // transposes of the C2R, gradient, Green and R2C stages
  const float post = (float)((double)src_mul / (double)m.cells());
  if (use_pmfft(m)) {
    PMB_TRY(pmfft_force_adjoint(m, mesh_cot, src_cot, spec3, make_tables(tables, m, has_masks),
                                make_green(green_kernel, transfer, radial, radial_len, post), s));
  } else {
    PMB_TRY(fft_r2c(m, 3, mesh_cot, spec3, work, s));
    PMB_TRY(green_gradient_adjoint(spec3, src_hat, m, make_tables(tables, m, has_masks),
                                   make_green(green_kernel, transfer, radial, radial_len, post), s));
    PMB_TRY(fft_c2r(m, 1, src_hat, src_cot, work, s));
  }
  // scatter adjoint of the density (constant particle value)
  return interp_grad_sorted(v.rec, v.perm, v.offs, n, m, 1, src_cot, nullptr, val_const, cell, 1, disp_cot, nullptr,
                            nullptr, s, v.status);
}

int pmb_force_vjp(const int16_t* pmid, const float* disp, int64_t n, int nx, int ny, int nz, float cell,
                  float val_const, float src_mul, const float* tables, int has_masks, int green_kernel,
                  const float* transfer, const float* radial, int radial_len, const float* force_meshes,
                  const float* acc_cot, float* disp_cot, void* workspace, int64_t workspace_bytes, void* stream) {
  return force_vjp_impl(pmid, disp, n, nx, ny, nz, cell, val_const, src_mul, tables, has_masks, green_kernel,
                        transfer, radial, radial_len, force_meshes, acc_cot, disp_cot, nullptr, workspace,
                        workspace_bytes, stream);
}

int pmb_force_vjp_presorted(const void* sorted, int64_t n, int nx, int ny, int nz, float cell, float val_const,
                            float src_mul, const float* tables, int has_masks, int green_kernel,
                            const float* transfer, const float* radial, int radial_len, const float* force_meshes,
                            const float* acc_cot, float* disp_cot, void* workspace, int64_t workspace_bytes,
                            void* stream) {
  PMB_REQUIRE(sorted != nullptr, "pmb_force_vjp_presorted: null sorted records");
  return force_vjp_impl(nullptr, nullptr, n, nx, ny, nz, cell, val_const, src_mul, tables, has_masks, green_kernel,
                        transfer, radial, radial_len, force_meshes, acc_cot, disp_cot, sorted, workspace,
                        workspace_bytes, stream);
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

int pmb_kick_adj2(float* vel, const float* acc, const float* vel_cot, float* acc_cot, int64_t n, float kick_a,
                  float kick_b, int two, int zero_cot, double* dot_a, double* dot_b, double* dot_force,
                  void* stream) {
  PMB_REQUIRE(dot_a != nullptr && (two == 0 || dot_b != nullptr), "pmb_kick_adj2: dot accumulators required");
  return kick_adj2(vel, acc, const_cast<float*>(vel_cot), acc_cot, n, kick_a, kick_b, two != 0, zero_cot != 0, dot_a,
                   dot_b, dot_force, nullptr, 0.f, nullptr, S(stream));
}

int pmb_kick_adj3(float* vel, const float* acc, float* vel_cot, float* acc_cot, int64_t n, float kick_a, float kick_b,
                  int two, int zero_cot, double* dot_a, double* dot_b, double* dot_force, const float* disp_cot,
                  float drift, double* dot_drift, void* stream) {
  PMB_REQUIRE(dot_a != nullptr && (two == 0 || dot_b != nullptr), "pmb_kick_adj3: dot accumulators required");
  PMB_REQUIRE(disp_cot == nullptr || dot_drift != nullptr, "pmb_kick_adj3: drift dot accumulator required");
  return kick_adj2(vel, acc, vel_cot, acc_cot, n, kick_a, kick_b, two != 0, zero_cot != 0, dot_a, dot_b, dot_force,
                   disp_cot, drift, dot_drift, S(stream));
}

int pmb_drift_cot_adj(const float* vel, const float* disp_cot, float* vel_cot, int64_t n, float drift, double* dot,
                      void* stream) {
  PMB_REQUIRE(dot != nullptr, "pmb_drift_cot_adj: dot accumulator required");
  return drift_cot_adj(vel, disp_cot, vel_cot, n, drift, dot, S(stream));
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

int pmb_sum(const float* a, int64_t n, double* out, void* stream) {
  PMB_REQUIRE(out != nullptr, "pmb_sum: output required");
  return sum(a, n, out, S(stream));
}

// ---------------------------------------------------------------------------
// Initial conditions
// ---------------------------------------------------------------------------
int pmb_white_noise_nested(uint32_t seed, int gx, int gy, int gz, void* modes_out, uint32_t* hashes_out,
                           void* stream) {
  PMB_REQUIRE(gx > 0 && gy > 0 && gz > 0, "pmb_white_noise_nested: bad grid");
  return white_noise(seed, Mesh3{gx, gy, gz}, (float2*)modes_out, hashes_out, S(stream));
}

int pmb_linear_modes(const void* modes_in, void* modes_out, float* amp_out, int gx, int gy, int gz,
                     const float* ktables, const double* transfer_k, const double* transfer, int ntab, double A_s,
                     double n_s, double omega_m, double k_pivot, double growth2, double box_vol, void* stream) {
  PMB_REQUIRE(gx > 0 && gy > 0 && gz > 0 && ntab >= 2, "pmb_linear_modes: bad arguments");
  const double c_light = 299792458.0 / 1e5;
  LinearPowerParams p;
  p.coef = 0.32 * A_s * k_pivot;
  p.k_pivot = k_pivot;
  p.n_s = n_s;
  p.pi_c2_over_om = M_PI * c_light * c_light / omega_m;
  p.growth2 = growth2;
  p.box_vol = (float)box_vol;
  return linear_modes((const float2*)modes_in, (float2*)modes_out, amp_out, Mesh3{gx, gy, gz}, ktables, transfer_k,
                      transfer, ntab, p, S(stream));
}

static int64_t lpt_layout(Mesh3 g, void* ws, int64_t cap, float2** pot1, float2** spec6, float** real6, float** L,
                          float2** Lhat, void** work) {
  Carve c(ws, cap);
  const int64_t ng = g.cells(), mc = g.half_cells();
  *pot1 = (float2*)c.take(8 * mc);
  *spec6 = (float2*)c.take(48 * mc);
  *real6 = (float*)c.take(24 * ng);
  *L = (float*)c.take(4 * ng);
  *Lhat = (float2*)c.take(8 * mc);
  int64_t w6 = fft_work_bytes(g, 6), w1 = fft_work_bytes(g, 1);
  if (w6 < 0 || w1 < 0) return -1;
  *work = c.take(w6 > w1 ? w6 : w1);
  return c.off;
}

int64_t pmb_lpt_workspace_bytes(int gx, int gy, int gz) {
  float2 *a, *b, *d;
  float *r, *l;
  void* w;
  return lpt_layout(Mesh3{gx, gy, gz}, nullptr, 0, &a, &b, &r, &l, &d, &w);
}

int pmb_lpt(const void* modes, int gx, int gy, int gz, float spacing, float cell_vol, const float* tables, int order,
            float D1, float V1, float D2, float V2, const int16_t* pmid, float* disp, float* vel, int64_t n,
            float cell, float* fields, int64_t* index_out, void* workspace, int64_t workspace_bytes, void* stream) {
  Mesh3 g{gx, gy, gz};
  PMB_REQUIRE(gx > 0 && gy > 0 && gz > 0, "pmb_lpt: bad grid");
  PMB_REQUIRE(order >= 0 && order <= 2, "pmb_lpt: order must be 0, 1 or 2");
  float2 *pot1, *spec6, *Lhat;
  float *real6, *L;
  void* work;
  int64_t need = lpt_layout(g, workspace, workspace_bytes, &pot1, &spec6, &real6, &L, &Lhat, &work);
  PMB_REQUIRE(need >= 0, "pmb_lpt: cuFFT plan creation failed");
  if (need > workspace_bytes) {
    set_last_error("pmb_lpt: workspace too small");
    return kScratchTooSmall;
  }
  cudaStream_t s = S(stream);
  const float inv_n = (float)(1.0 / (double)g.cells());
  PMB_TRY(lpt_strains((const float2*)modes, 1.0f / cell_vol, pot1, spec6, g, tables, inv_n, s));
  const float2* Lh = nullptr;
  if (order >= 2) {
    PMB_TRY(fft_c2r(g, 6, spec6, real6, work, s));
    PMB_TRY(lpt_source(real6, L, g.cells(), s));
    PMB_TRY(fft_r2c(g, 1, L, Lhat, work, s));
    Lh = Lhat;
  }
  PMB_TRY(lpt_gradients(pot1, Lh, spec6, g, tables, inv_n, s));
  PMB_TRY(fft_c2r(g, 6, spec6, fields, work, s));
  return lpt_displace(pmid, disp, vel, n, g, cell, spacing, fields, order, D1, V1, D2, V2, index_out, s);
}

static int64_t lpt_vjp_layout(Mesh3 g, void* ws, int64_t cap, float** cot6, float2** F6, float2** Lhat, float** L,
                              float2** pot1, float2** spec6, float** real6, void** work) {
  Carve c(ws, cap);
  const int64_t ng = g.cells(), mc = g.half_cells();
  *cot6 = (float*)c.take(24 * ng);
  *F6 = (float2*)c.take(48 * mc);
  *Lhat = (float2*)c.take(8 * mc);
  *L = (float*)c.take(4 * ng);
  *pot1 = (float2*)c.take(8 * mc);
  *spec6 = (float2*)c.take(48 * mc);
  *real6 = (float*)c.take(24 * ng);
  int64_t w6 = fft_work_bytes(g, 6), w1 = fft_work_bytes(g, 1);
  if (w6 < 0 || w1 < 0) return -1;
  *work = c.take(w6 > w1 ? w6 : w1);
  return c.off;
}

int64_t pmb_lpt_vjp_workspace_bytes(int gx, int gy, int gz) {
  float *a, *l, *r;
  float2 *f, *lh, *p, *sp;
  void* w;
  return lpt_vjp_layout(Mesh3{gx, gy, gz}, nullptr, 0, &a, &f, &lh, &l, &p, &sp, &r, &w);
}

int pmb_lpt_vjp(const void* modes, int gx, int gy, int gz, float cell_vol, const float* tables, int order, float D1,
                float V1, float D2, float V2, const int64_t* index, const float* fields, const float* disp_cot,
                const float* vel_cot, int64_t n, const float* amp, void* modes_cot, double* dots, void* workspace,
                int64_t workspace_bytes, void* stream) {
  Mesh3 g{gx, gy, gz};
  PMB_REQUIRE(gx > 0 && gy > 0 && gz > 0, "pmb_lpt_vjp: bad grid");
  PMB_REQUIRE(order >= 1 && order <= 2, "pmb_lpt_vjp: order must be 1 or 2");
  PMB_REQUIRE(dots != nullptr, "pmb_lpt_vjp: dots required");
  float *cot6, *L, *real6;
  float2 *F6, *Lhat, *pot1, *spec6;
  void* work;
  int64_t need = lpt_vjp_layout(g, workspace, workspace_bytes, &cot6, &F6, &Lhat, &L, &pot1, &spec6, &real6, &work);
  PMB_REQUIRE(need >= 0, "pmb_lpt_vjp: cuFFT plan creation failed");
  if (need > workspace_bytes) {
    set_last_error("pmb_lpt_vjp: workspace too small");
    return kScratchTooSmall;
  }
  cudaStream_t s = S(stream);
  const int64_t ng = g.cells();
  const float inv_n = (float)(1.0 / (double)ng);
  PMB_CUDA_CHECK(cudaMemsetAsync(cot6, 0, 24 * ng, s));
  PMB_TRY(lpt_field_cot(index, disp_cot, vel_cot, n, ng, fields, order, D1, V1, D2, V2, cot6, dots, s));
  PMB_TRY(fft_r2c(g, 6, cot6, F6, work, s));
  const float2* FS = nullptr;
  if (order >= 2) {
    PMB_TRY(lpt_grad2_adjoint(F6 + 3 * g.half_cells(), Lhat, g, tables, inv_n, s));
    PMB_TRY(fft_c2r(g, 1, Lhat, L, work, s));
    PMB_TRY(lpt_strains((const float2*)modes, 1.0f / cell_vol, pot1, spec6, g, tables, inv_n, s));
    PMB_TRY(fft_c2r(g, 6, spec6, real6, work, s));
    PMB_TRY(lpt_source_adjoint(real6, L, cot6, ng, s));
    PMB_TRY(fft_r2c(g, 6, cot6, spec6, work, s));
    FS = spec6;
  }
  const float scale = (float)(1.0 / ((double)cell_vol * (double)ng));
  return lpt_modes_adjoint(F6, FS, amp, (float2*)modes_cot, g, tables, scale, s);
}

// ---------------------------------------------------------------------------
// Power spectrum
// ---------------------------------------------------------------------------
int pmb_pk_shells(const void* spec, int nx, int ny, int nz, const float* sinc_tab, int mas_power, int num_shells,
                  double* sums, const void* spec_b, double* sums_b, double* sums_x, void* stream) {
  PMB_REQUIRE(nx > 0 && ny > 0 && nz > 0 && num_shells > 0, "pmb_pk_shells: bad arguments");
  PMB_REQUIRE(spec_b == nullptr || (sums_b != nullptr && sums_x != nullptr), "pmb_pk_shells: cross sums missing");
  cudaStream_t s = S(stream);
  PMB_CUDA_CHECK(cudaMemsetAsync(sums, 0, sizeof(double) * num_shells, s));
  if (spec_b != nullptr) {
    PMB_CUDA_CHECK(cudaMemsetAsync(sums_b, 0, sizeof(double) * num_shells, s));
    PMB_CUDA_CHECK(cudaMemsetAsync(sums_x, 0, sizeof(double) * num_shells, s));
  }
  return pk_shells((const float2*)spec, Mesh3{nx, ny, nz}, sinc_tab, mas_power, num_shells, sums,
                   (const float2*)spec_b, sums_b, sums_x, s);
}

int pmb_shell_stats(int nx, int ny, int nz, int num_shells, double* counts, double* ksum, void* stream) {
  PMB_REQUIRE(nx > 0 && ny > 0 && nz > 0 && num_shells > 0, "pmb_shell_stats: bad arguments");
  cudaStream_t s = S(stream);
  PMB_CUDA_CHECK(cudaMemsetAsync(counts, 0, sizeof(double) * num_shells, s));
  PMB_CUDA_CHECK(cudaMemsetAsync(ksum, 0, sizeof(double) * num_shells, s));
  return shell_stats(Mesh3{nx, ny, nz}, num_shells, counts, ksum, s);
}

int pmb_pk_shells_adjoint(const void* spec, int nx, int ny, int nz, const float* sinc_tab, int mas_power,
                          int num_shells, const double* wshell, float post, void* out, void* stream) {
  PMB_REQUIRE(nx > 0 && ny > 0 && nz > 0 && num_shells > 0, "pmb_pk_shells_adjoint: bad arguments");
  return pk_shells_adjoint((const float2*)spec, Mesh3{nx, ny, nz}, sinc_tab, mas_power, num_shells, wshell, post,
                           (float2*)out, S(stream));
}

int pmb_overdensity(const float* rho, float* delta, int64_t n, const double* total, void* stream) {
  return overdensity(rho, delta, n, total, S(stream));
}

// ---------------------------------------------------------------------------
// Learned Green's-function correction
// ---------------------------------------------------------------------------
int pmb_mlp_param_counts(int* n_weights, int* n_biases) {
  if (n_weights) *n_weights = kMlpWeights;
  if (n_biases) *n_biases = kMlpBiases;
  return kOk;
}

int pmb_mlp_table(const void* weights_bf16, const float* biases, float kscale, float a, float omega_m, float sigma8,
                  int len, float* table, void* stream) {
  PMB_REQUIRE(weights_bf16 != nullptr && biases != nullptr && table != nullptr && len > 0,
              "pmb_mlp_table: bad arguments");
  return mlp_table(weights_bf16, biases, MlpCond{kscale, a, omega_m, sigma8}, len, table, S(stream));
}

int pmb_mlp_backward(const void* weights_bf16, const float* biases, float kscale, float a, float omega_m,
                     float sigma8, int len, const double* table_cot, float* grad, void* stream) {
  PMB_REQUIRE(weights_bf16 != nullptr && biases != nullptr && table_cot != nullptr && grad != nullptr && len > 0,
              "pmb_mlp_backward: bad arguments");
  return mlp_backward(weights_bf16, biases, MlpCond{kscale, a, omega_m, sigma8}, len, table_cot, grad, S(stream));
}

int pmb_transfer_cot(const void* grad_cot_hat, const void* src_hat, int nx, int ny, int nz, const float* tables,
                     int has_masks, int len, double* out, void* stream) {
  Mesh3 m{nx, ny, nz};
  PMB_REQUIRE(nx > 0 && ny > 0 && nz > 0 && len > 0, "pmb_transfer_cot: bad arguments");
  return transfer_cot((const float2*)grad_cot_hat, (const float2*)src_hat, m, make_tables(tables, m, has_masks), len,
                      out, S(stream));
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
