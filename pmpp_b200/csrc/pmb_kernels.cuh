// Internal (C++) interfaces between the kernel files and the C-ABI layer.
#pragma once

#include <cufft.h>

#include "pmb_common.cuh"

namespace pmb {

// cic.cu
int64_t scan_tmp_elems(int64_t len);
int exclusive_scan_u32(const uint32_t* in, uint32_t* out, int64_t len, uint32_t* tile_sums, cudaStream_t s);
int64_t bin_scratch_bytes(int64_t n, Mesh3 m);
// Cell sort; shift (may be null: none) offsets the mesh origin, valid (may
// be null: all valid) leaves masked particles out of every row.
struct BinShift;
// status (may be null): the sorted buffer's status word, reset here and
// raised (DeviceFlag bits) by the sort; consumers given a raised word write
// nothing.
int bin_particles(const int16_t* pmid, float* disp, const float* vel, float drift, int64_t n, Mesh3 m, float cell,
                  Rec* rec, uint32_t* perm, uint32_t* offs, void* scratch, cudaStream_t s,
                  const BinShift* shift = nullptr, const uint8_t* valid = nullptr, uint32_t* status = nullptr);
double fixed_point_pow2(int64_t n);
int compute_scale(const float* val, int64_t count, int64_t n, double* scale_dev, unsigned int* tmp, cudaStream_t s);
// n: particles the sort placed (bounds the fixed-point sums)
int scatter_sorted(const Rec* rec, const uint32_t* perm, const uint32_t* offs, Mesh3 m, int C, const float* val,
                   int val_sorted, float val_const, const double* scale_dev, int mode, float src_mul, float* out,
                   cudaStream_t s, int64_t n, uint32_t* status);

// cic_general.cu: CIC onto a mesh of another cell size (no sort)
struct GeneralGrid {
  int gx, gy, gz;        // the particles' periodic mesh (cells of size a1)
  float a1, a2;          // particle-grid and target-mesh cell sizes
  float ox, oy, oz;      // target-mesh origin in the particles' frame
  Mesh3 t;               // target mesh shape
};
int64_t general_scatter_scratch_bytes(Mesh3 t, int C);
int general_scatter(const int16_t* pmid, const float* disp, const uint8_t* valid, int64_t n, GeneralGrid G, int C,
                    const float* val, float val_const, float* out, void* scratch, cudaStream_t s);
int general_gather(const int16_t* pmid, const float* disp, const uint8_t* valid, int64_t n, GeneralGrid G, int C,
                   const float* mesh, float* out, cudaStream_t s);
int general_interp_grad(const int16_t* pmid, const float* disp, const uint8_t* valid, int64_t n, GeneralGrid G,
                        int C, const float* mesh, const float* u, float u_const, float* disp_cot, float* wsum,
                        cudaStream_t s);
// offs (row offsets, may be null) enables the staged kernels.
int gather_sorted(const Rec* rec, const uint32_t* perm, const uint32_t* offs, int64_t n, Mesh3 m, int C,
                  const float* mesh, float* out, float* vel, float kick, float kick2, cudaStream_t s,
                  const uint32_t* status);
int interp_grad_sorted(const Rec* rec, const uint32_t* perm, const uint32_t* offs, int64_t n, Mesh3 m, int C,
                       const float* mesh, const float* u, float u_const, float cell, int accumulate, float* disp_cot,
                       float* wsum, float* u_sorted, cudaStream_t s, const uint32_t* status);
int wait_timeouts(unsigned int* count);
// device-wide DeviceFlag bits (the staged gathers' timeouts included), cleared
int device_flags_take(unsigned int* flags);
void set_gather_staging(int mode);
// poll limit of the first bounded wait of the staged / TMA-fed kernels
void set_wait_polls(uint32_t polls);
uint32_t wait_polls();

// spectral.cu
int fft_r2c(Mesh3 m, int batch, float* in, float2* out, void* work, cudaStream_t s);
int fft_c2r(Mesh3 m, int batch, float2* in, float* out, void* work, cudaStream_t s);
int64_t fft_work_bytes(Mesh3 m, int batch);
int64_t fft_work_bytes64(Mesh3 m, int batch);
int fft_d2z(Mesh3 m, int batch, double* in, double2* out, void* work, cudaStream_t s);
int fft_z2d(Mesh3 m, int batch, double2* in, double* out, void* work, cudaStream_t s);
// Gravity spectral multipliers (see spectral.cu for the exact semantics).
struct GreenParams {
  int green_kernel;     // 0 continuum -1/k^2, 1 discrete Laplacian
  float cell;           // mesh cell size (discrete Laplacian)
  const float* transfer;  // optional real transfer per half-spectrum cell, may be null
  const float* radial;    // optional radial table indexed by integer n^2, may be null
  int radial_len;
  float post_scale;       // applied last (1/M folds the inverse-FFT normalisation in)
};
int green_gradient(const float2* src_hat, float2* grad_hat, Mesh3 m, SpecTables t, GreenParams g, cudaStream_t s);
int green_gradient_adjoint(const float2* grad_cot_hat, float2* src_cot_hat, Mesh3 m, SpecTables t, GreenParams g,
                           cudaStream_t s);
int scale_real(float* x, int64_t count, float a, float b, cudaStream_t s);
// component d of the forward multiplier (streamed force)
int green_gradient_component(const float2* src_hat, float2* out, Mesh3 m, SpecTables t, GreenParams g, int d,
                             cudaStream_t s);
// interlaced-assignment phase: mode 0 s0 = (s0 + P s1) / 2, mode 1 its transpose
int interlace(float2* s0, float2* s1, Mesh3 m, int mode, cudaStream_t s);
// residual-potential force stages (mesh-CNN correction)
int green_potential(const float2* src, float2* out, Mesh3 m, SpecTables t, GreenParams g, cudaStream_t s);
int gradient_spectra(const float2* P, const float2* Q, float q_scale, float2* grad, Mesh3 m, SpecTables t, float post,
                     cudaStream_t s);
int gradient_adjoint_plain(const float2* A, float2* out, Mesh3 m, SpecTables t, float post, cudaStream_t s);

// observe.cu: windowed periodic projection of a mesh along one axis
int project_window(const float* mesh, Mesh3 m, int axis, int start, int stop, int max_width, float* out,
                   cudaStream_t s);
// acc (n,3) from three planar (3,n) channels
int interleave3(const float* planar, float* acc, int64_t n, cudaStream_t s);

// pmfft.cu: hand-written FFT passes for power-of-two meshes over the
// y-blocked half-spectrum layout (see pmfft.cu for the layout and modes).
bool pmfft_supported(Mesh3 m);
int pmfft_row_len(Mesh3 m);
int64_t pmfft_channel_elems(Mesh3 m);
int pmfft_z(Mesh3 m, int inverse, int batch, const float* in_r, const float2* in_c, float* out_r, float2* out_c,
            cudaStream_t s);
int pmfft_col(Mesh3 m, int mode, int nbatch, int ch_off, const float2* in, float2* out, SpecTables t, GreenParams g,
              cudaStream_t s);
int pmfft_col_batched(Mesh3 m, int mode, int nbatch, int ch_off, const float2* in, float2* out, SpecTables t,
                      GreenParams g, const float* tab_base, int64_t tab_stride, int has_masks, int oofs, int ostride,
                      int cstride, cudaStream_t s);
// one pass of a pruned force chain (prune_tables with masks; t.mx null: unpruned)
int pmfft_z_pruned(Mesh3 m, int inverse, int batch, const float* in_r, const float2* in_c, float* out_r, float2* out_c,
                   SpecTables prune_tables, cudaStream_t s);
int pmfft_col_pruned(Mesh3 m, int mode, int nbatch, int ch_off, const float2* in, float2* out, SpecTables t,
                     GreenParams g, bool prune, cudaStream_t s);
int pmfft_force_batched(Mesh3 m, int count, const float* src, float* force_meshes, float2* work,
                        const float* tab_base, int64_t tab_stride, int has_masks, GreenParams g, cudaStream_t s);
int pmfft_force(Mesh3 m, const float* src, float* force_meshes, float2* work, SpecTables t, GreenParams g,
                cudaStream_t s);
int pmfft_force_adjoint(Mesh3 m, const float* mesh_cot, float* src_cot, float2* work, SpecTables t, GreenParams g,
                        cudaStream_t s);
int pmfft_timeouts(unsigned int* count);
int pmfft_timeouts_clear();
int pmfft_set_col_ctas(int ctas);
// process-wide switch of pmb_set_pmfft (capi.cu)
bool pmfft_enabled();

}  // namespace pmb
