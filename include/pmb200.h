/*
 * pmb200.h -- C ABI of the PM++ B200 particle-mesh kernels (libpmb200.so).
 *
 * Every entry point only enqueues work on the CUDA stream it is given; it
 * never synchronises, never creates streams and never allocates device
 * memory: buffers and scratch come from the caller (the same ownership rules
 * as the reference's XLA FFI handlers, cuda/route_kernels.cu:1-7).  All
 * pointers are device pointers unless stated otherwise.  Return value: 0 on
 * success, a negative pmb status otherwise (-1 invalid argument, -2 CUDA
 * error, -3 cuFFT error, -4 unsupported shape, -5 scratch too small, -6 the
 * device flagged bad input or a timed-out wait, see pmb_device_status); the
 * message of the last failure on the calling thread is pmb_last_error().
 * Exceptions to "never allocates, never synchronises": the first call of a
 * cuFFT-route entry point for a new mesh shape creates its plan (cuFFT may
 * allocate and synchronise then; later calls reuse it, with the caller's work
 * area bound), and the status queries pmb_sorted_status / pmb_device_status /
 * pmb_*_timeouts are synchronous by design.
 *
 * Layouts (C order): pmid int16 (n,3); disp/vel/acc float (n,3); meshes float
 * (C,nx,ny,nz) planar channels; spectra float2 (C,nx,ny,nz/2+1).
 *
 * Each entry point names the reference interface it replaces (paths relative
 * to the PM++ source tree).
 */
#ifndef PMB200_H
#define PMB200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Version of this ABI; bumped on any signature change. */
int pmb_abi_version(void);
/* Message of the last failed call on this thread (never NULL). */
const char* pmb_last_error(void);

/* ---------------- particle sort by cell ----------------------------------
 * Replaces the key computation of core/utils.py:292-326 and the per-cell
 * ordering that cuda/route_kernels.cu:131-145, 615-724 maintain, using the
 * binning of cic/enmesh.py:139-147.  Particles are counting-sorted by the
 * mesh row (x, y) of their lower CIC corner; `sorted` receives 16-byte
 * records (fx, fy, fz, raveled cell key), the permutation (uint32), the
 * row offsets (uint32, nx*ny+1) and a status word.  With vel != NULL the
 * drift disp += vel * drift (nbody/integrator.py:223-225) is applied first and
 * written back to disp.  A displacement that is NaN or infinite (after the
 * drift) is binned at its anchor cell and raises flag 2 in the status word
 * (the reference's fail-closed checks, core/utils.py:206-231); every later
 * scatter, gather or adjoint given a flagged buffer writes nothing. */
int64_t pmb_sorted_bytes(int64_t n, int nx, int ny, int nz);
int64_t pmb_sort_scratch_bytes(int64_t n, int nx, int ny, int nz);
int pmb_sort_rows(const int16_t* pmid, float* disp, const float* vel, float drift, int64_t n, int nx, int ny, int nz,
                  float cell, void* sorted, void* scratch, int64_t scratch_bytes, void* stream);
/* pmb_sort_rows for the reference's scatter / gather options (cic/scatter.py:
 * 235-312, cic/gather.py:414-472; cic/pallas.py:133-141, 225-238): the mesh
 * origin sits at (ox, oy, oz) in the particles' frame -- split on the host
 * into whole cells q = floor(o / cell) and the remainder o - q * cell (rounded
 * once to float), the binning is (disp - remainder) / cell from the anchor
 * pmid - q -- and particles with valid[p] == 0 (uint8, device; NULL = all
 * valid) are left out of every row: they deposit nothing, gather 0, leave vel
 * unkicked and take zero adjoint terms (or keep disp_cot when accumulating).
 * Their records follow the last row, from offs[nx*ny] to n, with the key
 * 0xFFFFFFFF.  A zero offset and no mask give pmb_sort_rows' records. */
int pmb_sort_rows_ex(const int16_t* pmid, float* disp, const float* vel, float drift, int64_t n, int nx, int ny,
                     int nz, float cell, float ox, float oy, float oz, const uint8_t* valid, void* sorted,
                     void* scratch, int64_t scratch_bytes, void* stream);
/* Density scatter that allocates nothing and takes no workspace.  No
 * counterpart in the reference: it exists for callers that may not allocate
 * device memory (framework plugins whose host program owns every allocation
 * and hands them no scratch).  Same result as pmb_sort_rows +
 * pmb_scatter_rows (mode 0, constant val).  Its scratch is a fixed 32 MiB
 * device array inside the library (held on every GPU that loads it until
 * exit); problems needing more (28 B per particle + 12 B per mesh row) are
 * rejected before any work is queued.  Calls share that array, so calls that
 * overlap on the GPU race; the first call on a device resolves the array's
 * address and should come before any stream capture. */
int pmb_scatter_density_noalloc(const int16_t* pmid, const float* disp, int64_t n, int nx, int ny, int nz, float cell,
                                float val, float* out, void* stream);
/* Stable per-cell order of the reference key ((x*My+y)*Mz+z), ties keep
 * source order: keys_out[n] (uint32) and perm_out[n] (uint32). */
/* Status word of a sorted buffer (DeviceFlag bits: 2 non-finite displacement,
 * 4 non-finite deposit value).  Synchronises `stream`. */
int pmb_sorted_status(const void* sorted, int64_t n, int nx, int ny, int nz, uint32_t* flags, void* stream);
int pmb_sort_by_cell(const int16_t* pmid, const float* disp, int64_t n, int nx, int ny, int nz, float cell,
                     uint32_t* keys_out, uint32_t* perm_out, void* scratch, int64_t scratch_bytes, void* stream);
int64_t pmb_sort_by_cell_scratch_bytes(int64_t n, int nx, int ny, int nz);

/* ---------------- CIC on sorted particles --------------------------------
 * Deterministic scatter (cic/scatter.py:315-338, cic/pallas.py:268-303):
 * out[c] = sum_p val[p,c] * w_p.  val (n,C) or NULL for the constant
 * val_const; val is in particle order, or in sorted order when val_sorted
 * (as pmb_interp_grad_rows writes it to u_sorted).  mode 0 writes the sum;
 * mode 1 writes (sum - 1) * src_mul (the Poisson source of
 * nbody/gravity.py:628-630).  The sum is exact in 64-bit fixed point, so the
 * result does not depend on particle order.  A NaN or infinite val leaves out
 * untouched and raises flag 4 (pmb_sorted_status, pmb_device_status).
 * scratch: 16 bytes. */
int pmb_scatter_rows(const void* sorted, int64_t n, int nx, int ny, int nz, int C, const float* val, int val_sorted,
                     float val_const, int mode, float src_mul, float* out, void* scratch16, void* stream);
/* Gather (cic/gather.py:452-472, cic/pallas.py:305-318): out[p,c]; with
 * vel != NULL also vel += out * kick (nbody/integrator.py:536). */
int pmb_gather_rows(const void* sorted, int64_t n, int nx, int ny, int nz, int C, const float* mesh, float* out,
                    float* vel, float kick, void* stream);
/* pmb_gather_rows with a second half-kick vel += out * kick2 after the first
 * (the next step's opening kick, same acceleration; kick2 = 0: none).  With
 * vel != NULL, out may be NULL: the kicks only, no gathered values stored. */
int pmb_gather_rows2(const void* sorted, int64_t n, int nx, int ny, int nz, int C, const float* mesh, float* out,
                     float* vel, float kick, float kick2, void* stream);
/* Position term of the CIC adjoints (cic/gather.py:495-502,
 * cic/scatter.py:366-373): disp_cot[p] (+)= sum_b (sum_c u[p,c] mesh_c[i_b])
 * grad w_b / cell; optional wsum[p,c] = sum_b mesh_c[i_b] w_b and
 * u_sorted (n,C) = u in sorted order (input of a val_sorted scatter). */
int pmb_interp_grad_rows(const void* sorted, int64_t n, int nx, int ny, int nz, int C, const float* mesh,
                         const float* u, float u_const, float cell, int accumulate, float* disp_cot, float* wsum,
                         float* u_sorted, void* stream);

/* CIC onto a mesh whose cell size cell2 differs from the particles' cell
 * (the explicit cell_size argument of cic/scatter.py:235, cic/gather.py:414;
 * semantics of cic/pallas.py:192-222 and cic/enmesh.py:108-127): per axis,
 * p = mod((pmid * cell + disp) - o, g * cell) on the particles' periodic
 * (gx, gy, gz) mesh; corner b sits at i_b = floor(mod(p + b * cell2, g *
 * cell) / cell2) of the (nx, ny, nz) target mesh with the folded offset
 * p - i_b * cell2 giving weight 1 - |.| / cell2; corners outside the target
 * mesh are dropped.  valid (uint8, device, NULL = all valid) masks particles
 * as in pmb_sort_rows_ex.  No cell sort: the deposit sums exact 64-bit fixed
 * point with global integer atomics (deterministic) in the scratch of
 * pmb_cic_general_scratch_bytes and writes out = the deposit (not added to
 * out); the gather writes out[p, c]; interp_grad writes disp_cot[p] = sum_b
 * (sum_c u[p,c] mesh_c[i_b]) grad w_b / cell2 and wsum[p, c] (may be NULL). */
int64_t pmb_cic_general_scratch_bytes(int nx, int ny, int nz, int C);
int pmb_cic_general_scatter(const int16_t* pmid, const float* disp, const uint8_t* valid, int64_t n, int gx, int gy,
                            int gz, float cell, float ox, float oy, float oz, float cell2, int nx, int ny, int nz,
                            int C, const float* val, float val_const, float* out, void* scratch,
                            int64_t scratch_bytes, void* stream);
int pmb_cic_general_gather(const int16_t* pmid, const float* disp, const uint8_t* valid, int64_t n, int gx, int gy,
                           int gz, float cell, float ox, float oy, float oz, float cell2, int nx, int ny, int nz,
                           int C, const float* mesh, float* out, void* stream);
int pmb_cic_general_interp_grad(const int16_t* pmid, const float* disp, const uint8_t* valid, int64_t n, int gx,
                                int gy, int gz, float cell, float ox, float oy, float oz, float cell2, int nx, int ny,
                                int nz, int C, const float* mesh, const float* u, float u_const, float* disp_cot,
                                float* wsum, void* stream);

/* Mesh-row staging of pmb_gather_rows / pmb_interp_grad_rows (process-wide):
 * 0 (default) direct corner loads; 1 stage the rows a tile of particle rows
 * touches into shared memory with bulk asynchronous copies when the tile
 * holds enough particles to repay the copies; 2 stage every non-empty tile.
 * All modes give bit-identical results; staging is faster for spread-out
 * particles and slower for clustered ones. */
int pmb_set_gather_staging(int mode);
/* Count of bounded device waits (bulk-copy completions in the staged
 * gathers) that gave up since the library was loaded or the last
 * pmb_device_status; 0 in a healthy run.  Synchronous: reads a device
 * counter. */
int pmb_wait_timeouts(uint32_t* count);
/* Poll limit of the first bounded wait of every staged gather and FFT pass
 * (process-wide; a negative value restores the default 2^22 polls, 0 gives up
 * at once).  After a timeout a CTA still waits (2^22 polls) for the copies it
 * has in flight, raises the timeout counter and returns without writing the
 * tile: that launch's results are invalid. */
int pmb_set_wait_limit(int64_t polls);
/* Device-wide flags since the last call, cleared on return: 1 a bounded wait
 * gave up (either timeout counter), 2 a non-finite displacement reached a cell
 * sort, 4 a non-finite value reached a deposit.  Returns 0 when none is set,
 * else -6 with the conditions in pmb_last_error().  Synchronises the device. */
int pmb_device_status(uint32_t* flags);

/* ---------------- spectral ------------------------------------------------
 * 3-D R2C / C2R (numpy convention: forward unnormalised, the inverse is NOT
 * divided by nx*ny*nz here), batch meshes back to back.  These stand in for
 * jnp.fft.rfftn / irfftn at nbody/gravity.py:425, 528. */
int64_t pmb_fft_work_bytes(int nx, int ny, int nz, int batch);
int pmb_rfft3(int nx, int ny, int nz, int batch, float* in, void* out, void* work, void* stream);
int pmb_irfft3(int nx, int ny, int nz, int batch, void* in, float* out, void* work, void* stream);
/* tables: float [kx(nx) ky(ny) kz(nz/2+1) cx(nx) cy(ny) cz(nz/2+1)] plus,
 * when has_masks, [mx(nx) my(ny) mz(nz/2+1)] (core/configuration.py:301-307,
 * 365-376; core/utils.py:15-37).  green_kernel 0 = continuum -1/k^2
 * (gravity.py:283-285), 1 = discrete Laplacian (gravity.py:122-171, 345-352;
 * pass the effective k tables).  transfer: optional real multiplier per
 * half-spectrum cell (corrections/core.py:333-334); radial: optional table
 * indexed by integer |n|^2.  grad_hat = 3 spectra (i c_d) K S_hat * post_scale
 * (gravity.py:389-399, 506-543). */
int pmb_green_gradient(const void* src_hat, void* grad_hat, int nx, int ny, int nz, const float* tables, int has_masks,
                       int green_kernel, const float* transfer, const float* radial, int radial_len, float post_scale,
                       void* stream);
/* Adjoint of pmb_green_gradient: src_cot_hat = K sum_d conj(i c_d) A_d * post_scale. */
int pmb_green_gradient_adjoint(const void* grad_cot_hat, void* src_cot_hat, int nx, int ny, int nz,
                               const float* tables, int has_masks, int green_kernel, const float* transfer,
                               const float* radial, int radial_len, float post_scale, void* stream);

/* Interlaced CIC assignment (replaces the phase-and-average step of
 * nbody/gravity.py:440-463, _interlacing_phase / _gravity_potential_interlaced).
 * spec0 / spec1: half spectra (nx, ny, nz/2+1) complex64 of the regular deposit
 * and of the deposit shifted by half a cell on every axis (pmb_sort_rows_ex
 * offset cell/2 on x, y and z, then pmb_scatter_rows).
 * P = exp(-i (kx + ky + kz) cell / 2), k as fftfreq on x and y and rfftfreq on z.
 *   mode 0: spec0 = (spec0 + P spec1) / 2 (the interlaced source spectrum);
 *   mode 1: spec1 = conj(P) spec0 / 2, spec0 = spec0 / 2 (its transpose: a source
 *           cotangent spectrum split into the two deposits' cotangents).
 * The transpose is exact when the mesh Nyquist planes carry no signal (meshes
 * finer than the particle grid, whose particle-Nyquist masks zero them). */
int pmb_interlace_spectra(void* spec0, void* spec1, int nx, int ny, int nz, int mode, void* stream);

/* ---------------- mesh-CNN residual potential ------------------------------
 * Kernels of the mesh-CNN potential correction (replace the haiku network of
 * corrections/mesh_cnn.py:66-110 and its use in corrections/core.py:321-331;
 * the host composes the network).  Tensors are channel-planar float32
 * (C, nx, ny, nz).
 * pmb_cnn_conv3d: periodic 3x3x3 convolution (haiku Conv3D after wrap padding
 *   by one, 'VALID'): out_z[co] = bias[co] (+ res[co]) + sum_tap sum_ci
 *   in[ci](p + off) W[tap][ci][co], W as (3, 3, 3, ci, co); act 1 also writes
 *   out_h = gelu(out_z) (jax.nn.gelu, tanh form); act 2 multiplies by
 *   gelu'(zref) (a backward step).  transposed: the input gradient of a layer
 *   with weights (3, 3, 3, co, ci), read at p - off.  Channel pairs: (2, C),
 *   (C, C), (C, 1), C in {4, 8, 16} (forward orientation).
 * pmb_cnn_conv3d_wgrad: dW[tap][ci][co] += sum_p in[ci](p + off) dout[co](p),
 *   db[co] += sum_p dout[co](p) (FP64 accumulators, db nullable).
 * pmb_cnn_stem_input: x0 = [S * inv_s, phi * inv_p].
 * pmb_cnn_residual: R = g phi + c tanh(o); pmb_cnn_residual_adjoint: its
 *   transpose, dots[0] += sum Rc phi, dots[1] += sum Rc tanh(o).
 * pmb_cnn_norm_adjoint: dS = dx0[0] inv_s - S cS, dphi += dx0[1] inv_p - phi cP.
 * pmb_green_potential: P = K(k) S_hat * post (the potential spectrum, same
 *   tables and options as pmb_green_gradient); pmb_gradient_spectra:
 *   grad_d = (i c_d) (P + res_scale Q) * post (Q nullable);
 *   pmb_gradient_adjoint_plain: out = sum_d conj(i c_d) A_d * post. */
int pmb_cnn_conv3d(const float* in, int ci, const float* W, const float* bias, const float* res, const float* zref,
                   int act, float* out_z, float* out_h, int co, int nx, int ny, int nz, int transposed,
                   void* stream);
int pmb_cnn_conv3d_wgrad(const float* in, int ci, const float* dout, int co, int nx, int ny, int nz, double* dW,
                         double* db, void* stream);
int pmb_cnn_stem_input(const float* S, const float* phi, int64_t n, float inv_s, float inv_p, float* x0,
                       void* stream);
int pmb_cnn_residual(const float* phi, const float* o, int64_t n, float g, float c, float* R, void* stream);
int pmb_cnn_residual_adjoint(const float* Rc, const float* phi, const float* o, int64_t n, float g, float c,
                             float* dphi, float* dout, double* dots, void* stream);
int pmb_cnn_norm_adjoint(const float* dx0, const float* S, const float* phi, int64_t n, float inv_s, float cS,
                         float inv_p, float cP, float* dS, float* dphi, void* stream);
int pmb_green_potential(const void* src_hat, void* pot_hat, int nx, int ny, int nz, const float* tables, int has_masks,
                        int green_kernel, const float* transfer, const float* radial, int radial_len, float post_scale,
                        void* stream);
int pmb_gradient_spectra(const void* pot_hat, const void* res_hat, float res_scale, void* grad_hat, int nx, int ny,
                         int nz, const float* tables, float post_scale, void* stream);
int pmb_gradient_adjoint_plain(const void* grad_cot_hat, void* out_hat, int nx, int ny, int nz, const float* tables,
                               float post_scale, void* stream);

/* Windowed periodic projection of a C-order (nx, ny, nz) float mesh along one
 * axis (replaces the sum of nbody/observers.py:50-54 density_projection_observer
 * and the wraparound_slice sums of observers.py:113-124, core/utils.py:420-463).
 * out (the other two axes, C order) = sum over t < count of the planes
 * (start + t) mod n_axis, count = min(stop - start, max_width) (max_width < 0:
 * no cap; 0 when stop <= start).  Full projection: start 0, stop n_axis.
 * FP64 sums in a fixed order: deterministic. */
int pmb_project_density(const float* mesh, int nx, int ny, int nz, int axis, int start, int stop, int max_width,
                        float* out, void* stream);

/* ---------------- hand-written PM FFT passes -------------------------------
 * For meshes whose sides are powers of two (nx, ny in 64..1024, nz in
 * 128..1024) the fused force and its adjoint run their spectral stages as a
 * chain of hand-written passes over a y-blocked half-spectrum layout:
 * channel-major, then rows ((y/32)*nx + x)*32 + y%32 of P = nz/2 + 8 complex
 * values (columns above nz/2 zero).  pmb_pmfft_channel_elems gives the complex
 * values per channel (-1 when the mesh is not supported).  Same numpy
 * conventions as pmb_rfft3 / pmb_irfft3; the inverse drops the imaginary
 * parts of the kz = 0 and nz/2 bins like irfftn.
 *
 * pmb_pmfft_z: real rows -> blocked spectrum (inverse = 0) or back
 *   (inverse = 1), batch channels.
 * pmb_pmfft_col: one column pass; mode 0 y forward, 1 y inverse, 2 y inverse
 *   of channel ch_off into (i c_y Q, i c_z Q) (2 output channels), 3 y forward
 *   of channels ch_off, ch_off+1 combined as (-i c_y) Y + (-i c_z) Z, 4 x
 *   forward, 5 x inverse, 6 x forward + Green multiplier + x inverse into
 *   (i c_x phi, phi) (2 output channels), 7 x forward of channels 0, 1 +
 *   adjoint multiplier + x inverse, 8 the same without the x inverse.  Modes 0, 1, 4, 5 transform nbatch
 *   channels starting at ch_off; tables, transfer, radial and post_scale are
 *   those of pmb_green_gradient (tables may be null for modes 0, 1, 4, 5).
 * pmb_set_pmfft(0) routes pmb_force / pmb_force_vjp through cuFFT and the
 * separate multiplier kernels instead (default 1).
 * pmb_pmfft_z2 / pmb_pmfft_col2: the same passes as one stage of a pruned
 *   force chain (prune = 1 with particle-Nyquist masks in tables): on a mesh
 *   finer than the particle grid the masks zero every mode outside
 *   |ky| <= ny_p/2, kz <= nz_p/2 (and the same in kx), so the forward y
 *   passes (modes 0, 3) run only the live kz columns and store only the live
 *   ky rows, the x passes (6, 7) run only live (ky, kz) columns, the inverse
 *   y passes (1, 2) run only live kz columns and read only live ky rows, and
 *   the z C2R takes the dead kz columns as zeros (the z R2C is unchanged).
 *   Every pass of a chain must then be run pruned with the same tables (the
 *   skipped parts of the intermediate spectra are never written); the results
 *   equal the unpruned chain's.  pmb_force / pmb_force_vjp run their chains
 *   pruned whenever has_masks is set.
 * pmb_pmfft_timeouts: bounded copy waits in these passes that gave up.
 * pmb_pmfft_set_col_ctas(0, 1 or 2): resident CTAs per SM of the column
 *   passes, 0 = the default (one); a tuning knob, results are identical. */
int pmb_set_pmfft(int enabled);
int pmb_pmfft_supported(int nx, int ny, int nz);
int64_t pmb_pmfft_channel_elems(int nx, int ny, int nz);
int pmb_pmfft_z(int nx, int ny, int nz, int inverse, int batch, const void* in, void* out, void* stream);
int pmb_pmfft_col(int nx, int ny, int nz, int mode, int nbatch, int ch_off, const void* in, void* out,
                  const float* tables, int has_masks, const float* transfer, const float* radial, int radial_len,
                  float post_scale, void* stream);
int pmb_pmfft_z2(int nx, int ny, int nz, int inverse, int batch, const void* in, void* out, const float* tables,
                 int has_masks, int prune, void* stream);
int pmb_pmfft_col2(int nx, int ny, int nz, int mode, int nbatch, int ch_off, const void* in, void* out,
                   const float* tables, int has_masks, const float* transfer, const float* radial, int radial_len,
                   float post_scale, int prune, void* stream);
int pmb_pmfft_timeouts(uint32_t* count);
int pmb_pmfft_set_col_ctas(int ctas);

/* ---------------- fused PM force ------------------------------------------
 * One PM force evaluation (nbody/gravity.py:786-814 -> _gravity_from_density
 * :626-633 -> _streamed_acceleration_from_potential :506-543): optional
 * drift, cell sort, deterministic scatter to the Poisson source, R2C, Green x
 * gradient, batched C2R into force_meshes (3,nx,ny,nz), 3-channel gather into
 * acc (n,3), optional fused half-kick vel_kick += acc * kick.  On return
 * the first pmb_sorted_bytes(n, nx, ny, nz) bytes of the workspace hold the
 * sorted records of the (post-drift) positions. */
int64_t pmb_force_workspace_bytes(int64_t n, int nx, int ny, int nz);
int pmb_force(const int16_t* pmid, float* disp, const float* drift_vel, float drift, int64_t n, int nx, int ny, int nz,
              float cell, float val_const, float src_mul, const float* tables, int has_masks, int green_kernel,
              const float* transfer, const float* radial, int radial_len, float* force_meshes, float* acc,
              float* vel_kick, float kick, void* workspace, int64_t workspace_bytes, void* stream);
/* pmb_force with a second fused half-kick vel_kick += acc * kick2 after the
 * first (the next KDK step's opening kick; kick2 = 0: none).  With vel_kick
 * != NULL, acc may be NULL: the kicks are applied and no acceleration is
 * stored (a run whose next force overwrites it anyway). */
int pmb_force2(const int16_t* pmid, float* disp, const float* drift_vel, float drift, int64_t n, int nx, int ny, int nz,
               float cell, float val_const, float src_mul, const float* tables, int has_masks, int green_kernel,
               const float* transfer, const float* radial, int radial_len, float* force_meshes, float* acc,
               float* vel_kick, float kick, float kick2, void* workspace, int64_t workspace_bytes, void* stream);
/* Low-memory forward force: the streamed gravity of nbody/gravity.py:643-658
 * (forward only, no correction tape): sort (optional drift), deposit of the
 * Poisson source, R2C, then one force component at a time -- its Green x
 * gradient spectrum, C2R into one real mesh, a 1-channel gather -- and acc
 * (n,3) assembled from the three.  Holds one real mesh and two half spectra
 * (about 12 bytes per cell) instead of the fused force's three real meshes
 * and its spectral channels (about 36); cuFFT route, same arithmetic per
 * component as pmb_force's cuFFT route. */
int64_t pmb_force_streamed_workspace_bytes(int64_t n, int nx, int ny, int nz);
int pmb_force_streamed(const int16_t* pmid, float* disp, const float* drift_vel, float drift, int64_t n, int nx,
                       int ny, int nz, float cell, float val_const, float src_mul, const float* tables, int has_masks,
                       int green_kernel, const float* transfer, const float* radial, int radial_len, float* acc,
                       void* workspace, int64_t workspace_bytes, void* stream);
/* Transpose of pmb_force w.r.t. disp given force_meshes at the same disp
 * (the force VJP of nbody/integrator.py:620-686): disp_cot (n,3) +=
 * gather-adjoint position term + scatter-adjoint term of the density. */
int64_t pmb_force_vjp_workspace_bytes(int64_t n, int nx, int ny, int nz);
int pmb_force_vjp(const int16_t* pmid, const float* disp, int64_t n, int nx, int ny, int nz, float cell,
                  float val_const, float src_mul, const float* tables, int has_masks, int green_kernel,
                  const float* transfer, const float* radial, int radial_len, const float* force_meshes,
                  const float* acc_cot, float* disp_cot, void* workspace, int64_t workspace_bytes, void* stream);
/* pmb_force_vjp without its cell sort: sorted holds the records of exactly
 * these positions (pmb_sort_rows output, or the head of a pmb_force
 * workspace after a force evaluation at the same positions). */
int pmb_force_vjp_presorted(const void* sorted, int64_t n, int nx, int ny, int nz, float cell, float val_const,
                            float src_mul, const float* tables, int has_masks, int green_kernel,
                            const float* transfer, const float* radial, int radial_len, const float* force_meshes,
                            const float* acc_cot, float* disp_cot, void* workspace, int64_t workspace_bytes,
                            void* stream);

/* ---------------- time integration ---------------------------------------
 * y += x * f in float (drift integrator.py:225, kick :536). */
int pmb_axpy(float* y, const float* x, int64_t n, float f, void* stream);
/* Kick adjoint (integrator.py:566-580); dot (double, device) += sum vel_cot*acc. */
int pmb_kick_adj(float* vel, const float* acc, const float* vel_cot, float* acc_cot, int64_t n, float kick,
                 double* dot, void* stream);
/* One or two consecutive kick adjoints with the same acc (kick_a first),
 * bit-identical to as many pmb_kick_adj calls: dot_a (and dot_b) += sum
 * vel_cot*acc; dot_force (may be null) += sum acc_cot*acc of the updated
 * cotangent (the Omega_m term of the force adjoint that follows);
 * zero_cot = 1 treats acc_cot as zero on entry. */
int pmb_kick_adj2(float* vel, const float* acc, const float* vel_cot, float* acc_cot, int64_t n, float kick_a,
                  float kick_b, int two, int zero_cot, double* dot_a, double* dot_b, double* dot_force,
                  void* stream);
/* pmb_kick_adj2 preceded, in the same pass, by the cotangent half of the
 * drift adjoint that comes before the kicks in a reverse sweep (disp_cot may
 * be null: none): vel_cot += disp_cot * drift and dot_drift += sum disp_cot *
 * vel (vel on entry); bit-identical to pmb_drift_cot_adj then pmb_kick_adj2. */
int pmb_kick_adj3(float* vel, const float* acc, float* vel_cot, float* acc_cot, int64_t n, float kick_a, float kick_b,
                  int two, int zero_cot, double* dot_a, double* dot_b, double* dot_force, const float* disp_cot,
                  float drift, double* dot_drift, void* stream);
/* Cotangent half of pmb_drift_adj (vel_cot += disp_cot * drift, dot += sum
 * disp_cot * vel); the position half is a drift by -drift, fused into the
 * next pmb_force's sort (bit-identical to pmb_drift_adj's position update). */
int pmb_drift_cot_adj(const float* vel, const float* disp_cot, float* vel_cot, int64_t n, float drift, double* dot,
                      void* stream);
/* Drift adjoint (integrator.py:459-474); dot += sum disp_cot*vel. */
int pmb_drift_adj(float* disp, const float* vel, const float* disp_cot, float* vel_cot, int64_t n, float drift,
                  double* dot, void* stream);
/* dot (double, device) += sum a*b. */
int pmb_dot(const float* a, const float* b, int64_t n, double* dot, void* stream);
/* out (double, device) += sum a. */
int pmb_sum(const float* a, int64_t n, double* out, void* stream);

/* ---------------- initial conditions --------------------------------------
 * Nested white noise (initial_conditions/modes.py:223-268): hashed Gaussian
 * rFFT modes (gx, gy, gz/2+1) identical for shared low-k modes across
 * resolutions.  hashes_out (optional, uint32 [2 x cells]) receives the real /
 * imaginary stream hashes (modes.py:205-208). */
int pmb_white_noise_nested(uint32_t seed, int gx, int gy, int gz, void* modes_out, uint32_t* hashes_out,
                           void* stream);
/* Linear modes delta = omega sqrt(V P_lin(|k|)) (modes.py:397-454): ktables =
 * float [kx ky kz] of the particle grid; P_lin from the tabulated transfer
 * function (FP64, cosmology/boltzmann.py:428-484) times growth2 = D(a)^2 (1
 * without growth).  modes_in may be NULL to only write the amplitude
 * amp_out (float per half-spectrum cell, optional). */
int pmb_linear_modes(const void* modes_in, void* modes_out, float* amp_out, int gx, int gy, int gz,
                     const float* ktables, const double* transfer_k, const double* transfer, int ntab, double A_s,
                     double n_s, double omega_m, double k_pivot, double growth2, double box_vol, void* stream);
/* 1LPT/2LPT displacements and velocities (initial_conditions/lpt.py:337-449):
 * modes = linear modes on the particle grid; tables = float [kx ky kz cx cy
 * cz] of the particle grid; (D1, V1, D2, V2) = growth factors D_m and
 * a^2 H dD_m/dlna at a_start.  disp/vel (n,3) are updated in place for
 * particles at pmid/disp (lattice positions); fields (6, gx, gy, gz) receive
 * the sampled gradient fields and index_out (int64, n) the grid index of each
 * particle, both reused by pmb_lpt_vjp. */
int64_t pmb_lpt_workspace_bytes(int gx, int gy, int gz);
int pmb_lpt(const void* modes, int gx, int gy, int gz, float spacing, float cell_vol, const float* tables, int order,
            float D1, float V1, float D2, float V2, const int16_t* pmid, float* disp, float* vel, int64_t n,
            float cell, float* fields, int64_t* index_out, void* workspace, int64_t workspace_bytes, void* stream);
/* Adjoint of pmb_lpt w.r.t. the modes (the hand-written transpose of
 * lpt.py:379-431; packed d/dRe + i d/dIm convention, the complex conjugate of
 * JAX's gradient convention).  amp (optional) chains through the linear-mode
 * amplitude.  dots (double[4], device, accumulated): sum g_m . disp_cot and
 * sum g_m . vel_cot for m = 1, 2 (growth-factor cotangents). */
int64_t pmb_lpt_vjp_workspace_bytes(int gx, int gy, int gz);
int pmb_lpt_vjp(const void* modes, int gx, int gy, int gz, float cell_vol, const float* tables, int order, float D1,
                float V1, float D2, float V2, const int64_t* index, const float* fields, const float* disp_cot,
                const float* vel_cot, int64_t n, const float* amp, void* modes_cot, double* dots, void* workspace,
                int64_t workspace_bytes, void* stream);

/* ---------------- power spectrum ------------------------------------------
 * FP64 shell sums of |d|^2 * mult * W^-2p over integer-radius shells
 * (analysis/power_spectrum.py:120-176); sinc_tab = float sinc(n/M) per axis
 * [nx ny nz/2+1].  With spec_b, also the auto sums of b and the cross sums. */
int pmb_pk_shells(const void* spec, int nx, int ny, int nz, const float* sinc_tab, int mas_power, int num_shells,
                  double* sums, const void* spec_b, double* sums_b, double* sums_x, void* stream);
/* Mode counts and sum of |n| * mult per shell (power_spectrum.py:46-74). */
int pmb_shell_stats(int nx, int ny, int nz, int num_shells, double* counts, double* ksum, void* stream);
/* Adjoint of the shell power: out = 2 spec W^-2p wshell[shell] * post. */
int pmb_pk_shells_adjoint(const void* spec, int nx, int ny, int nz, const float* sinc_tab, int mas_power,
                          int num_shells, const double* wshell, float post, void* out, void* stream);
/* delta = rho / (total / n) - 1 (power_spectrum.py:371-374). */
int pmb_overdensity(const float* rho, float* delta, int64_t n, const double* total, void* stream);

/* ---------------- learned Green's-function correction ----------------------
 * A width-64 sin-MLP T(|k|, a, Omega_m, sigma8) = 1 + f(x) multiplying the
 * Green's function (the potential-transfer hook of corrections/core.py:
 * 286-334; cf. the radial filter of corrections/radial.py:29-216).  Weights
 * bf16 [W1 (64x4) W2 (64x64) W3 (64x64) W4 (64)], biases float [b1 b2 b3 (64
 * each) b4]; FP32 accumulation.  pmb_mlp_table evaluates T on the table of
 * integer |n|^2 = 0..len-1 (|k|/k_Ny = sqrt(n^2) * kscale) that
 * pmb_green_gradient reads as `radial`. */
int pmb_mlp_param_counts(int* n_weights, int* n_biases);
int pmb_mlp_table(const void* weights_bf16, const float* biases, float kscale, float a, float omega_m, float sigma8,
                  int len, float* table, void* stream);
/* grad (float, weights then biases) += d/dparams sum_n table_cot[n] T[n]. */
int pmb_mlp_backward(const void* weights_bf16, const float* biases, float kscale, float a, float omega_m,
                     float sigma8, int len, const double* table_cot, float* grad, void* stream);
/* out[n^2] += dL/dT for one force adjoint: grad_cot_hat = rFFT of the three
 * force-mesh cotangents, src_hat = rFFT of the Poisson source at the same
 * positions. */
int pmb_transfer_cot(const void* grad_cot_hat, const void* src_hat, int nx, int ny, int nz, const float* tables,
                     int has_masks, int len, double* out, void* stream);

/* ---------------- host-side FP64 cosmology (no device work) ---------------
 * Growth table [order 1..2][deriv 0..2][na] from the growth ODE integrated
 * with the adaptive Dormand-Prince scheme of numerics/ode.py:304-422 at the
 * scale factors growth_a (cosmology/boltzmann.py:177-249); dtable_dom
 * (optional) receives d table / d Omega_m by complex-step differentiation. */
int pmb_growth_table(double omega_m, double omega_k, double w0, double wa, const double* growth_a, int na,
                     double a_lpt_step, double rtol, double atol, double dt0, double* table, double* dtable_dom);
/* kind 0: drift factor (integrator.py:125-146) for (a_vel, a_prev, a_next);
 * kind 1: kick factor (integrator.py:149-170) for (a_acc, a_prev, a_next).
 * dfactor_dom (optional) needs dtable_dom. */
int pmb_time_factor(int kind, double a0, double a1, double a2, double omega_m, double omega_k, double w0, double wa,
                    const double* growth_a, int na, const double* table, const double* dtable_dom, double* factor,
                    double* dfactor_dom);
/* LPT growth factors at a (initial_conditions/lpt.py:412-417): out[m-1][0..2]
 * = (D_m, dD_m/dlna, a^2 H dD_m/dlna) for m = 1, 2; dout = d/d Omega_m. */
int pmb_lpt_factors(double a, double omega_m, double omega_k, double w0, double wa, const double* growth_a, int na,
                    const double* table, const double* dtable_dom, double* out, double* dout);
/* Eisenstein & Hu transfer fit (cosmology/boltzmann.py:33-137). */
int pmb_transfer_fit(const double* k, int64_t nk, double omega_m, double omega_b, double h, double T_cmb,
                     int nowiggle, double* out);
/* Linear power without growth (cosmology/boltzmann.py:428-484) from a
 * tabulated transfer function (tk, tt). */
int pmb_linear_power(const double* k, int64_t nk, const double* tk, const double* tt, int ntab, double A_s,
                     double n_s, double omega_m, double h, double k_pivot_Mpc, double* out);

/* ---------------- float64 build ---------------------------------------------
 * The reference's x64 configuration (jax_enable_x64): the same operations in
 * double precision with cuFFT D2Z / Z2D, for float64 parity.  Not the
 * optimised path: the deposit uses double atomics without a sort.
 * pmb_force64: optional drift disp += drift_vel * drift, CIC deposit of val,
 * source (rho - 1) * src_mul, D2Z, Green x gradient (tables: float64
 * [kx ky kz cx cy cz (mx my mz)], the discrete-Laplacian k and FastPM's
 * derivative when a correction asks for them; transfer: the correction's
 * float64 multiplier per half-spectrum cell, or NULL, corrections/core.py:
 * 333-334), 3 x Z2D into force_meshes (3, nx, ny, nz),
 * gather into acc with optional vel_kick += acc * kick (nbody/gravity.py:
 * 786-814, nbody/integrator.py:202-238, 512-538).  pmb_deposit64: the density
 * alone (cic/scatter.py:315-338).  pmb_lpt64 / pmb_linear_modes64 /
 * pmb_white_noise_nested64 / pmb_pk_shells64 / pmb_overdensity64: float64
 * versions of the float32 entry points of the same names. */
int64_t pmb_force64_workspace_bytes(int nx, int ny, int nz);
int pmb_force64(const int16_t* pmid, double* disp, const double* drift_vel, double drift, int64_t n, int nx, int ny,
                int nz, double cell, double val, double src_mul, const double* tables, int has_masks,
                const double* transfer, double* force_meshes, double* acc, double* vel_kick, double kick,
                void* workspace, int64_t workspace_bytes, void* stream);
int pmb_deposit64(const int16_t* pmid, const double* disp, int64_t n, int nx, int ny, int nz, double cell, double val,
                  double* rho, void* stream);
int pmb_axpy64(double* y, const double* x, int64_t n, double f, void* stream);
int pmb_sum64(const double* a, int64_t n, double* out, void* stream);
/* Force adjoint of pmb_force64 at the same positions (replaces the float64
 * jax.vjp of gravity, nbody/gravity.py:786-814, as the float32
 * pmb_force_vjp does): disp_cot += (d acc / d disp)^T acc_cot -- the gather
 * adjoint's position term, the deposit of acc_cot, D2Z, the transposed
 * Green x gradient (post src_mul / cells), Z2D and the deposit adjoint's
 * position term with the deposited value val (cic/gather.py:475-548,
 * cic/scatter.py:341-437).  force_meshes are pmb_force64's at these
 * positions. */
int64_t pmb_force_vjp64_workspace_bytes(int nx, int ny, int nz);
int pmb_force_vjp64(const int16_t* pmid, const double* disp, int64_t n, int nx, int ny, int nz, double cell,
                    double val, double src_mul, const double* tables, int has_masks, const double* transfer,
                    const double* force_meshes, const double* acc_cot, double* disp_cot, void* workspace,
                    int64_t workspace_bytes, void* stream);
/* Interlaced forms of pmb_force64 / pmb_force_vjp64 (nbody/gravity.py:440-463,
 * 809-811): a second deposit on the mesh shifted by half a cell, one batched
 * D2Z, the average (S + S_shift P) / 2 with P = exp(-i (kx + ky + kz) cell / 2)
 * as the source spectrum, then the same multiplier, Z2D and gather at the
 * regular origin; the adjoint splits the source cotangent back with conj(P)
 * / 2 and / 2 and takes both deposits' adjoints.  Same arguments; the
 * workspaces hold the second mesh and spectrum. */
int64_t pmb_force64_interlaced_workspace_bytes(int nx, int ny, int nz);
int pmb_force64_interlaced(const int16_t* pmid, double* disp, const double* drift_vel, double drift, int64_t n, int nx,
                           int ny, int nz, double cell, double val, double src_mul, const double* tables,
                           int has_masks, const double* transfer, double* force_meshes, double* acc, double* vel_kick,
                           double kick, void* workspace, int64_t workspace_bytes, void* stream);
int64_t pmb_force_vjp64_interlaced_workspace_bytes(int nx, int ny, int nz);
int pmb_force_vjp64_interlaced(const int16_t* pmid, const double* disp, int64_t n, int nx, int ny, int nz,
                               double cell, double val, double src_mul, const double* tables, int has_masks,
                               const double* transfer, const double* force_meshes, const double* acc_cot,
                               double* disp_cot, void* workspace, int64_t workspace_bytes, void* stream);
/* *out += sum a[i] b[i] in float64 (the Omega_m cotangent dots of the float64
 * reverse sweep, nbody/integrator.py:173-199). */
int pmb_dot64(const double* a, const double* b, int64_t n, double* out, void* stream);
int64_t pmb_fft64_work_bytes(int nx, int ny, int nz, int batch);
int pmb_rfft3_64(int nx, int ny, int nz, int batch, double* in, void* out, void* work, void* stream);
int pmb_irfft3_64(int nx, int ny, int nz, int batch, void* in, double* out, void* work, void* stream);
int pmb_white_noise_nested64(uint32_t seed, int gx, int gy, int gz, void* out, void* stream);
int pmb_linear_modes64(const void* modes_in, void* modes_out, int gx, int gy, int gz, const double* kvec,
                       const double* tk, const double* tt, int ntab, double A_s, double n_s, double omega_m,
                       double k_pivot, double growth2, double box_vol, void* stream);
int64_t pmb_lpt64_workspace_bytes(int gx, int gy, int gz);
int pmb_lpt64(const void* modes, int gx, int gy, int gz, double spacing, double cell_vol, const double* tables,
              int order, double D1, double V1, double D2, double V2, const int16_t* pmid, double* disp, double* vel,
              int64_t n, double cell, double* fields, void* workspace, int64_t workspace_bytes, void* stream);
/* pmb_lpt64 with index_out (nullable): each particle's Lagrangian grid cell,
 * which the float64 LPT adjoint needs, as pmb_lpt's index_out. */
int pmb_lpt64_ex(const void* modes, int gx, int gy, int gz, double spacing, double cell_vol, const double* tables,
                 int order, double D1, double V1, double D2, double V2, const int16_t* pmid, double* disp,
                 double* vel, int64_t n, double cell, double* fields, int64_t* index_out, void* workspace,
                 int64_t workspace_bytes, void* stream);
/* float64 pmb_lpt_vjp (replaces the x64 jax.vjp of lpt, initial_conditions/
 * lpt.py:337-449, as pmb_lpt_vjp does in float32): same arguments in double
 * precision (modes / modes_cot complex128, fields, cotangents and amp
 * float64), the same packed dL/dRe + i dL/dIm convention and growth-factor
 * dots. */
int64_t pmb_lpt_vjp64_workspace_bytes(int gx, int gy, int gz);
int pmb_lpt_vjp64(const void* modes, int gx, int gy, int gz, double cell_vol, const double* tables, int order,
                  double D1, double V1, double D2, double V2, const int64_t* index, const double* fields,
                  const double* disp_cot, const double* vel_cot, int64_t n, const double* amp, void* modes_cot,
                  double* dots, void* workspace, int64_t workspace_bytes, void* stream);
/* Position term of the float64 deposit's adjoint for a constant deposited
 * value (cic/scatter.py:366-370): disp_cot += val * sum_b mesh_cot[i_b]
 * grad w_b / cell, particles binned directly (no sort), as pmb_deposit64. */
int pmb_scatter_vjp64(const int16_t* pmid, const double* disp, int64_t n, int nx, int ny, int nz, double cell,
                      double val, const double* mesh_cot, double* disp_cot, void* stream);
int pmb_pk_shells64(const void* spec, int nx, int ny, int nz, const double* sinc_tab, int mas_power, int num_shells,
                    double* sums, void* stream);
/* float64 form of pmb_pk_shells_adjoint (power_spectrum.py:120-143 transposed):
 * out = 2 spec W^-2p wshell[shell] * post, complex128 half spectra. */
int pmb_pk_shells_adjoint64(const void* spec, int nx, int ny, int nz, const double* sinc_tab, int mas_power,
                            int num_shells, const double* wshell, double post, void* out, void* stream);
int pmb_overdensity64(const double* rho, double* delta, int64_t n, const double* total, void* stream);

/* ---------------- ensembles of independent simulations --------------------
 * No single counterpart in the reference, which advances one simulation per
 * call (nbody/solver.py:253-273) and batches only by a Python loop or a vmap
 * over equal shapes.  An ensemble advances many PM simulations of uneven
 * sizes together, one persistent launch per PM stage over all of them; each
 * simulation gets exactly the single-simulation arithmetic of pmb_sort_rows /
 * pmb_scatter_rows (mode 1) / pmb_green_gradient / pmb_gather_rows / pmb_axpy.
 *
 * pmb_ens_create (host only): nsims descriptions -- particle counts,
 * mesh_shapes[3*s], mesh cell sizes, deposit per particle (mesh cells /
 * particles), Poisson source factor 1.5*Omega_m, particle-Nyquist mask flag --
 * and the number of kick-drift-kick steps whose factors it stores.
 * Simulations with equal mesh shape must be consecutive (one batched FFT per
 * shape); ordering them by decreasing mesh size balances the persistent
 * scatter.  The handle owns host memory only.
 * pmb_ens_workspace_bytes: device workspace for pmb_ens_bind (256-byte
 * aligned).  pmb_ens_size: 0 particles, 1 mesh cells, 2 half-spectrum cells,
 * 3 scatter tiles, 4 distinct mesh shapes.
 * pmb_ens_bind: concatenated particle arrays (simulation order), the
 * concatenated Poisson source meshes rho (sum of cells), their spectra
 * (sum of half cells), three gradient spectra and three force meshes per
 * simulation ([3][cells] each, simulation after simulation), the spectral
 * tables of every mesh (pmb_green_gradient layout) at table_offsets[s] floats
 * into `tables` (host array of offsets).  Enqueues the descriptor upload.
 * pmb_ens_set_factors: host table [nsteps][nsims][3] of float factors
 * (opening kick K1, drift D, closing kick K2 of each step,
 * nbody/integrator.py:125-170).  pmb_ens_set_step: device step counter.
 * pmb_ens_force: sort (with drift: disp += vel*D of the current step), scatter
 * of the Poisson source, R2C, Green x gradient, 3 x C2R, gather into acc
 * (with kick: vel += acc*K2 of the current step).
 * pmb_ens_step: vel += acc*K1, pmb_ens_force(drift, kick), step += 1 -- a
 * kick-drift-kick step that a CUDA graph can capture once and replay.
 * pmb_ens_stage: one stage alone (0 kick, 1 sort, 2 scatter, 3 R2C, 4 Green,
 * 5 C2R, 6 gather) for tuning.  pmb_ens_set_tiles: per-simulation scatter
 * tile rows (rx, ry <= 4); pmb_ens_set_launch: threads and CTAs per SM of a
 * particle or cell stage.  Changes of tiles take effect at the next
 * uncaptured call. */
int pmb_ens_create(int nsims, const int64_t* counts, const int32_t* mesh_shapes, const float* cells,
                   const float* vals, const float* src_muls, const int32_t* has_masks, int max_steps, void** handle);
int pmb_ens_destroy(void* handle);
int64_t pmb_ens_workspace_bytes(const void* handle);
int64_t pmb_ens_size(const void* handle, int which);
int pmb_ens_bind(void* handle, const int16_t* pmid, float* disp, float* vel, float* acc, float* rho, void* rho_hat,
                 void* grad_hat, float* force, const float* tables, const int64_t* table_offsets, void* workspace,
                 int64_t workspace_bytes, void* stream);
int pmb_ens_set_tiles(void* handle, const int32_t* rx, const int32_t* ry);
int pmb_ens_set_launch(void* handle, int stage, int threads, int ctas_per_sm);
int pmb_ens_set_factors(void* handle, int nsteps, const float* factors, void* stream);
int pmb_ens_set_step(void* handle, int step, void* stream);
int pmb_ens_stage(void* handle, int stage, int drift, int kick, void* stream);
int pmb_ens_force(void* handle, int drift, int kick, void* stream);
int pmb_ens_step(void* handle, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* PMB200_H */
