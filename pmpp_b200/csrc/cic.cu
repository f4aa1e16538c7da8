// Cell sort, deterministic CIC scatter, CIC gather and their adjoints.
//
// Reference semantics: cic/enmesh.py:34-165 (binning, weights, weight
// gradients), cic/scatter.py:315-437 and cic/gather.py:452-548 (forward and
// hand-written VJPs), cic/pallas.py:268-409 (the GPU kernels this replaces).
//
// B200 design:
//  * particles are counting-sorted by the mesh row (x, y) of their lower CIC
//    corner.  Bin order is the reference's raveled cell-key order
//    ((x*My + y)*Mz + z, core/utils.py:292-326) at row granularity;
//  * the scatter is a pull kernel: one CTA owns an RX x RY block of output
//    rows, reads the particles of the (RX+1) x (RY+1) source rows that can
//    reach it, and accumulates in shared memory in 64-bit fixed point.  The
//    result is independent of accumulation order (bit-deterministic), every
//    output cell is written exactly once with coalesced stores, and no
//    global atomics or mesh zero-fill pass are needed;
//  * gathers and adjoint position terms walk particles in sorted order so the
//    eight corner loads of neighbouring threads hit the same cache lines.
#include <cstdio>

#include "pmb_cic_device.cuh"
#include "pmb_common.cuh"
#include "pmb_kernels.cuh"
#include "pmb_tma.cuh"

namespace pmb {

// ---------------------------------------------------------------------------
// Binning
// ---------------------------------------------------------------------------
// Count particles per row.  Optionally applies the drift disp += vel * D
// first (integrator.py:223-225, two roundings as in the reference) and writes
// the drifted displacement back.  Ranks come from warp-aggregated atomics.
__global__ void bin_count_kernel(const int16_t* __restrict__ pmid, float* __restrict__ disp,
                                 const float* __restrict__ vel, float drift, int64_t n, Mesh3 m, float cell,
                                 uint32_t* __restrict__ counts, uint32_t* __restrict__ row_of,
                                 uint32_t* __restrict__ rank_of) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  bool active = i < n;
  uint32_t row = 0xFFFFFFFFu;
  if (active) {
    float d0 = disp[3 * i], d1 = disp[3 * i + 1], d2 = disp[3 * i + 2];
    if (vel != nullptr) {
      d0 = __fadd_rn(d0, __fmul_rn(vel[3 * i], drift));
      d1 = __fadd_rn(d1, __fmul_rn(vel[3 * i + 1], drift));
      d2 = __fadd_rn(d2, __fmul_rn(vel[3 * i + 2], drift));
      disp[3 * i] = d0;
      disp[3 * i + 1] = d1;
      disp[3 * i + 2] = d2;
    }
    Binned b = bin_particle(pmid, d0, d1, d2, i, m, cell);
    row = (uint32_t)((int64_t)b.cx * m.ny + b.cy);
  }
  unsigned full = __ballot_sync(0xFFFFFFFFu, active);
  if (!active) return;
  unsigned peers = __match_any_sync(full, row);
  int leader = __ffs(peers) - 1;
  int lane = threadIdx.x & 31;
  uint32_t base = 0;
  if (lane == leader) base = atomicAdd(&counts[row], (uint32_t)__popc(peers));
  base = __shfl_sync(peers, base, leader);
  row_of[i] = row;
  rank_of[i] = base + __popc(peers & ((1u << lane) - 1u));
}

__global__ void bin_place_kernel(const int16_t* __restrict__ pmid, const float* __restrict__ disp, int64_t n,
                                 Mesh3 m, float cell, const uint32_t* __restrict__ offs,
                                 const uint32_t* __restrict__ row_of, const uint32_t* __restrict__ rank_of,
                                 Rec* __restrict__ rec, uint32_t* __restrict__ perm) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  Binned b = bin_particle(pmid, disp[3 * i], disp[3 * i + 1], disp[3 * i + 2], i, m, cell);
  uint32_t dst = offs[row_of[i]] + rank_of[i];
  Rec r;
  r.fx = b.fx;
  r.fy = b.fy;
  r.fz = b.fz;
  r.key = (uint32_t)(((int64_t)b.cx * m.ny + b.cy) * m.nz + b.cz);
  rec[dst] = r;
  perm[dst] = (uint32_t)i;
}

// Exclusive scan of row counts, three phases over tiles of 4096 entries.
constexpr int kScanThreads = 1024;
constexpr int kScanPer = 4;
constexpr int kScanTile = kScanThreads * kScanPer;

__device__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* sh, uint32_t* total) {
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t x = v;
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) sh[warp] = x;
  __syncthreads();
  if (warp == 0) {
    uint32_t w = lane < (blockDim.x >> 5) ? sh[lane] : 0;
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xFFFFFFFFu, w, o);
      if (lane >= o) w += y;
    }
    sh[lane] = w;
  }
  __syncthreads();
  uint32_t warp_off = warp ? sh[warp - 1] : 0;
  if (total) *total = sh[(blockDim.x >> 5) - 1];
  uint32_t r = warp_off + x - v;
  __syncthreads();
  return r;
}

__global__ void scan_tiles_kernel(const uint32_t* __restrict__ in, uint32_t* __restrict__ out, int64_t n,
                                  uint32_t* __restrict__ tile_sums) {
  __shared__ uint32_t sh[32];
  int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanPer;
  uint32_t v[kScanPer];
  uint32_t s = 0;
  for (int j = 0; j < kScanPer; ++j) {
    v[j] = (base + j < n) ? in[base + j] : 0u;
    s += v[j];
  }
  uint32_t total;
  uint32_t off = block_exclusive_scan(s, sh, &total);
  for (int j = 0; j < kScanPer; ++j) {
    if (base + j < n) out[base + j] = off;
    off += v[j];
  }
  if (threadIdx.x == 0) tile_sums[blockIdx.x] = total;
}

__global__ void scan_sums_kernel(uint32_t* __restrict__ sums, int64_t ntiles, uint32_t* __restrict__ grand) {
  __shared__ uint32_t sh[32];
  uint32_t carry = 0;
  for (int64_t b = 0; b < ntiles; b += blockDim.x) {
    int64_t i = b + threadIdx.x;
    uint32_t v = i < ntiles ? sums[i] : 0u;
    uint32_t total;
    uint32_t off = block_exclusive_scan(v, sh, &total);
    if (i < ntiles) sums[i] = carry + off;
    carry += total;
  }
  if (threadIdx.x == 0) *grand = carry;
}

__global__ void scan_add_kernel(uint32_t* __restrict__ out, int64_t n, const uint32_t* __restrict__ sums) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] += sums[i / kScanTile];
}

int64_t scan_tmp_elems(int64_t len) { return (len + kScanTile - 1) / kScanTile + 1; }

// Exclusive scan of len uint32 values (in == out allowed); tile_sums needs
// scan_tmp_elems(len) entries.
int exclusive_scan_u32(const uint32_t* in, uint32_t* out, int64_t len, uint32_t* tile_sums, cudaStream_t s) {
  if (len <= 0) return kOk;
  const int64_t ntiles = (len + kScanTile - 1) / kScanTile;
  scan_tiles_kernel<<<(unsigned)ntiles, kScanThreads, 0, s>>>(in, out, len, tile_sums);
  scan_sums_kernel<<<1, 1024, 0, s>>>(tile_sums, ntiles, tile_sums + ntiles);
  scan_add_kernel<<<(unsigned)((len + 255) / 256), 256, 0, s>>>(out, len, tile_sums);
  PMB_CUDA_CHECK(cudaGetLastError());
  return kOk;
}

int64_t bin_scratch_bytes(int64_t n, Mesh3 m) {
  int64_t rows = m.rows();
  int64_t ntiles = (rows + 1 + kScanTile - 1) / kScanTile;
  return align_up(4 * (rows + 1), 256) * 2 + align_up(4 * n, 256) * 2 + align_up(4 * (ntiles + 1), 256);
}

// Sort particles by lower-corner row.  Outputs rec[n], perm[n] and
// offs[rows + 1] (offs lives inside the caller's scratch, returned pointer).
int bin_particles(const int16_t* pmid, float* disp, const float* vel, float drift, int64_t n, Mesh3 m, float cell,
                  Rec* rec, uint32_t* perm, uint32_t* offs, void* scratch, cudaStream_t s) {
  int64_t rows = m.rows();
  char* p = (char*)scratch;
  uint32_t* counts = (uint32_t*)p;
  p += align_up(4 * (rows + 1), 256);
  uint32_t* row_of = (uint32_t*)p;
  p += align_up(4 * n, 256);
  uint32_t* rank_of = (uint32_t*)p;
  p += align_up(4 * n, 256);
  uint32_t* tile_sums = (uint32_t*)p;
  int64_t len = rows + 1;
  int64_t ntiles = (len + kScanTile - 1) / kScanTile;
  PMB_CUDA_CHECK(cudaMemsetAsync(counts, 0, 4 * len, s));
  if (n > 0) {
    int th = 256;
    bin_count_kernel<<<(unsigned)((n + th - 1) / th), th, 0, s>>>(pmid, disp, vel, drift, n, m, cell, counts, row_of,
                                                                    rank_of);
  }
  (void)ntiles;
  int st = exclusive_scan_u32(counts, offs, len, tile_sums, s);
  if (st != kOk) return st;
  if (n > 0) {
    int th = 256;
    bin_place_kernel<<<(unsigned)((n + th - 1) / th), th, 0, s>>>(pmid, disp, n, m, cell, offs, row_of, rank_of,
                                                                    rec, perm);
  }
  PMB_CUDA_CHECK(cudaGetLastError());
  return kOk;
}

// ---------------------------------------------------------------------------
// Fixed-point scale for the deterministic scatter
// ---------------------------------------------------------------------------
// Contributions val*w are converted to int64 units of 1/scale with the power
// of two scale = 2^e / 2^ceil(log2 max|val|), e = 62 - ceil(log2(n + 1)) (at
// most 52), so that the sum of up to n contributions of magnitude <= max|val|
// cannot overflow and val*w*scale is exact in float.
__global__ void absmax_kernel(const float* __restrict__ v, int64_t count, unsigned int* __restrict__ out) {
  float mx = 0.f;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (int64_t)gridDim.x * blockDim.x) {
    float a = fabsf(v[i]);
    if (a > mx || a != a) mx = (a != a) ? __int_as_float(0x7f800000) : a;
  }
  for (int o = 16; o; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xFFFFFFFFu, mx, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, __float_as_uint(mx));
}

__global__ void scale_from_absmax_kernel(const unsigned int* __restrict__ bits, double pow2e, double* __restrict__ scale) {
  float mx = __uint_as_float(*bits);
  // A non-finite maximum leaves no usable scale: flag it with a NaN scale.
  if (!(mx < __int_as_float(0x7f800000))) {
    *scale = __longlong_as_double(0x7ff8000000000000ll);
    return;
  }
  *scale = fixed_point_scale(pow2e, mx);
}

double fixed_point_pow2(int64_t n) {
  int e = 62;
  int64_t t = n + 1;
  int lg = 0;
  while ((int64_t(1) << lg) < t) ++lg;
  e -= lg;
  if (e > 52) e = 52;
  return ldexp(1.0, e);
}

int compute_scale(const float* val, int64_t count, int64_t n, double* scale_dev, unsigned int* tmp, cudaStream_t s) {
  PMB_CUDA_CHECK(cudaMemsetAsync(tmp, 0, sizeof(unsigned int), s));
  if (count > 0) {
    int blocks = (int)((count + 255) / 256);
    if (blocks > 4096) blocks = 4096;
    absmax_kernel<<<blocks, 256, 0, s>>>(val, count, tmp);
  }
  scale_from_absmax_kernel<<<1, 1, 0, s>>>(tmp, fixed_point_pow2(n), scale_dev);
  PMB_CUDA_CHECK(cudaGetLastError());
  return kOk;
}

// ---------------------------------------------------------------------------
// Pull scatter
// ---------------------------------------------------------------------------
// Epilogue: mode 0 writes the density sum, mode 1 writes the Poisson source
// (rho - 1) * src_mul (gravity.py:628-630), both in float.
template <int C>
__global__ void __launch_bounds__(256) scatter_pull_kernel(const Rec* __restrict__ rec, const uint32_t* __restrict__ perm,
                                                           const uint32_t* __restrict__ offs, Mesh3 m, int RX, int RY,
                                                           const float* __restrict__ val, int val_sorted,
                                                           float val_const, const double* __restrict__ scale_dev,
                                                           int mode, float src_mul, float* __restrict__ out) {
  extern __shared__ __align__(16) unsigned int acc_smem[];  // ScatterSmem::acc_bytes(RX, RY, C, nz)
  __shared__ ScatterSmem sm;
  const int nby = (m.ny + RY - 1) / RY;
  const int x0 = (int)(blockIdx.x / nby) * RX;
  const int y0 = (int)(blockIdx.x % nby) * RY;
  scatter_tile<C>(rec, perm, offs, m, RX, RY, x0, y0, val, val_sorted, val_const, *scale_dev, mode, src_mul, out,
                  acc_smem, sm);
}

void scatter_block_shape(Mesh3 m, int C, int* RX, int* RY) {
  // First of 2x2, 1x2, 1x1 output rows whose accumulator fits the budget:
  // 100 KB for one or two channels, 40 KB for three or four (more resident
  // blocks beat the extra particle re-reads there; larger blocks measured
  // slower everywhere).
  const int64_t budget = (C >= 3 ? 40 : 100) * 1024;
  static const int shapes[3][2] = {{2, 2}, {1, 2}, {1, 1}};
  int rx = 1, ry = 1;
  for (const auto& sh : shapes) {
    if (ScatterSmem::acc_bytes(sh[0], sh[1], C, m.nz) <= budget) {
      rx = sh[0];
      ry = sh[1];
      break;
    }
  }
  *RX = rx < m.nx ? rx : m.nx;
  *RY = ry < m.ny ? ry : m.ny;
}

int scatter_sorted(const Rec* rec, const uint32_t* perm, const uint32_t* offs, Mesh3 m, int C, const float* val,
                   int val_sorted, float val_const, const double* scale_dev, int mode, float src_mul, float* out,
                   cudaStream_t s) {
  int RX, RY;
  scatter_block_shape(m, C, &RX, &RY);
  const int64_t smem = ScatterSmem::acc_bytes(RX, RY, C, m.nz);
  if (smem > 200 * 1024) return kUnsupported;
  const int nbx = (m.nx + RX - 1) / RX, nby = (m.ny + RY - 1) / RY;
  const unsigned grid = (unsigned)((int64_t)nbx * nby);
#define PMB_LAUNCH_SCATTER(CC)                                                                                   \
  do {                                                                                                           \
    PMB_CUDA_CHECK(smem_optin((const void*)scatter_pull_kernel<CC>, 200 * 1024));                              \
    scatter_pull_kernel<CC><<<grid, 256, (size_t)smem, s>>>(rec, perm, offs, m, RX, RY, val, val_sorted,         \
                                                             val_const, scale_dev, mode, src_mul, out);         \
  } while (0)
  switch (C) {
    case 1: PMB_LAUNCH_SCATTER(1); break;
    case 2: PMB_LAUNCH_SCATTER(2); break;
    case 3: PMB_LAUNCH_SCATTER(3); break;
    case 4: PMB_LAUNCH_SCATTER(4); break;
    default: return kUnsupported;
  }
#undef PMB_LAUNCH_SCATTER
  PMB_CUDA_CHECK(cudaGetLastError());
  return kOk;
}

// ---------------------------------------------------------------------------
// Gather and adjoint position terms
// ---------------------------------------------------------------------------
// out[src, c] = sum_b mesh_c[i_b] w_b (gather.py:452-472, pallas.py:305-318).
// With vel the half-kick vel += out * kick is applied in place (integrator.py:536),
// and with kick2 != 0 the next step's opening half-kick after it, saving passes
// over the particles.
template <int C>
__global__ void gather_kernel(const Rec* __restrict__ rec, const uint32_t* __restrict__ perm, int64_t n, Mesh3 m,
                              const float* __restrict__ mesh, float* __restrict__ out, float* __restrict__ vel,
                              float kick, float kick2) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  gather_one<C>(rec[i], perm[i], m, mesh, out, vel, kick, kick2);
}

// ---------------------------------------------------------------------------
// Staged gathers: the mesh rows a tile of particle rows touches are copied
// into shared memory with bulk asynchronous copies, then every particle of
// the tile interpolates from shared memory.
// ---------------------------------------------------------------------------
__device__ unsigned int g_wait_timeouts_cic = 0;

// 0: direct corner loads (default); 1: stage the rows of tiles with enough
// particles; 2: stage every non-empty tile.  Staging wins on spread-out
// particles and loses on clustered ones, whose corner loads already hit in
// L1/L2, so it is opt-in.
static int g_gather_staging = 0;

void set_gather_staging(int mode) { g_gather_staging = mode; }

constexpr int kStageMaxRX = 4;
constexpr int64_t kStageBudget = 110 * 1024;

// Shared bytes of the staged rows of an RX x RY tile with C channels.
inline int64_t stage_bytes(int RX, int RY, int C, int nz) { return (int64_t)(RX + 1) * (RY + 1) * C * nz * 4; }

// Tile of particle rows whose staged mesh rows fit the budget; false when the
// mesh rows cannot be bulk-copied (nz % 4 != 0 or a misaligned mesh).
bool stage_shape(Mesh3 m, int C, const float* mesh, int* RX, int* RY) {
  if (g_gather_staging == 0 || m.nz % 4 != 0 || ((uintptr_t)mesh & 15) != 0) return false;
  static const int shapes[5][2] = {{4, 4}, {2, 4}, {2, 2}, {1, 2}, {1, 1}};
  for (const auto& sh : shapes) {
    if (sh[0] <= m.nx && sh[1] <= m.ny && stage_bytes(sh[0], sh[1], C, m.nz) <= kStageBudget) {
      *RX = sh[0];
      *RY = sh[1];
      return true;
    }
  }
  return false;
}

// Tiles with fewer particles than this load their corners directly: staging
// costs the tile's rows, a direct gather about one 32-byte sector per corner
// and channel of every particle.
inline uint32_t stage_threshold(int64_t smem, int C) {
  return g_gather_staging == 2 ? 1u : (uint32_t)(smem / (8 * 32 * C));
}

// Copies the (RX+1) x (RY+1) mesh rows (periodic) of C channels starting at
// row (x0, y0) into stage[c][ix][iy][nz].  Returns false (after flagging the
// timeout) when the copies do not complete.
__device__ __forceinline__ bool stage_mesh_rows(float* stage, const float* __restrict__ mesh, Mesh3 m, int C, int x0,
                                                int y0, int RX, int RY, uint64_t* bar) {
  const int SX = RX + 1, SY = RY + 1;
  if (threadIdx.x == 0) {
    mbar_init(bar, 1);
    const uint32_t row_bytes = (uint32_t)m.nz * 4u;
    mbar_expect_tx(bar, row_bytes * (uint32_t)(SX * SY * C));
    const int64_t cells = m.cells();
    for (int c = 0; c < C; ++c)
      for (int ix = 0; ix < SX; ++ix) {
        const int x = x0 + ix >= m.nx ? x0 + ix - m.nx : x0 + ix;
        for (int iy = 0; iy < SY; ++iy) {
          const int y = y0 + iy >= m.ny ? y0 + iy - m.ny : y0 + iy;
          bulk_copy_g2s(stage + ((c * SX + ix) * SY + iy) * m.nz, mesh + c * cells + ((int64_t)x * m.ny + y) * m.nz,
                        row_bytes, bar);
        }
      }
  }
  __syncthreads();
  return mbar_wait_or_flag(bar, 0, &g_wait_timeouts_cic);
}

// Particle segments of the tile: rows (x0 + k, y0 .. y0+RY-1) are contiguous
// in the sorted records for each k.  Returns the particle count.
__device__ __forceinline__ uint32_t tile_segments(const uint32_t* __restrict__ offs, Mesh3 m, int x0, int y0, int RX,
                                                  int RY, uint32_t* seg_b, uint32_t* seg_n) {
  if (threadIdx.x < RX) {
    const int x = x0 + threadIdx.x;
    uint32_t b = 0, c = 0;
    if (x < m.nx) {
      const int y1 = y0 + RY < m.ny ? y0 + RY : m.ny;
      b = offs[(int64_t)x * m.ny + y0];
      c = offs[(int64_t)x * m.ny + y1] - b;
    }
    seg_b[threadIdx.x] = b;
    seg_n[threadIdx.x] = c;
  }
  __syncthreads();
  uint32_t total = 0;
  for (int k = 0; k < RX; ++k) total += seg_n[k];
  return total;
}

// Sorted index and tile-local row (k, iy) of the j-th particle of the tile.
__device__ __forceinline__ uint32_t tile_particle(uint32_t j, const uint32_t* seg_b, const uint32_t* seg_n, int* k) {
  int kk = 0;
  while (j >= seg_n[kk]) {
    j -= seg_n[kk];
    ++kk;
  }
  *k = kk;
  return seg_b[kk] + j;
}

// Same arithmetic as gather_one, reading the staged rows.
template <int C>
__global__ void __launch_bounds__(256) gather_staged_kernel(const Rec* __restrict__ rec, const uint32_t* __restrict__ perm,
                                                            const uint32_t* __restrict__ offs, Mesh3 m, int RX, int RY,
                                                            uint32_t min_stage, const float* __restrict__ mesh,
                                                            float* __restrict__ out, float* __restrict__ vel,
                                                            float kick, float kick2) {
  extern __shared__ __align__(16) float stage[];
  __shared__ __align__(8) uint64_t bar;
  __shared__ uint32_t seg_b[kStageMaxRX], seg_n[kStageMaxRX];
  const int nby = (m.ny + RY - 1) / RY;
  const int x0 = (int)(blockIdx.x / nby) * RX, y0 = (int)(blockIdx.x % nby) * RY;
  const uint32_t total = tile_segments(offs, m, x0, y0, RX, RY, seg_b, seg_n);
  if (total == 0) return;
  if (total < min_stage) {
    // too few particles to pay for staging the rows: load corners directly
    for (uint32_t j = threadIdx.x; j < total; j += blockDim.x) {
      int k;
      const uint32_t i = tile_particle(j, seg_b, seg_n, &k);
      gather_one<C>(rec[i], perm[i], m, mesh, out, vel, kick, kick2);
    }
    return;
  }
  if (!stage_mesh_rows(stage, mesh, m, C, x0, y0, RX, RY, &bar)) return;
  const int SX = RX + 1, SY = RY + 1, nz = m.nz;
  for (uint32_t j = threadIdx.x; j < total; j += blockDim.x) {
    int k;
    const uint32_t i = tile_particle(j, seg_b, seg_n, &k);
    const Rec r = rec[i];
    const uint32_t row = r.key / (uint32_t)nz;
    const int cz = (int)(r.key - row * (uint32_t)nz);
    const int iy = (int)(row - (uint32_t)(x0 + k) * (uint32_t)m.ny) - y0;
    const int z1 = cz + 1 == nz ? 0 : cz + 1;
    const float wx[2] = {axis_weight(r.fx, 0), axis_weight(r.fx, 1)};
    const float wy[2] = {axis_weight(r.fy, 0), axis_weight(r.fy, 1)};
    const float wz[2] = {axis_weight(r.fz, 0), axis_weight(r.fz, 1)};
    const uint32_t src = perm[i];
#pragma unroll
    for (int c = 0; c < C; ++c) {
      float a = 0.f;
#pragma unroll
      for (int b = 0; b < 8; ++b) {
        const int bx = b & 1, by = (b >> 1) & 1, bz = (b >> 2) & 1;
        const float v = stage[((c * SX + k + bx) * SY + iy + by) * nz + (bz ? z1 : cz)];
        a = __fadd_rn(a, __fmul_rn(v, __fmul_rn(__fmul_rn(wx[bx], wy[by]), wz[bz])));
      }
      out[(int64_t)src * C + c] = a;
      if (vel != nullptr) vel[(int64_t)src * C + c] = kicked(vel[(int64_t)src * C + c], a, kick, kick2);
    }
  }
}

// Direct gather with two particles per thread: both particles' 8C corner
// loads are issued before either sum, doubling the loads in flight of this
// latency-bound kernel (10% faster on clustered particles at 512^3, same
// arithmetic per particle as gather_one).
template <int C>
__global__ void __launch_bounds__(256) gather_kernel_x2(const Rec* __restrict__ rec, const uint32_t* __restrict__ perm,
                                                        int64_t n, Mesh3 m, const float* __restrict__ mesh,
                                                        float* __restrict__ out, float* __restrict__ vel, float kick,
                                                        float kick2) {
  const int64_t i0 = (int64_t)blockIdx.x * (2 * blockDim.x) + threadIdx.x;
  const int64_t i1 = i0 + blockDim.x;
  if (i0 >= n) return;
  const bool two = i1 < n;
  const Rec r0 = rec[i0];
  const Rec r1 = two ? rec[i1] : r0;
  Corners k0, k1;
  corners_of(r0, m, k0);
  corners_of(r1, m, k1);
  const uint32_t s0 = perm[i0], s1 = two ? perm[i1] : s0;
  // velocities of the folded kicks, loaded ahead of the corner loads so their
  // latency (particle-order addresses) overlaps them instead of following
  // each channel's sum
  float u0[C], u1[C];
  if (vel != nullptr) {
#pragma unroll
    for (int c = 0; c < C; ++c) {
      u0[c] = vel[(int64_t)s0 * C + c];
      u1[c] = vel[(int64_t)s1 * C + c];
    }
  }
  const int64_t cells = m.cells();
#pragma unroll
  for (int c = 0; c < C; ++c) {
    const float* mc = mesh + (int64_t)c * cells;
    float v0[8], v1[8];
#pragma unroll
    for (int b = 0; b < 8; ++b) {
      v0[b] = __ldg(mc + k0.idx[b]);
      v1[b] = __ldg(mc + k1.idx[b]);
    }
    float a0 = 0.f, a1 = 0.f;
#pragma unroll
    for (int b = 0; b < 8; ++b) {
      a0 = __fadd_rn(a0, __fmul_rn(v0[b], k0.w[b]));
      a1 = __fadd_rn(a1, __fmul_rn(v1[b], k1.w[b]));
    }
    out[(int64_t)s0 * C + c] = a0;
    if (vel != nullptr) vel[(int64_t)s0 * C + c] = kicked(u0[c], a0, kick, kick2);
    if (two) {
      out[(int64_t)s1 * C + c] = a1;
      if (vel != nullptr) vel[(int64_t)s1 * C + c] = kicked(u1[c], a1, kick, kick2);
    }
  }
}

int gather_sorted(const Rec* rec, const uint32_t* perm, const uint32_t* offs, int64_t n, Mesh3 m, int C,
                  const float* mesh, float* out, float* vel, float kick, float kick2, cudaStream_t s) {
  if (n == 0) return kOk;
  int RX, RY;
  if (offs != nullptr && stage_shape(m, C, mesh, &RX, &RY)) {
    const int64_t smem = stage_bytes(RX, RY, C, m.nz);
    const uint32_t min_stage = stage_threshold(smem, C);
    const unsigned grid = (unsigned)((int64_t)((m.nx + RX - 1) / RX) * ((m.ny + RY - 1) / RY));
#define PMB_LAUNCH_GS(CC)                                                                                      \
  do {                                                                                                         \
    PMB_CUDA_CHECK(smem_optin((const void*)gather_staged_kernel<CC>, (int)kStageBudget));                     \
    gather_staged_kernel<CC><<<grid, 256, (size_t)smem, s>>>(rec, perm, offs, m, RX, RY, min_stage, mesh, out, vel, \
                                                              kick, kick2);                                     \
  } while (0)
    switch (C) {
      case 1: PMB_LAUNCH_GS(1); break;
      case 2: PMB_LAUNCH_GS(2); break;
      case 3: PMB_LAUNCH_GS(3); break;
      case 4: PMB_LAUNCH_GS(4); break;
      default: return kUnsupported;
    }
#undef PMB_LAUNCH_GS
    PMB_CUDA_CHECK(cudaGetLastError());
    return kOk;
  }
  const int th = 256;
  const unsigned g = (unsigned)((n + th - 1) / th);
  if (C == 3) {
    gather_kernel_x2<3><<<(unsigned)((n + 2 * th - 1) / (2 * th)), th, 0, s>>>(rec, perm, n, m, mesh, out, vel, kick,
                                                                              kick2);
    PMB_CUDA_CHECK(cudaGetLastError());
    return kOk;
  }
  switch (C) {
    case 1: gather_kernel<1><<<g, th, 0, s>>>(rec, perm, n, m, mesh, out, vel, kick, kick2); break;
    case 2: gather_kernel<2><<<g, th, 0, s>>>(rec, perm, n, m, mesh, out, vel, kick, kick2); break;
    case 3: gather_kernel<3><<<g, th, 0, s>>>(rec, perm, n, m, mesh, out, vel, kick, kick2); break;
    case 4: gather_kernel<4><<<g, th, 0, s>>>(rec, perm, n, m, mesh, out, vel, kick, kick2); break;
    default: return kUnsupported;
  }
  PMB_CUDA_CHECK(cudaGetLastError());
  return kOk;
}

int wait_timeouts(unsigned int* count) {
  PMB_CUDA_CHECK(cudaMemcpyFromSymbol(count, g_wait_timeouts_cic, sizeof(unsigned int)));
  return kOk;
}

// Position term of the CIC adjoints.  With per-particle weights u (N, C) or a
// constant u_const:
//   inner_b = sum_c u_c * mesh_c[i_b]
//   disp_cot[src] (+)= (sum_b inner_b * grad w_b) / cell
// This is gather.py:495-502 (u = val_cot) and scatter.py:366-370 (u = val).
// Optionally also emits wsum[src, c] = sum_b mesh_c[i_b] w_b (the scatter
// adjoint's val cotangent, scatter.py:372-373) and u_sorted[i, c] =
// u[src, c] (the weights in sorted order, so a following scatter of u reads
// them coalesced instead of through the permutation).
// Per-particle body shared by the direct and staged kernels; fetch(c, b)
// returns channel c of corner b (bit a of b: +1 along axis a).  With
// accumulate, dprev (if given) holds disp_cot[src] loaded by the caller ahead
// of the corner loads.
template <int C, class Fetch>
__device__ __forceinline__ void interp_grad_one(const Rec& r, uint32_t src, int64_t i, const Fetch& fetch,
                                                const float* __restrict__ u, float u_const, float cell, int accumulate,
                                                float* __restrict__ disp_cot, float* __restrict__ wsum,
                                                float* __restrict__ u_sorted, const float* dprev = nullptr) {
  const float f[3] = {r.fx, r.fy, r.fz};
  float wa[3][2], sg[3][2];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    wa[a][0] = axis_weight(f[a], 0);
    wa[a][1] = axis_weight(f[a], 1);
    sg[a][0] = axis_sign(f[a], 0);
    sg[a][1] = axis_sign(f[a], 1);
  }
  float uu[C];
#pragma unroll
  for (int c = 0; c < C; ++c) uu[c] = u ? u[(int64_t)src * C + c] : u_const;
  if (u_sorted != nullptr) {
#pragma unroll
    for (int c = 0; c < C; ++c) u_sorted[i * C + c] = uu[c];
  }
  float g0 = 0.f, g1 = 0.f, g2 = 0.f;
  float ws[C];
#pragma unroll
  for (int c = 0; c < C; ++c) ws[c] = 0.f;
#pragma unroll
  for (int b = 0; b < 8; ++b) {
    const int bx = b & 1, by = (b >> 1) & 1, bz = (b >> 2) & 1;
    float inner = 0.f;
    const float w = __fmul_rn(__fmul_rn(wa[0][bx], wa[1][by]), wa[2][bz]);
#pragma unroll
    for (int c = 0; c < C; ++c) {
      const float mv = fetch(c, b);
      inner = __fadd_rn(inner, __fmul_rn(uu[c], mv));
      ws[c] = __fadd_rn(ws[c], __fmul_rn(mv, w));
    }
    // grad_i = sign_i * w_{i+1} * w_{i+2} (enmesh.py:155-160)
    const float gx = __fmul_rn(__fmul_rn(sg[0][bx], wa[1][by]), wa[2][bz]);
    const float gy = __fmul_rn(__fmul_rn(sg[1][by], wa[2][bz]), wa[0][bx]);
    const float gz = __fmul_rn(__fmul_rn(sg[2][bz], wa[0][bx]), wa[1][by]);
    g0 = __fadd_rn(g0, __fmul_rn(inner, gx));
    g1 = __fadd_rn(g1, __fmul_rn(inner, gy));
    g2 = __fadd_rn(g2, __fmul_rn(inner, gz));
  }
  g0 = __fdiv_rn(g0, cell);
  g1 = __fdiv_rn(g1, cell);
  g2 = __fdiv_rn(g2, cell);
  float* dc = disp_cot + 3 * (int64_t)src;
  if (accumulate) {
    dc[0] = __fadd_rn(dprev ? dprev[0] : dc[0], g0);
    dc[1] = __fadd_rn(dprev ? dprev[1] : dc[1], g1);
    dc[2] = __fadd_rn(dprev ? dprev[2] : dc[2], g2);
  } else {
    dc[0] = g0;
    dc[1] = g1;
    dc[2] = g2;
  }
  if (wsum != nullptr) {
#pragma unroll
    for (int c = 0; c < C; ++c) wsum[(int64_t)src * C + c] = ws[c];
  }
}

template <int C>
__global__ void interp_grad_kernel(const Rec* __restrict__ rec, const uint32_t* __restrict__ perm, int64_t n, Mesh3 m,
                                   const float* __restrict__ mesh, const float* __restrict__ u, float u_const,
                                   float cell, int accumulate, float* __restrict__ disp_cot,
                                   float* __restrict__ wsum, float* __restrict__ u_sorted) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const Rec r = rec[i];
  Corners k;
  corners_of(r, m, k);
  const int64_t cells = m.cells();
  auto fetch = [&](int c, int b) { return __ldg(mesh + (int64_t)c * cells + k.idx[b]); };
  interp_grad_one<C>(r, perm[i], i, fetch, u, u_const, cell, accumulate, disp_cot, wsum, u_sorted);
}

// Two particles per thread, as gather_kernel_x2.
template <int C>
__global__ void __launch_bounds__(256) interp_grad_kernel_x2(const Rec* __restrict__ rec,
                                                             const uint32_t* __restrict__ perm, int64_t n, Mesh3 m,
                                                             const float* __restrict__ mesh,
                                                             const float* __restrict__ u, float u_const, float cell,
                                                             int accumulate, float* __restrict__ disp_cot,
                                                             float* __restrict__ wsum, float* __restrict__ u_sorted) {
  const int64_t i0 = (int64_t)blockIdx.x * (2 * blockDim.x) + threadIdx.x;
  const int64_t i1 = i0 + blockDim.x;
  if (i0 >= n) return;
  const bool two = i1 < n;
  const Rec r0 = rec[i0];
  const Rec r1 = two ? rec[i1] : r0;
  Corners k0, k1;
  corners_of(r0, m, k0);
  corners_of(r1, m, k1);
  const uint32_t s0 = perm[i0], s1 = two ? perm[i1] : s0;
  // accumulated position cotangents, loaded ahead of the corner loads: read
  // after each particle's sums, their particle-order latency ran in series
  float d0[3] = {0.f, 0.f, 0.f}, d1[3] = {0.f, 0.f, 0.f};
  if (accumulate) {
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      d0[a] = disp_cot[3 * (int64_t)s0 + a];
      d1[a] = disp_cot[3 * (int64_t)s1 + a];
    }
  }
  const int64_t cells = m.cells();
  float v0[C][8], v1[C][8];
#pragma unroll
  for (int c = 0; c < C; ++c)
#pragma unroll
    for (int b = 0; b < 8; ++b) {
      v0[c][b] = __ldg(mesh + (int64_t)c * cells + k0.idx[b]);
      v1[c][b] = __ldg(mesh + (int64_t)c * cells + k1.idx[b]);
    }
  auto f0 = [&](int c, int b) { return v0[c][b]; };
  interp_grad_one<C>(r0, s0, i0, f0, u, u_const, cell, accumulate, disp_cot, wsum, u_sorted, d0);
  if (two) {
    auto f1 = [&](int c, int b) { return v1[c][b]; };
    interp_grad_one<C>(r1, s1, i1, f1, u, u_const, cell, accumulate, disp_cot, wsum, u_sorted, d1);
  }
}

template <int C>
__global__ void __launch_bounds__(256) interp_grad_staged_kernel(
    const Rec* __restrict__ rec, const uint32_t* __restrict__ perm, const uint32_t* __restrict__ offs, Mesh3 m, int RX,
    int RY, uint32_t min_stage, const float* __restrict__ mesh, const float* __restrict__ u, float u_const, float cell,
    int accumulate, float* __restrict__ disp_cot, float* __restrict__ wsum, float* __restrict__ u_sorted) {
  extern __shared__ __align__(16) float stage[];
  __shared__ __align__(8) uint64_t bar;
  __shared__ uint32_t seg_b[kStageMaxRX], seg_n[kStageMaxRX];
  const int nby = (m.ny + RY - 1) / RY;
  const int x0 = (int)(blockIdx.x / nby) * RX, y0 = (int)(blockIdx.x % nby) * RY;
  const uint32_t total = tile_segments(offs, m, x0, y0, RX, RY, seg_b, seg_n);
  if (total == 0) return;
  if (total < min_stage) {
    const int64_t cells = m.cells();
    for (uint32_t j = threadIdx.x; j < total; j += blockDim.x) {
      int k;
      const uint32_t i = tile_particle(j, seg_b, seg_n, &k);
      const Rec r = rec[i];
      Corners kc;
      corners_of(r, m, kc);
      auto fetch = [&](int c, int b) { return __ldg(mesh + (int64_t)c * cells + kc.idx[b]); };
      interp_grad_one<C>(r, perm[i], i, fetch, u, u_const, cell, accumulate, disp_cot, wsum, u_sorted);
    }
    return;
  }
  if (!stage_mesh_rows(stage, mesh, m, C, x0, y0, RX, RY, &bar)) return;
  const int SX = RX + 1, SY = RY + 1, nz = m.nz;
  for (uint32_t j = threadIdx.x; j < total; j += blockDim.x) {
    int k;
    const uint32_t i = tile_particle(j, seg_b, seg_n, &k);
    const Rec r = rec[i];
    const uint32_t row = r.key / (uint32_t)nz;
    const int cz = (int)(r.key - row * (uint32_t)nz);
    const int iy = (int)(row - (uint32_t)(x0 + k) * (uint32_t)m.ny) - y0;
    const int z1 = cz + 1 == nz ? 0 : cz + 1;
    auto fetch = [&](int c, int b) {
      const int bx = b & 1, by = (b >> 1) & 1, bz = (b >> 2) & 1;
      return stage[((c * SX + k + bx) * SY + iy + by) * nz + (bz ? z1 : cz)];
    };
    interp_grad_one<C>(r, perm[i], i, fetch, u, u_const, cell, accumulate, disp_cot, wsum, u_sorted);
  }
}

int interp_grad_sorted(const Rec* rec, const uint32_t* perm, const uint32_t* offs, int64_t n, Mesh3 m, int C,
                       const float* mesh, const float* u, float u_const, float cell, int accumulate, float* disp_cot,
                       float* wsum, float* u_sorted, cudaStream_t s) {
  if (n == 0) return kOk;
  int RX, RY;
  if (offs != nullptr && stage_shape(m, C, mesh, &RX, &RY)) {
    const int64_t smem = stage_bytes(RX, RY, C, m.nz);
    const uint32_t min_stage = stage_threshold(smem, C);
    const unsigned grid = (unsigned)((int64_t)((m.nx + RX - 1) / RX) * ((m.ny + RY - 1) / RY));
#define PMB_LAUNCH_IS(CC)                                                                                       \
  do {                                                                                                          \
    PMB_CUDA_CHECK(smem_optin((const void*)interp_grad_staged_kernel<CC>, (int)kStageBudget));                 \
    interp_grad_staged_kernel<CC><<<grid, 256, (size_t)smem, s>>>(rec, perm, offs, m, RX, RY, min_stage, mesh, u, \
                                                                   u_const, cell, accumulate, disp_cot, wsum,   \
                                                                   u_sorted);                                   \
  } while (0)
    switch (C) {
      case 1: PMB_LAUNCH_IS(1); break;
      case 2: PMB_LAUNCH_IS(2); break;
      case 3: PMB_LAUNCH_IS(3); break;
      case 4: PMB_LAUNCH_IS(4); break;
      default: return kUnsupported;
    }
#undef PMB_LAUNCH_IS
    PMB_CUDA_CHECK(cudaGetLastError());
    return kOk;
  }
  const int th = 256;
  const unsigned g = (unsigned)((n + th - 1) / th);
  const unsigned g2 = (unsigned)((n + 2 * th - 1) / (2 * th));
  if (C == 1) {
    interp_grad_kernel_x2<1><<<g2, th, 0, s>>>(rec, perm, n, m, mesh, u, u_const, cell, accumulate, disp_cot, wsum,
                                               u_sorted);
    PMB_CUDA_CHECK(cudaGetLastError());
    return kOk;
  }
  if (C == 3) {
    interp_grad_kernel_x2<3><<<g2, th, 0, s>>>(rec, perm, n, m, mesh, u, u_const, cell, accumulate, disp_cot, wsum,
                                               u_sorted);
    PMB_CUDA_CHECK(cudaGetLastError());
    return kOk;
  }
  switch (C) {
    case 1: interp_grad_kernel<1><<<g, th, 0, s>>>(rec, perm, n, m, mesh, u, u_const, cell, accumulate, disp_cot, wsum, u_sorted); break;
    case 2: interp_grad_kernel<2><<<g, th, 0, s>>>(rec, perm, n, m, mesh, u, u_const, cell, accumulate, disp_cot, wsum, u_sorted); break;
    case 3: interp_grad_kernel<3><<<g, th, 0, s>>>(rec, perm, n, m, mesh, u, u_const, cell, accumulate, disp_cot, wsum, u_sorted); break;
    case 4: interp_grad_kernel<4><<<g, th, 0, s>>>(rec, perm, n, m, mesh, u, u_const, cell, accumulate, disp_cot, wsum, u_sorted); break;
    default: return kUnsupported;
  }
  PMB_CUDA_CHECK(cudaGetLastError());
  return kOk;
}

}  // namespace pmb
