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

// Sticky device-wide flags (DeviceFlag bits), read and cleared by
// pmb_device_status.
__device__ unsigned int g_device_flags = 0;

// Raises flag f in the sorted buffer's status word (if any) and device-wide.
__device__ __forceinline__ void raise_flag(uint32_t* status, unsigned int f) {
  if (status != nullptr) atomicOr(status, f);
  atomicOr(&g_device_flags, f);
}

// Consumers of a sorted buffer whose sort was flagged write nothing.
__device__ __forceinline__ bool flagged(const uint32_t* status) { return status != nullptr && *status != 0u; }

// ---------------------------------------------------------------------------
// Binning
// ---------------------------------------------------------------------------
// Count particles per row.  Optionally applies the drift disp += vel * D
// first (integrator.py:223-225, two roundings as in the reference) and writes
// the drifted displacement back.  Ranks come from warp-aggregated atomics.
// With a shift the mesh origin moves (BinShift); particles with valid[i] == 0
// go to the extra bin after the last row (their records trail the sorted
// array with kMaskedKey).
__global__ void bin_count_kernel(const int16_t* __restrict__ pmid, float* __restrict__ disp,
                                 const float* __restrict__ vel, float drift, int64_t n, Mesh3 m, float cell,
                                 BinShift sh, const uint8_t* __restrict__ valid, uint32_t* __restrict__ counts,
                                 uint32_t* __restrict__ row_of, uint32_t* __restrict__ rank_of,
                                 uint32_t* __restrict__ status) {
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
    if (!(isfinite(d0) && isfinite(d1) && isfinite(d2))) raise_flag(status, kFlagNonFiniteDisp);
    if (valid != nullptr && !valid[i]) {
      row = (uint32_t)m.rows();
    } else {
      Binned b = bin_particle(pmid, d0, d1, d2, i, m, cell, sh);
      row = (uint32_t)((int64_t)b.cx * m.ny + b.cy);
    }
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
                                 Mesh3 m, float cell, BinShift sh, const uint32_t* __restrict__ offs,
                                 const uint32_t* __restrict__ row_of, const uint32_t* __restrict__ rank_of,
                                 Rec* __restrict__ rec, uint32_t* __restrict__ perm) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t row = row_of[i];
  uint32_t dst = offs[row] + rank_of[i];
  Rec r;
  if (row == (uint32_t)m.rows()) {
    r.fx = r.fy = r.fz = 0.f;
    r.key = kMaskedKey;
  } else {
    Binned b = bin_particle(pmid, disp[3 * i], disp[3 * i + 1], disp[3 * i + 2], i, m, cell, sh);
    r.fx = b.fx;
    r.fy = b.fy;
    r.fz = b.fz;
    r.key = (uint32_t)(((int64_t)b.cx * m.ny + b.cy) * m.nz + b.cz);
  }
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
                  Rec* rec, uint32_t* perm, uint32_t* offs, void* scratch, cudaStream_t s, const BinShift* shift,
                  const uint8_t* valid, uint32_t* status) {
  BinShift sh{0, 0, 0, 0.f, 0.f, 0.f};
  if (shift != nullptr) sh = *shift;
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
  if (status != nullptr) PMB_CUDA_CHECK(cudaMemsetAsync(status, 0, 4, s));
  if (n > 0) {
    int th = 256;
    bin_count_kernel<<<(unsigned)((n + th - 1) / th), th, 0, s>>>(pmid, disp, vel, drift, n, m, cell, sh, valid,
                                                                    counts, row_of, rank_of, status);
  }
  (void)ntiles;
  int st = exclusive_scan_u32(counts, offs, len, tile_sums, s);
  if (st != kOk) return st;
  if (n > 0) {
    int th = 256;
    bin_place_kernel<<<(unsigned)((n + th - 1) / th), th, 0, s>>>(pmid, disp, n, m, cell, sh, offs, row_of,
                                                                    rank_of, rec, perm);
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
                                                           int mode, float src_mul, float* __restrict__ out,
                                                           uint32_t* __restrict__ status) {
  extern __shared__ __align__(16) unsigned int acc_smem[];  // ScatterSmem::acc_bytes(RX, RY, C, nz)
  __shared__ ScatterSmem sm;
  if (flagged(status)) return;
  if (!(*scale_dev == *scale_dev)) {  // NaN scale: a non-finite value
    if (threadIdx.x == 0) raise_flag(status, kFlagNonFiniteValue);
    return;
  }
  const int nby = (m.ny + RY - 1) / RY;
  const int x0 = (int)(blockIdx.x / nby) * RX;
  const int y0 = (int)(blockIdx.x % nby) * RY;
  scatter_tile<C>(rec, perm, offs, m, RX, RY, x0, y0, val, val_sorted, val_const, *scale_dev, mode, src_mul, out,
                  acc_smem, sm);
}

// ---------------------------------------------------------------------------
// Pull scatter with 32-bit planes (meshes with nz % 4 == 0)
// ---------------------------------------------------------------------------
// Same exact fixed-point sums as scatter_tile, in 8 bytes per output cell:
// each contribution q = rint(val * w * scale) (64-bit in scatter_tile) is
// split as q = h * 2^s + l with h = rint(q / 2^s) and |l| <= 2^(s-1), and h
// and l are summed by signed 32-bit shared atomics on two planes.  The block
// picks s from its particle count K (every cell takes at most K
// contributions, K < 2^L) and the global bound |q| <= 2^E:
//   s >= E - 21        keeps |q / 2^s| < 2^22, so h and l come from float
//                      additions of the magic constant 1.5 * 2^23 (exact,
//                      round-half-even like the 64-bit conversion);
//   s >= L + E - 31    keeps |sum h| < 2^31;    s <= 32 - L keeps |sum l| < 2^31;
//   s <= 22            keeps l exact in the same float addition.
// A block without such an s (tiny particle counts give E up to 52, or a
// block holding very many particles) adds the 64-bit q with 64-bit atomics
// on the same 8 bytes.  The recombined sum h * 2^s + l equals the 64-bit sum
// exactly, so the output is bit-identical to scatter_tile's.
//
// Work is handed out in chunks of 32 particles of one source row, so a warp
// always works on one row and its corner set is a compile-time case (no
// divergence, no bounds tests per corner).
constexpr float kMagic = 12582912.0f;  // 1.5 * 2^23
constexpr int kMagicBits = 0x4B400000;

struct SplitAcc {
  unsigned int* acc;
  int cells;
  float y_scale;  // scale * 2^-s
  float two_s;    // 2^s
  // q = rint(contrib * scale) as h * 2^s + l: t = y + M rounds y = q / 2^s
  // to h (the float ulp at M is 1), y - h is exact (Sterbenz), and
  // fma(y - h, 2^s, M) rounds (y - h) 2^s to l in the same way.
  __device__ __forceinline__ void add(int a, float contrib) const {
    const float y = __fmul_rn(contrib, y_scale);
    const float t = __fadd_rn(y, kMagic);
    const float r = __fsub_rn(y, __fsub_rn(t, kMagic));
    const float u = __fmaf_rn(r, two_s, kMagic);
    atomicAdd(reinterpret_cast<int*>(&acc[a]), __float_as_int(u) - kMagicBits);
    atomicAdd(reinterpret_cast<int*>(&acc[cells + a]), __float_as_int(t) - kMagicBits);
  }
};

// Deposit of one particle of source row (SX, SY) relative to the block.
template <int C, int RX, int RY, int SX, int SY, bool SPLIT>
__device__ __forceinline__ void deposit_row(const Rec& r, const float* v, int nz, int cz, const SplitAcc& A,
                                            unsigned long long* acc64, double scale) {
  const int cz1 = cz + 1 == nz ? 0 : cz + 1;
  const float wz0 = axis_weight(r.fz, 0), wz1 = axis_weight(r.fz, 1);
#pragma unroll
  for (int bx = 0; bx < 2; ++bx) {
    const int lx = SX + bx;
    if (lx < 0 || lx >= RX) continue;
    const float wx = axis_weight(r.fx, bx);
#pragma unroll
    for (int by = 0; by < 2; ++by) {
      const int ly = SY + by;
      if (ly < 0 || ly >= RY) continue;
      const float wxy = __fmul_rn(wx, axis_weight(r.fy, by));
      const float w0 = __fmul_rn(wxy, wz0), w1 = __fmul_rn(wxy, wz1);
#pragma unroll
      for (int c = 0; c < C; ++c) {
        const int base = ((lx * RY + ly) * C + c) * nz;
        const float c0 = __fmul_rn(v[c], w0), c1 = __fmul_rn(v[c], w1);
        if (SPLIT) {
          A.add(base + cz, c0);
          A.add(base + cz1, c1);
        } else {
          atomicAdd(&acc64[base + cz], (unsigned long long)__double2ll_rn((double)c0 * scale));
          atomicAdd(&acc64[base + cz1], (unsigned long long)__double2ll_rn((double)c1 * scale));
        }
      }
    }
  }
}

// Dispatch on the source row index k = (SX + 1) * (RY + 1) + (SY + 1).
template <int C, int RX, int RY, bool SPLIT, int K = 0>
__device__ __forceinline__ void deposit_k(int k, const Rec& r, const float* v, int nz, int cz, const SplitAcc& A,
                                          unsigned long long* acc64, double scale) {
  if constexpr (K < (RX + 1) * (RY + 1)) {
    if (k == K) {
      deposit_row<C, RX, RY, K / (RY + 1) - 1, K % (RY + 1) - 1, SPLIT>(r, v, nz, cz, A, acc64, scale);
      return;
    }
    deposit_k<C, RX, RY, SPLIT, K + 1>(k, r, v, nz, cz, A, acc64, scale);
  }
}

// Epilogue of the split scatters: (float)(sum / scale) as scatter_tile
// computes it, for the block's RX x RY rows of C channels.  With |h|, |l| <
// 2^22 both convert exactly through the magic constant and one fma forms
// h 2^s + l with a single rounding; |sum| < 2^53, so this equals the
// double-precision route (which the other cells take).
template <int C, int RX, int RY>
__device__ __forceinline__ void split_epilogue(const unsigned int* acc, int cells, bool split, int s, double scale,
                                               float two_s, Mesh3 m, int x0, int y0, int mode, float src_mul,
                                               float* __restrict__ out) {
  const double inv = 1.0 / scale;
  const float invf = (float)inv;
  const bool fconv = split && invf >= 0x1p-126f;
  const int64_t mcells = m.cells();
  const int nz = m.nz, nz4 = nz >> 2;
  const unsigned long long* acc64 = reinterpret_cast<const unsigned long long*>(acc);
#pragma unroll
  for (int lx = 0; lx < RX; ++lx) {
    if (x0 + lx >= m.nx) break;
#pragma unroll
    for (int ly = 0; ly < RY; ++ly) {
      if (y0 + ly >= m.ny) break;
      const int64_t row_off = ((int64_t)(x0 + lx) * m.ny + (y0 + ly)) * nz;
#pragma unroll
      for (int c = 0; c < C; ++c) {
        const int a0 = ((lx * RY + ly) * C + c) * nz;
        float* o = out + (int64_t)c * mcells + row_off;
        for (int z4 = threadIdx.x; z4 < nz4; z4 += blockDim.x) {
          float res[4];
          if (split) {
            const int4 lo = *reinterpret_cast<const int4*>(&acc[a0 + 4 * z4]);
            const int4 hi = *reinterpret_cast<const int4*>(&acc[cells + a0 + 4 * z4]);
            const int los[4] = {lo.x, lo.y, lo.z, lo.w};
            const int his[4] = {hi.x, hi.y, hi.z, hi.w};
#pragma unroll
            for (int q = 0; q < 4; ++q) {
              const int h = his[q], l = los[q];
              if (fconv && h > -(1 << 22) && h < (1 << 22) && l > -(1 << 22) && l < (1 << 22)) {
                const float hf = __fsub_rn(__int_as_float(kMagicBits + h), kMagic);
                const float lf = __fsub_rn(__int_as_float(kMagicBits + l), kMagic);
                res[q] = __fmul_rn(__fmaf_rn(hf, two_s, lf), invf);
              } else {
                res[q] = (float)((double)((long long)h * (1ll << s) + (long long)l) * inv);
              }
            }
          } else {
#pragma unroll
            for (int q = 0; q < 4; ++q) res[q] = (float)((double)(long long)acc64[a0 + 4 * z4 + q] * inv);
          }
          if (mode == 1) {
#pragma unroll
            for (int q = 0; q < 4; ++q) res[q] = __fmul_rn(__fsub_rn(res[q], 1.0f), src_mul);
          }
          *reinterpret_cast<float4*>(o + 4 * z4) = make_float4(res[0], res[1], res[2], res[3]);
        }
      }
    }
  }
}

// Split parameters of a block holding ntot particles (contributions per cell
// at most ntot * dup): the plane shift s and whether the 32-bit planes apply.
__device__ __forceinline__ void split_shift(uint32_t ntot, int dup, int E, double scale, int& s, bool& split) {
  const uint64_t kmax = (uint64_t)ntot * (uint64_t)dup;
  const int L = kmax ? 64 - __clzll((long long)kmax) : 0;  // kmax < 2^L
  s = E - 21;
  if (L + E - 31 > s) s = L + E - 31;
  if (s < 1) s = 1;
  split = s <= 22 && s <= 32 - L && scale < 0x1p126;
}

template <int C, int RX, int RY>
__global__ void __launch_bounds__(256) scatter_split_kernel(const Rec* __restrict__ rec,
                                                            const uint32_t* __restrict__ perm,
                                                            const uint32_t* __restrict__ offs, Mesh3 m,
                                                            const float* __restrict__ val, int val_sorted,
                                                            float val_const, const double* __restrict__ scale_dev,
                                                            int E, int dup, int mode, float src_mul,
                                                            float* __restrict__ out, uint32_t* __restrict__ status) {
  constexpr int NSRC = (RX + 1) * (RY + 1);
  if (flagged(status)) return;
  if (!(*scale_dev == *scale_dev)) {  // NaN scale: a non-finite value
    if (threadIdx.x == 0) raise_flag(status, kFlagNonFiniteValue);
    return;
  }
  extern __shared__ __align__(16) unsigned int acc[];  // 8 * RX * RY * C * nz bytes
  __shared__ uint32_t seg_beg[NSRC], seg_cnt[NSRC], item_pre[NSRC + 1];
  __shared__ uint32_t s_ntot;
  const int nby = (m.ny + RY - 1) / RY;
  const int x0 = (int)(blockIdx.x / nby) * RX, y0 = (int)(blockIdx.x % nby) * RY;
  const int nz = m.nz;
  const int cells = RX * RY * C * nz;
  {
    uint4* a4 = reinterpret_cast<uint4*>(acc);
    const int n4 = (2 * cells) >> 2;
    for (int t = threadIdx.x; t < n4; t += blockDim.x) a4[t] = make_uint4(0u, 0u, 0u, 0u);
  }
  if (threadIdx.x < 32) {
    // source segments and their 32-particle work items (warp prefix sums)
    const int k = threadIdx.x;
    uint32_t b = 0, c = 0;
    if (k < NSRC) {
      const int px = pmod(x0 + k / (RY + 1) - 1, m.nx), py = pmod(y0 + k % (RY + 1) - 1, m.ny);
      const int64_t row = (int64_t)px * m.ny + py;
      b = offs[row];
      c = offs[row + 1] - b;
    }
    uint32_t items = (c + 31) >> 5, tot = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, items, o);
      const uint32_t z = __shfl_up_sync(0xFFFFFFFFu, tot, o);
      if (k >= o) {
        items += y;
        tot += z;
      }
    }
    if (k < NSRC) {
      seg_beg[k] = b;
      seg_cnt[k] = c;
      item_pre[k + 1] = items;
    }
    if (k == 0) item_pre[0] = 0;
    if (k == 31) s_ntot = tot;
  }
  __syncthreads();
  const uint32_t ntot = s_ntot;
  const uint32_t nitems = item_pre[NSRC];
  const double scale = *scale_dev;
  int s;
  bool split;
  split_shift(ntot, dup, E, scale, s, split);
  SplitAcc A;
  A.acc = acc;
  A.cells = cells;
  A.y_scale = split ? __fmul_rn((float)scale, __int_as_float((127 - s) << 23)) : 0.f;
  A.two_s = __int_as_float((127 + s) << 23);
  unsigned long long* acc64 = reinterpret_cast<unsigned long long*>(acc);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  const bool zpow2 = (nz & (nz - 1)) == 0;
  int k = 0;
  for (uint32_t it = warp; it < nitems; it += nwarps) {
    while (it >= item_pre[k + 1]) ++k;
    const uint32_t j = ((it - item_pre[k]) << 5) + lane;
    if (j < seg_cnt[k]) {
      const uint32_t i = seg_beg[k] + j;
      const Rec r = rec[i];
      const int cz = zpow2 ? (int)(r.key & (uint32_t)(nz - 1)) : (int)(r.key % (uint32_t)nz);
      float v[C];
      if (val != nullptr) {
        const int64_t src = val_sorted ? (int64_t)i : (int64_t)perm[i];
#pragma unroll
        for (int c = 0; c < C; ++c) v[c] = val[src * C + c];
      } else {
#pragma unroll
        for (int c = 0; c < C; ++c) v[c] = val_const;
      }
      if (split)
        deposit_k<C, RX, RY, true>(k, r, v, nz, cz, A, acc64, scale);
      else
        deposit_k<C, RX, RY, false>(k, r, v, nz, cz, A, acc64, scale);
    }
  }
  __syncthreads();
  split_epilogue<C, RX, RY>(acc, cells, split, s, scale, A.two_s, m, x0, y0, mode, src_mul, out);
}

// One output row per block (1 x 1 tile) with the particle visits of its four
// source rows flattened over the block's threads: consecutive threads take
// consecutive records whatever their source row, so every lane is busy (the
// per-row 32-particle chunks of scatter_split_kernel leave the last chunk of
// each row part-empty).  A particle of source row (x0 - 1 + sx, y0 - 1 + sy)
// reaches the row through its corner (1 - sx, 1 - sy).  Same split planes
// and epilogue, so the output is bit-identical.  Used for three channels,
// where it measured 14-15% faster at 512^3 / 1024^3.
template <int C>
__global__ void __launch_bounds__(256) scatter_flat_kernel(const Rec* __restrict__ rec,
                                                           const uint32_t* __restrict__ perm,
                                                           const uint32_t* __restrict__ offs, Mesh3 m,
                                                           const float* __restrict__ val, int val_sorted,
                                                           float val_const, const double* __restrict__ scale_dev,
                                                           int E, int dup, int mode, float src_mul,
                                                           float* __restrict__ out, uint32_t* __restrict__ status) {
  if (flagged(status)) return;
  if (!(*scale_dev == *scale_dev)) {  // NaN scale: a non-finite value
    if (threadIdx.x == 0) raise_flag(status, kFlagNonFiniteValue);
    return;
  }
  extern __shared__ __align__(16) unsigned int acc[];  // 8 * C * nz bytes
  __shared__ uint32_t s_beg[4], s_pre[5];
  const int x0 = (int)(blockIdx.x / m.ny), y0 = (int)(blockIdx.x % m.ny);
  const int nz = m.nz;
  const int cells = C * nz;
  {
    uint4* a4 = reinterpret_cast<uint4*>(acc);
    const int n4 = (2 * cells) >> 2;
    for (int t = threadIdx.x; t < n4; t += blockDim.x) a4[t] = make_uint4(0u, 0u, 0u, 0u);
  }
  if (threadIdx.x < 32) {
    const int k = threadIdx.x;
    uint32_t b = 0, c = 0;
    if (k < 4) {
      const int px = pmod(x0 - 1 + (k >> 1), m.nx), py = pmod(y0 - 1 + (k & 1), m.ny);
      const int64_t row = (int64_t)px * m.ny + py;
      b = offs[row];
      c = offs[row + 1] - b;
    }
    uint32_t tot = c;
#pragma unroll
    for (int o = 1; o < 4; o <<= 1) {
      const uint32_t z = __shfl_up_sync(0xFFFFFFFFu, tot, o);
      if (k >= o) tot += z;
    }
    if (k < 4) {
      s_beg[k] = b;
      s_pre[k + 1] = tot;
    }
    if (k == 0) s_pre[0] = 0;
  }
  __syncthreads();
  const uint32_t p1 = s_pre[1], p2 = s_pre[2], p3 = s_pre[3], ntot = s_pre[4];
  // record index = visit index + (segment begin - segment prefix), mod 2^32
  const uint32_t d0 = s_beg[0], d1 = s_beg[1] - p1, d2 = s_beg[2] - p2, d3 = s_beg[3] - p3;
  const double scale = *scale_dev;
  int s;
  bool split;
  split_shift(ntot, dup, E, scale, s, split);
  SplitAcc A;
  A.acc = acc;
  A.cells = cells;
  A.y_scale = split ? __fmul_rn((float)scale, __int_as_float((127 - s) << 23)) : 0.f;
  A.two_s = __int_as_float((127 + s) << 23);
  unsigned long long* acc64 = reinterpret_cast<unsigned long long*>(acc);
  const bool zpow2 = (nz & (nz - 1)) == 0;
  for (uint32_t vi = threadIdx.x; vi < ntot; vi += blockDim.x) {
    const int k = (vi >= p1) + (vi >= p2) + (vi >= p3);
    const uint32_t i = vi + (k == 0 ? d0 : k == 1 ? d1 : k == 2 ? d2 : d3);
    const Rec r = rec[i];
    const int cz = zpow2 ? (int)(r.key & (uint32_t)(nz - 1)) : (int)(r.key % (uint32_t)nz);
    const int cz1 = cz + 1 == nz ? 0 : cz + 1;
    float v[C];
    if (val != nullptr) {
      const int64_t src = val_sorted ? (int64_t)i : (int64_t)perm[i];
#pragma unroll
      for (int c = 0; c < C; ++c) v[c] = val[src * C + c];
    } else {
#pragma unroll
      for (int c = 0; c < C; ++c) v[c] = val_const;
    }
    const float wxy = __fmul_rn(axis_weight(r.fx, 1 - (k >> 1)), axis_weight(r.fy, 1 - (k & 1)));
    const float w0 = __fmul_rn(wxy, axis_weight(r.fz, 0)), w1 = __fmul_rn(wxy, axis_weight(r.fz, 1));
#pragma unroll
    for (int c = 0; c < C; ++c) {
      const float c0 = __fmul_rn(v[c], w0), c1 = __fmul_rn(v[c], w1);
      if (split) {
        A.add(c * nz + cz, c0);
        A.add(c * nz + cz1, c1);
      } else {
        atomicAdd(&acc64[c * nz + cz], (unsigned long long)__double2ll_rn((double)c0 * scale));
        atomicAdd(&acc64[c * nz + cz1], (unsigned long long)__double2ll_rn((double)c1 * scale));
      }
    }
  }
  __syncthreads();
  split_epilogue<C, 1, 1>(acc, cells, split, s, scale, A.two_s, m, x0, y0, mode, src_mul, out);
}

// Block shape of the split scatter for C channels, or false when the mesh
// rows cannot take the vector epilogue or the accumulator does not fit.
bool split_block_shape(Mesh3 m, int C, const float* out, int* RX, int* RY) {
  if (m.nz % 4 != 0 || ((uintptr_t)out & 15) != 0) return false;
  const int rx = C == 1 ? 2 : 1, ry = C <= 2 ? 2 : 1;
  if ((int64_t)8 * rx * ry * C * m.nz > 200 * 1024) return false;
  *RX = rx;
  *RY = ry;
  return true;
}

int fixed_point_exponent(int64_t n) {
  int e = 0;
  const double p = fixed_point_pow2(n);
  while (ldexp(1.0, e) < p) ++e;
  return e;
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
                   cudaStream_t s, int64_t n, uint32_t* status) {
  int RX, RY;
  if (n >= 0 && C >= 1 && C <= 4 && split_block_shape(m, C, out, &RX, &RY)) {
    const int E = fixed_point_exponent(n);
    const int dup = (m.nx == 1 ? 2 : 1) * (m.ny == 1 ? 2 : 1) * (m.nz == 1 ? 2 : 1);
    const int64_t smem = (int64_t)8 * RX * RY * C * m.nz;
    const unsigned grid = (unsigned)((int64_t)((m.nx + RX - 1) / RX) * ((m.ny + RY - 1) / RY));
#define PMB_LAUNCH_SPLIT(CC, X, Y)                                                                              \
  do {                                                                                                          \
    PMB_CUDA_CHECK(smem_optin((const void*)scatter_split_kernel<CC, X, Y>, 200 * 1024));                       \
    scatter_split_kernel<CC, X, Y><<<grid, 256, (size_t)smem, s>>>(rec, perm, offs, m, val, val_sorted,         \
                                                                   val_const, scale_dev, E, dup, mode, src_mul, \
                                                                   out, status);                                \
  } while (0)
    switch (C) {
      case 1: PMB_LAUNCH_SPLIT(1, 2, 2); break;
      case 2: PMB_LAUNCH_SPLIT(2, 1, 2); break;
      case 3:
        PMB_CUDA_CHECK(smem_optin((const void*)scatter_flat_kernel<3>, 200 * 1024));
        scatter_flat_kernel<3><<<grid, 256, (size_t)smem, s>>>(rec, perm, offs, m, val, val_sorted, val_const,
                                                               scale_dev, E, dup, mode, src_mul, out, status);
        break;
      default: PMB_LAUNCH_SPLIT(4, 1, 1); break;
    }
#undef PMB_LAUNCH_SPLIT
    PMB_CUDA_CHECK(cudaGetLastError());
    return kOk;
  }
  scatter_block_shape(m, C, &RX, &RY);
  const int64_t smem = ScatterSmem::acc_bytes(RX, RY, C, m.nz);
  if (smem > 200 * 1024) return kUnsupported;
  const int nbx = (m.nx + RX - 1) / RX, nby = (m.ny + RY - 1) / RY;
  const unsigned grid = (unsigned)((int64_t)nbx * nby);
#define PMB_LAUNCH_SCATTER(CC)                                                                                   \
  do {                                                                                                           \
    PMB_CUDA_CHECK(smem_optin((const void*)scatter_pull_kernel<CC>, 200 * 1024));                              \
    scatter_pull_kernel<CC><<<grid, 256, (size_t)smem, s>>>(rec, perm, offs, m, RX, RY, val, val_sorted,         \
                                                             val_const, scale_dev, mode, src_mul, out, status); \
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
                              float kick, float kick2, const uint32_t* __restrict__ status) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || flagged(status)) return;
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

// Poll limit of the first bounded wait of every staged or TMA-fed kernel
// (process-wide, pmb_set_wait_limit).
static uint32_t g_wait_polls = kWaitPolls;

void set_wait_polls(uint32_t polls) { g_wait_polls = polls; }
uint32_t wait_polls() { return g_wait_polls; }

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
                                                int y0, int RX, int RY, uint64_t* bar, uint32_t polls) {
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
  return mbar_wait_or_flag(bar, 0, &g_wait_timeouts_cic, polls);
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
                                                            float kick, float kick2, uint32_t polls,
                                                            const uint32_t* __restrict__ status) {
  extern __shared__ __align__(16) float stage[];
  __shared__ __align__(8) uint64_t bar;
  __shared__ uint32_t seg_b[kStageMaxRX], seg_n[kStageMaxRX];
  if (flagged(status)) return;
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
  if (!stage_mesh_rows(stage, mesh, m, C, x0, y0, RX, RY, &bar, polls)) return;
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
      if (out != nullptr) out[(int64_t)src * C + c] = a;
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
                                                        float kick2, const uint32_t* __restrict__ status) {
  const int64_t i0 = (int64_t)blockIdx.x * (2 * blockDim.x) + threadIdx.x;
  const int64_t i1 = i0 + blockDim.x;
  if (i0 >= n || flagged(status)) return;
  const bool two = i1 < n;
  // masked particles (trailing records) interpolate from cell 0 and write zero
  bool mk0, mk1;
  const Rec r0 = unmasked_or_origin(rec[i0], &mk0);
  const Rec r1 = two ? unmasked_or_origin(rec[i1], &mk1) : r0;
  if (!two) mk1 = mk0;
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
    if (out != nullptr) out[(int64_t)s0 * C + c] = mk0 ? 0.f : a0;
    if (vel != nullptr && !mk0) vel[(int64_t)s0 * C + c] = kicked(u0[c], a0, kick, kick2);
    if (two) {
      if (out != nullptr) out[(int64_t)s1 * C + c] = mk1 ? 0.f : a1;
      if (vel != nullptr && !mk1) vel[(int64_t)s1 * C + c] = kicked(u1[c], a1, kick, kick2);
    }
  }
}

// Records after the last row (masked particles) in the staged kernels, which
// only visit rows: zero gathered values; for the adjoint position terms zero
// (or keep, when accumulating) the cotangent, zero wsum and copy u to
// u_sorted.
__global__ void masked_tail_gather_kernel(const uint32_t* __restrict__ perm, const uint32_t* __restrict__ offs_end,
                                          int64_t n, int C, float* __restrict__ out,
                                          const uint32_t* __restrict__ status) {
  if (flagged(status)) return;
  for (int64_t i = (int64_t)*offs_end + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    for (int c = 0; c < C; ++c)
      if (out != nullptr) out[(int64_t)perm[i] * C + c] = 0.f;
}

__global__ void masked_tail_interp_kernel(const uint32_t* __restrict__ perm, const uint32_t* __restrict__ offs_end,
                                          int64_t n, int C, const float* __restrict__ u, float u_const,
                                          int accumulate, float* __restrict__ disp_cot, float* __restrict__ wsum,
                                          float* __restrict__ u_sorted, const uint32_t* __restrict__ status) {
  if (flagged(status)) return;
  for (int64_t i = (int64_t)*offs_end + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t src = perm[i];
    if (!accumulate) disp_cot[3 * src] = disp_cot[3 * src + 1] = disp_cot[3 * src + 2] = 0.f;
    for (int c = 0; c < C; ++c) {
      if (wsum != nullptr) wsum[src * C + c] = 0.f;
      if (u_sorted != nullptr) u_sorted[i * C + c] = u ? u[src * C + c] : u_const;
    }
  }
}

int gather_sorted(const Rec* rec, const uint32_t* perm, const uint32_t* offs, int64_t n, Mesh3 m, int C,
                  const float* mesh, float* out, float* vel, float kick, float kick2, cudaStream_t s,
                  const uint32_t* status) {
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
                                                              kick, kick2, g_wait_polls, status);               \
  } while (0)
    switch (C) {
      case 1: PMB_LAUNCH_GS(1); break;
      case 2: PMB_LAUNCH_GS(2); break;
      case 3: PMB_LAUNCH_GS(3); break;
      case 4: PMB_LAUNCH_GS(4); break;
      default: return kUnsupported;
    }
#undef PMB_LAUNCH_GS
    masked_tail_gather_kernel<<<148, 256, 0, s>>>(perm, offs + m.rows(), n, C, out, status);
    PMB_CUDA_CHECK(cudaGetLastError());
    return kOk;
  }
  const int th = 256;
  const unsigned g = (unsigned)((n + th - 1) / th);
  if (C == 3) {
    gather_kernel_x2<3><<<(unsigned)((n + 2 * th - 1) / (2 * th)), th, 0, s>>>(rec, perm, n, m, mesh, out, vel, kick,
                                                                              kick2, status);
    PMB_CUDA_CHECK(cudaGetLastError());
    return kOk;
  }
  switch (C) {
    case 1: gather_kernel<1><<<g, th, 0, s>>>(rec, perm, n, m, mesh, out, vel, kick, kick2, status); break;
    case 2: gather_kernel<2><<<g, th, 0, s>>>(rec, perm, n, m, mesh, out, vel, kick, kick2, status); break;
    case 3: gather_kernel<3><<<g, th, 0, s>>>(rec, perm, n, m, mesh, out, vel, kick, kick2, status); break;
    case 4: gather_kernel<4><<<g, th, 0, s>>>(rec, perm, n, m, mesh, out, vel, kick, kick2, status); break;
    default: return kUnsupported;
  }
  PMB_CUDA_CHECK(cudaGetLastError());
  return kOk;
}

// Reads and clears the device-wide flags (the staged gathers' wait counter
// becomes kFlagWaitTimeout).  Synchronous.
int device_flags_take(unsigned int* flags) {
  unsigned int f = 0, w = 0;
  PMB_CUDA_CHECK(cudaMemcpyFromSymbol(&f, g_device_flags, sizeof(unsigned int)));
  PMB_CUDA_CHECK(cudaMemcpyFromSymbol(&w, g_wait_timeouts_cic, sizeof(unsigned int)));
  const unsigned int zero = 0;
  PMB_CUDA_CHECK(cudaMemcpyToSymbol(g_device_flags, &zero, sizeof(unsigned int)));
  PMB_CUDA_CHECK(cudaMemcpyToSymbol(g_wait_timeouts_cic, &zero, sizeof(unsigned int)));
  *flags = f | (w ? (unsigned)kFlagWaitTimeout : 0u);
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
                                                float* __restrict__ u_sorted, const float* dprev = nullptr,
                                                bool masked = false) {
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
  if (masked) {
    // a masked particle takes no adjoint: zero, or unchanged when accumulating
    if (!accumulate) dc[0] = dc[1] = dc[2] = 0.f;
    if (wsum != nullptr) {
#pragma unroll
      for (int c = 0; c < C; ++c) wsum[(int64_t)src * C + c] = 0.f;
    }
    return;
  }
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
                                   float* __restrict__ wsum, float* __restrict__ u_sorted,
                                   const uint32_t* __restrict__ status) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || flagged(status)) return;
  bool mk;
  const Rec r = unmasked_or_origin(rec[i], &mk);
  Corners k;
  corners_of(r, m, k);
  const int64_t cells = m.cells();
  auto fetch = [&](int c, int b) { return __ldg(mesh + (int64_t)c * cells + k.idx[b]); };
  interp_grad_one<C>(r, perm[i], i, fetch, u, u_const, cell, accumulate, disp_cot, wsum, u_sorted, nullptr, mk);
}

// Two particles per thread, as gather_kernel_x2.
template <int C>
__global__ void __launch_bounds__(256) interp_grad_kernel_x2(const Rec* __restrict__ rec,
                                                             const uint32_t* __restrict__ perm, int64_t n, Mesh3 m,
                                                             const float* __restrict__ mesh,
                                                             const float* __restrict__ u, float u_const, float cell,
                                                             int accumulate, float* __restrict__ disp_cot,
                                                             float* __restrict__ wsum, float* __restrict__ u_sorted,
                                                             const uint32_t* __restrict__ status) {
  const int64_t i0 = (int64_t)blockIdx.x * (2 * blockDim.x) + threadIdx.x;
  const int64_t i1 = i0 + blockDim.x;
  if (i0 >= n || flagged(status)) return;
  const bool two = i1 < n;
  bool mk0, mk1;
  const Rec r0 = unmasked_or_origin(rec[i0], &mk0);
  const Rec r1 = two ? unmasked_or_origin(rec[i1], &mk1) : r0;
  if (!two) mk1 = mk0;
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
  interp_grad_one<C>(r0, s0, i0, f0, u, u_const, cell, accumulate, disp_cot, wsum, u_sorted, d0, mk0);
  if (two) {
    auto f1 = [&](int c, int b) { return v1[c][b]; };
    interp_grad_one<C>(r1, s1, i1, f1, u, u_const, cell, accumulate, disp_cot, wsum, u_sorted, d1, mk1);
  }
}

template <int C>
__global__ void __launch_bounds__(256) interp_grad_staged_kernel(
    const Rec* __restrict__ rec, const uint32_t* __restrict__ perm, const uint32_t* __restrict__ offs, Mesh3 m, int RX,
    int RY, uint32_t min_stage, const float* __restrict__ mesh, const float* __restrict__ u, float u_const, float cell,
    int accumulate, float* __restrict__ disp_cot, float* __restrict__ wsum, float* __restrict__ u_sorted,
    uint32_t polls, const uint32_t* __restrict__ status) {
  extern __shared__ __align__(16) float stage[];
  __shared__ __align__(8) uint64_t bar;
  __shared__ uint32_t seg_b[kStageMaxRX], seg_n[kStageMaxRX];
  if (flagged(status)) return;
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
  if (!stage_mesh_rows(stage, mesh, m, C, x0, y0, RX, RY, &bar, polls)) return;
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
                       float* wsum, float* u_sorted, cudaStream_t s, const uint32_t* status) {
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
                                                                   u_sorted, g_wait_polls, status);             \
  } while (0)
    switch (C) {
      case 1: PMB_LAUNCH_IS(1); break;
      case 2: PMB_LAUNCH_IS(2); break;
      case 3: PMB_LAUNCH_IS(3); break;
      case 4: PMB_LAUNCH_IS(4); break;
      default: return kUnsupported;
    }
#undef PMB_LAUNCH_IS
    masked_tail_interp_kernel<<<148, 256, 0, s>>>(perm, offs + m.rows(), n, C, u, u_const, accumulate, disp_cot, wsum,
                                                  u_sorted, status);
    PMB_CUDA_CHECK(cudaGetLastError());
    return kOk;
  }
  const int th = 256;
  const unsigned g = (unsigned)((n + th - 1) / th);
  const unsigned g2 = (unsigned)((n + 2 * th - 1) / (2 * th));
  if (C == 1) {
    interp_grad_kernel_x2<1><<<g2, th, 0, s>>>(rec, perm, n, m, mesh, u, u_const, cell, accumulate, disp_cot, wsum,
                                               u_sorted, status);
    PMB_CUDA_CHECK(cudaGetLastError());
    return kOk;
  }
  if (C == 3) {
    interp_grad_kernel_x2<3><<<g2, th, 0, s>>>(rec, perm, n, m, mesh, u, u_const, cell, accumulate, disp_cot, wsum,
                                               u_sorted, status);
    PMB_CUDA_CHECK(cudaGetLastError());
    return kOk;
  }
  switch (C) {
    case 1: interp_grad_kernel<1><<<g, th, 0, s>>>(rec, perm, n, m, mesh, u, u_const, cell, accumulate, disp_cot, wsum, u_sorted, status); break;
    case 2: interp_grad_kernel<2><<<g, th, 0, s>>>(rec, perm, n, m, mesh, u, u_const, cell, accumulate, disp_cot, wsum, u_sorted, status); break;
    case 3: interp_grad_kernel<3><<<g, th, 0, s>>>(rec, perm, n, m, mesh, u, u_const, cell, accumulate, disp_cot, wsum, u_sorted, status); break;
    case 4: interp_grad_kernel<4><<<g, th, 0, s>>>(rec, perm, n, m, mesh, u, u_const, cell, accumulate, disp_cot, wsum, u_sorted, status); break;
    default: return kUnsupported;
  }
  PMB_CUDA_CHECK(cudaGetLastError());
  return kOk;
}

}  // namespace pmb
