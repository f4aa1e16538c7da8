// Device-side CIC building blocks shared by the single-simulation kernels
// (cic.cu) and the persistent ensemble kernels (ensemble.cu).
//
// Reference semantics: cic/enmesh.py:34-165 (binning and weights),
// cic/scatter.py:315-338 and cic/gather.py:452-472 (deposit / interpolation).
#pragma once

#include "pmb_common.cuh"

namespace pmb {

struct Binned {
  int cx, cy, cz;
  float fx, fy, fz;
};

// Lower CIC corner and fractions of one particle: d = disp / cell in IEEE
// float, corner = pmid + floor(d) (periodic), fraction = d - floor(d).
// A non-finite displacement is binned as zero (the anchor cell) so that every
// index stays in the mesh; the sort flags it (kFlagNonFiniteDisp).
__device__ __forceinline__ float finite_or_zero(float x) { return isfinite(x) ? x : 0.f; }

__device__ __forceinline__ Binned bin_particle(const int16_t* __restrict__ pmid, const float d0, const float d1,
                                               const float d2, int64_t i, Mesh3 m, float cell) {
  Binned b;
  float q0 = finite_or_zero(__fdiv_rn(d0, cell)), q1 = finite_or_zero(__fdiv_rn(d1, cell)),
        q2 = finite_or_zero(__fdiv_rn(d2, cell));
  float l0 = floorf(q0), l1 = floorf(q1), l2 = floorf(q2);
  b.fx = __fsub_rn(q0, l0);
  b.fy = __fsub_rn(q1, l1);
  b.fz = __fsub_rn(q2, l2);
  b.cx = pmod((int)pmid[3 * i + 0] + (int)l0, m.nx);
  b.cy = pmod((int)pmid[3 * i + 1] + (int)l1, m.ny);
  b.cz = pmod((int)pmid[3 * i + 2] + (int)l2, m.nz);
  return b;
}

// Origin of the mesh in the particles' frame, split as whole cells q and a
// remainder r in [0, cell): the reference's common-grid offset path
// (cic/pallas.py:225-238, cic/enmesh.py:128-147) bins (disp - r) / cell from
// the anchor pmid - q.  A zero shift reproduces bin_particle bit for bit
// (d - 0 == d for every float).
struct BinShift {
  int qx, qy, qz;
  float rx, ry, rz;
};

__device__ __forceinline__ Binned bin_particle(const int16_t* __restrict__ pmid, float d0, float d1, float d2,
                                               int64_t i, Mesh3 m, float cell, const BinShift& sh) {
  Binned b;
  const float q0 = finite_or_zero(__fdiv_rn(__fsub_rn(d0, sh.rx), cell)),
              q1 = finite_or_zero(__fdiv_rn(__fsub_rn(d1, sh.ry), cell)),
              q2 = finite_or_zero(__fdiv_rn(__fsub_rn(d2, sh.rz), cell));
  const float l0 = floorf(q0), l1 = floorf(q1), l2 = floorf(q2);
  b.fx = __fsub_rn(q0, l0);
  b.fy = __fsub_rn(q1, l1);
  b.fz = __fsub_rn(q2, l2);
  b.cx = pmod((int)pmid[3 * i + 0] - sh.qx + (int)l0, m.nx);
  b.cy = pmod((int)pmid[3 * i + 1] - sh.qy + (int)l1, m.ny);
  b.cz = pmod((int)pmid[3 * i + 2] - sh.qz + (int)l2, m.nz);
  return b;
}

// Key of the records of particles left out by a validity mask (cic/pallas.py:
// 133-141): they follow the last mesh row, deposit nothing, gather zero and
// take no adjoint.  No cell has this key (meshes hold fewer than 2^32 - 1
// cells).
constexpr uint32_t kMaskedKey = 0xFFFFFFFFu;

// A record that is safe to interpolate from (cell 0) in place of a masked one.
__device__ __forceinline__ Rec unmasked_or_origin(const Rec& r, bool* masked) {
  *masked = r.key == kMaskedKey;
  if (!*masked) return r;
  Rec z;
  z.fx = z.fy = z.fz = 0.f;
  z.key = 0u;
  return z;
}

constexpr int kMaxSrcRows = 25;  // (RX+1)*(RY+1) with RX, RY <= 4

// Shared-memory bookkeeping of one scatter tile.
struct ScatterSmem {
  uint32_t seg_beg[kMaxSrcRows];
  uint32_t seg_pre[kMaxSrcRows + 1];
  // dynamic accumulator bytes of an RX x RY block with C channels
  static constexpr int64_t acc_bytes(int RX, int RY, int C, int nz) { return (int64_t)12 * RX * RY * C * nz; }
};

// One RX x RY block of output rows at (x0, y0) of mesh m: pulls the
// particles of the (RX+1) x (RY+1) source rows that reach the block
// (offs[row] .. offs[row+1] in the sorted records; offs points at this
// mesh's first row), accumulates val * w as 64-bit fixed-point integers
// (units of 1/scale) in shared memory, and writes every output cell once:
// mode 0 the deposit, mode 1 the Poisson source (rho - 1) * src_mul
// (gravity.py:628-630).  val (C values per particle, may be null for the
// constant val_const) is indexed by source particle (perm) or, with
// val_sorted, by sorted position.
//
// Integer sums do not depend on the order in which particles arrive, so the
// result is bit-deterministic.  Accumulator: 12 bytes per output cell-channel
// (ScatterSmem::acc_bytes).  When the block's source segments hold fewer
// than 2^16 particles, each 64-bit contribution q = a*2^32 + b*2^16 + c (a
// signed, 0 <= b, c < 2^16) is added as three 32-bit shared atomics on
// separate planes: the b and c sums stay below 2^32 and the a sum below 2^31,
// so the recombined total is exactly the 64-bit sum, while 32-bit atomics
// tolerate many particles per cell (clustering) far better than 64-bit ones.
// Larger blocks use one 64-bit atomic per contribution on the first 8 bytes
// per cell.  Either way the result is the same exact sum.  Must be called by
// all threads of the block; leaves the block synchronised.
template <int C>
__device__ __forceinline__ void scatter_tile(const Rec* __restrict__ rec, const uint32_t* __restrict__ perm,
                                             const uint32_t* __restrict__ offs, Mesh3 m, int RX, int RY, int x0,
                                             int y0, const float* __restrict__ val, int val_sorted, float val_const,
                                             double scale, int mode, float src_mul, float* __restrict__ out,
                                             unsigned int* acc, ScatterSmem& sm) {
  const int nz = m.nz;
  const int nsrc = (RX + 1) * (RY + 1);
  const int cells = RX * RY * C * nz;
  {
    uint4* a4 = reinterpret_cast<uint4*>(acc);
    const int n4 = (3 * cells) >> 2;
    for (int t = threadIdx.x; t < n4; t += blockDim.x) a4[t] = make_uint4(0u, 0u, 0u, 0u);
    for (int t = 4 * n4 + threadIdx.x; t < 3 * cells; t += blockDim.x) acc[t] = 0u;
  }
  if (threadIdx.x < nsrc) {
    const int k = threadIdx.x;
    const int px = pmod(x0 + k / (RY + 1) - 1, m.nx), py = pmod(y0 + k % (RY + 1) - 1, m.ny);
    const int64_t row = (int64_t)px * m.ny + py;
    const uint32_t b = offs[row];
    sm.seg_beg[k] = b;
    sm.seg_pre[k + 1] = offs[row + 1] - b;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t run = 0;
    for (int k = 0; k < nsrc; ++k) {
      const uint32_t c = sm.seg_pre[k + 1];
      sm.seg_pre[k] = run;
      run += c;
    }
    sm.seg_pre[nsrc] = run;
  }
  __syncthreads();
  const uint32_t ntot = sm.seg_pre[nsrc];
  const bool split = ntot < 65536u;
  unsigned long long* acc64 = reinterpret_cast<unsigned long long*>(acc);
  // the scale is a power of two: contrib * scale is exact in float when the
  // scale itself is a float (always, unless max|val| < 2^-74)
  const bool fscale = scale < 0x1p126;
  const float scalef = fscale ? (float)scale : 0.f;
  int k = 0;  // source segment of idx; idx only grows, so the search resumes
  const bool zpow2 = (nz & (nz - 1)) == 0;
  for (uint32_t idx = threadIdx.x; idx < ntot; idx += blockDim.x) {
    while (idx >= sm.seg_pre[k + 1]) ++k;
    const int sx = k / (RY + 1) - 1, sy = k % (RY + 1) - 1;
    const uint32_t i = sm.seg_beg[k] + (idx - sm.seg_pre[k]);
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
#pragma unroll
    for (int bx = 0; bx < 2; ++bx) {
      const int lx = sx + bx;
      if (lx < 0 || lx >= RX || x0 + lx >= m.nx) continue;
      const float wx = axis_weight(r.fx, bx);
#pragma unroll
      for (int by = 0; by < 2; ++by) {
        const int ly = sy + by;
        if (ly < 0 || ly >= RY || y0 + ly >= m.ny) continue;
        const float wxy = __fmul_rn(wx, axis_weight(r.fy, by));
#pragma unroll
        for (int bz = 0; bz < 2; ++bz) {
          int z = cz + bz;
          if (z >= nz) z -= nz;
          const float w = __fmul_rn(wxy, axis_weight(r.fz, bz));
#pragma unroll
          for (int c = 0; c < C; ++c) {
            const float contrib = __fmul_rn(v[c], w);
            const long long q = fscale ? __float2ll_rn(__fmul_rn(contrib, scalef))
                                       : __double2ll_rn((double)contrib * scale);
            const int a = ((lx * RY + ly) * C + c) * nz + z;
            if (split) {
              atomicAdd(&acc[a], (unsigned int)(q >> 32));
              atomicAdd(&acc[cells + a], (unsigned int)((q >> 16) & 0xFFFF));
              atomicAdd(&acc[2 * cells + a], (unsigned int)(q & 0xFFFF));
            } else {
              atomicAdd(&acc64[a], (unsigned long long)q);
            }
          }
        }
      }
    }
  }
  __syncthreads();
  const double inv = 1.0 / scale;
  const int64_t mcells = m.cells();
  for (int lx = 0; lx < RX; ++lx) {
    if (x0 + lx >= m.nx) break;
    for (int ly = 0; ly < RY; ++ly) {
      if (y0 + ly >= m.ny) break;
      const int64_t row_off = ((int64_t)(x0 + lx) * m.ny + (y0 + ly)) * nz;
#pragma unroll
      for (int c = 0; c < C; ++c) {
        const int a0 = ((lx * RY + ly) * C + c) * nz;
        float* o = out + (int64_t)c * mcells + row_off;
        for (int z = threadIdx.x; z < nz; z += blockDim.x) {
          const int a = a0 + z;
          const long long sum = split ? (long long)(((unsigned long long)acc[a] << 32) +
                                                    ((unsigned long long)acc[cells + a] << 16) +
                                                    (unsigned long long)acc[2 * cells + a])
                                      : (long long)acc64[a];
          float rho = (float)((double)sum * inv);
          if (mode == 1) rho = __fmul_rn(__fsub_rn(rho, 1.0f), src_mul);
          o[z] = rho;
        }
      }
    }
  }
  __syncthreads();
}

struct Corners {
  int64_t idx[8];
  float w[8];
};

// Raveled indices and weights of the eight CIC corners of a sorted record;
// corner c moves +1 along axis a when bit a of c is set.
__device__ __forceinline__ void corners_of(const Rec& r, Mesh3 m, Corners& k) {
  const uint32_t key = r.key;
  int cx, cy, cz;
  if (((m.nz & (m.nz - 1)) | (m.ny & (m.ny - 1))) == 0) {
    // power-of-two rows and planes: shifts instead of divisions
    const int lz = __ffs(m.nz) - 1, ly = __ffs(m.ny) - 1;
    cz = (int)(key & (uint32_t)(m.nz - 1));
    cy = (int)((key >> lz) & (uint32_t)(m.ny - 1));
    cx = (int)(key >> (lz + ly));
  } else {
    cz = (int)(key % (uint32_t)m.nz);
    const uint32_t rowk = key / (uint32_t)m.nz;
    cy = (int)(rowk % (uint32_t)m.ny);
    cx = (int)(rowk / (uint32_t)m.ny);
  }
  // lower corner and the (periodic) steps to the upper one along each axis
  const int64_t plane = (int64_t)m.ny * m.nz;
  const int64_t base = (int64_t)key;  // raveled lower cell, (cx * ny + cy) * nz + cz
  const int64_t dx = cx + 1 == m.nx ? -(int64_t)cx * plane : plane;
  const int64_t dy = cy + 1 == m.ny ? -(int64_t)cy * m.nz : (int64_t)m.nz;
  const int64_t dz = cz + 1 == m.nz ? -(int64_t)cz : 1;
  const float wx[2] = {axis_weight(r.fx, 0), axis_weight(r.fx, 1)};
  const float wy[2] = {axis_weight(r.fy, 0), axis_weight(r.fy, 1)};
  const float wz[2] = {axis_weight(r.fz, 0), axis_weight(r.fz, 1)};
#pragma unroll
  for (int c = 0; c < 8; ++c) {
    const int bx = c & 1, by = (c >> 1) & 1, bz = (c >> 2) & 1;
    k.idx[c] = base + (bx ? dx : 0) + (by ? dy : 0) + (bz ? dz : 0);
    k.w[c] = __fmul_rn(__fmul_rn(wx[bx], wy[by]), wz[bz]);
  }
}

// out[src, c] = sum_b mesh_c[i_b] w_b for one sorted record; with vel the
// half-kick vel += out * kick is applied in place (integrator.py:536).
// vel + a k1 (+ a k2): one or two half-kicks with the same acceleration, in
// order, each with two roundings as the separate update would (k2 == 0: none).
__device__ __forceinline__ float kicked(float v, float a, float k1, float k2) {
  v = __fadd_rn(v, __fmul_rn(a, k1));
  if (k2 != 0.f) v = __fadd_rn(v, __fmul_rn(a, k2));
  return v;
}

template <int C>
__device__ __forceinline__ void gather_one(const Rec& r, uint32_t src, Mesh3 m, const float* __restrict__ mesh,
                                           float* __restrict__ out, float* __restrict__ vel, float kick,
                                           float kick2 = 0.f) {
  if (r.key == kMaskedKey) {
    // masked particle: zero value, velocity untouched (a zero kick)
#pragma unroll
    for (int c = 0; c < C; ++c)
      if (out != nullptr) out[(int64_t)src * C + c] = 0.f;
    return;
  }
  Corners k;
  corners_of(r, m, k);
  // velocities loaded ahead of the corner loads (latency overlapped)
  float u[C];
  if (vel != nullptr) {
#pragma unroll
    for (int c = 0; c < C; ++c) u[c] = vel[(int64_t)src * C + c];
  }
  const int64_t cells = m.cells();
#pragma unroll
  for (int c = 0; c < C; ++c) {
    const float* mc = mesh + (int64_t)c * cells;
    float a = 0.f;
#pragma unroll
    for (int b = 0; b < 8; ++b) a = __fadd_rn(a, __fmul_rn(__ldg(mc + k.idx[b]), k.w[b]));
    if (out != nullptr) out[(int64_t)src * C + c] = a;
    if (vel != nullptr) vel[(int64_t)src * C + c] = kicked(u[c], a, kick, kick2);
  }
}

}  // namespace pmb
