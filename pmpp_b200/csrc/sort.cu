// Stable per-cell particle sort: least-significant-digit radix sort of the
// raveled lower-corner cell key with the source index as payload.  LSD radix
// passes are stable, so equal keys keep source order -- the tie rule of the
// reference's merges (cuda/route_kernels.cu:641-644, 1093-1096).  The key is
// ((x*My + y)*Mz + z) of the CIC lower corner (core/utils.py:292-326 applied to
// the binning of cic/enmesh.py:139-147).
#include "pmb_common.cuh"
#include "pmb_kernels.cuh"
#include "pmb_sort.cuh"

namespace pmb {

namespace {
constexpr int kThreads = 256;
constexpr int kItems = 16;
constexpr int kTile = kThreads * kItems;
constexpr int kRadix = 256;
constexpr int kWarps = kThreads / 32;

__global__ void keys_kernel(const int16_t* __restrict__ pmid, const float* __restrict__ disp, int64_t n, Mesh3 m,
                            float cell, uint32_t* __restrict__ keys, uint32_t* __restrict__ vals) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int c[3];
  const int dims[3] = {m.nx, m.ny, m.nz};
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const float q = __fdiv_rn(disp[3 * i + a], cell);
    c[a] = pmod((int)pmid[3 * i + a] + (int)floorf(q), dims[a]);
  }
  keys[i] = (uint32_t)(((int64_t)c[0] * m.ny + c[1]) * m.nz + c[2]);
  vals[i] = (uint32_t)i;
}

// Per-tile digit histogram, written digit-major: hist[d * ntiles + tile].
__global__ void hist_kernel(const uint32_t* __restrict__ keys, int64_t n, int shift, uint32_t* __restrict__ hist,
                            int64_t ntiles) {
  __shared__ uint32_t h[kRadix];
  for (int t = threadIdx.x; t < kRadix; t += blockDim.x) h[t] = 0;
  __syncthreads();
  const int64_t base = (int64_t)blockIdx.x * kTile;
  for (int j = 0; j < kItems; ++j) {
    const int64_t e = base + (int64_t)j * kThreads + threadIdx.x;
    if (e < n) atomicAdd(&h[(keys[e] >> shift) & 0xFF], 1u);
  }
  __syncthreads();
  for (int t = threadIdx.x; t < kRadix; t += blockDim.x) hist[(int64_t)t * ntiles + blockIdx.x] = h[t];
}

// Stable scatter: elements of a tile are ranked in index order (round j,
// thread t) -> j*256 + t, using warp match for intra-warp ranks and a
// per-round prefix over warps.
__global__ void scatter_kernel(const uint32_t* __restrict__ keys, const uint32_t* __restrict__ vals, int64_t n,
                               int shift, const uint32_t* __restrict__ offs, int64_t ntiles,
                               uint32_t* __restrict__ keys_out, uint32_t* __restrict__ vals_out) {
  __shared__ uint32_t base[kRadix];
  __shared__ uint32_t wcount[kWarps][kRadix];
  for (int t = threadIdx.x; t < kRadix; t += blockDim.x) base[t] = offs[(int64_t)t * ntiles + blockIdx.x];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t tile0 = (int64_t)blockIdx.x * kTile;
  for (int j = 0; j < kItems; ++j) {
    for (int t = threadIdx.x; t < kWarps * kRadix; t += blockDim.x) (&wcount[0][0])[t] = 0;
    __syncthreads();
    const int64_t e = tile0 + (int64_t)j * kThreads + threadIdx.x;
    const bool act = e < n;
    uint32_t k = 0, v = 0, d = 0xFFFFFFFFu;
    if (act) {
      k = keys[e];
      v = vals[e];
      d = (k >> shift) & 0xFF;
    }
    const unsigned live = __ballot_sync(0xFFFFFFFFu, act);
    unsigned peers = 0;
    uint32_t rank = 0;
    if (act) {
      peers = __match_any_sync(live, d);
      rank = __popc(peers & ((1u << lane) - 1u));
      if (lane == __ffs(peers) - 1) wcount[warp][d] = __popc(peers);
    }
    __syncthreads();
    // exclusive prefix over warps for every digit, then advance the base
    for (int t = threadIdx.x; t < kRadix; t += blockDim.x) {
      uint32_t run = base[t];
      for (int w = 0; w < kWarps; ++w) {
        const uint32_t c = wcount[w][t];
        wcount[w][t] = run;
        run += c;
      }
      base[t] = run;
    }
    __syncthreads();
    if (act) {
      const uint32_t dst = wcount[warp][d] + rank;
      keys_out[dst] = k;
      vals_out[dst] = v;
    }
    __syncthreads();
  }
}

}  // namespace

int64_t radix_scratch_bytes(int64_t n) {
  const int64_t ntiles = (n + kTile - 1) / kTile;
  const int64_t len = (int64_t)kRadix * (ntiles > 0 ? ntiles : 1);
  return align_up(4 * n, 256) * 2 + align_up(4 * len, 256) + align_up(4 * scan_tmp_elems(len), 256);
}

int sort_by_cell(const int16_t* pmid, const float* disp, int64_t n, Mesh3 m, float cell, uint32_t* keys_out,
                 uint32_t* perm_out, void* scratch, cudaStream_t s) {
  if (n == 0) return kOk;
  const int64_t ntiles = (n + kTile - 1) / kTile;
  char* p = (char*)scratch;
  uint32_t* k2 = (uint32_t*)p;
  p += align_up(4 * n, 256);
  uint32_t* v2 = (uint32_t*)p;
  p += align_up(4 * n, 256);
  uint32_t* hist = (uint32_t*)p;
  p += align_up(4 * (int64_t)kRadix * ntiles, 256);
  uint32_t* tsum = (uint32_t*)p;
  keys_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(pmid, disp, n, m, cell, keys_out, perm_out);
  // number of 8-bit digits needed for keys < nx*ny*nz
  const uint64_t maxkey = (uint64_t)m.cells() - 1;
  int bits = 0;
  while (bits < 32 && (maxkey >> bits) != 0) ++bits;
  int passes = (bits + 7) / 8;
  if (passes == 0) passes = 1;
  if (passes % 2) ++passes;  // even pass count leaves the result in the output buffers
  uint32_t *ka = keys_out, *va = perm_out, *kb = k2, *vb = v2;
  for (int pass = 0; pass < passes; ++pass) {
    const int shift = 8 * pass;
    if (shift >= 32) {
      // padding pass: a plain copy keeps the ping-pong parity
      PMB_CUDA_CHECK(cudaMemcpyAsync(kb, ka, 4 * n, cudaMemcpyDeviceToDevice, s));
      PMB_CUDA_CHECK(cudaMemcpyAsync(vb, va, 4 * n, cudaMemcpyDeviceToDevice, s));
    } else {
      hist_kernel<<<(unsigned)ntiles, kThreads, 0, s>>>(ka, n, shift, hist, ntiles);
      int st = exclusive_scan_u32(hist, hist, (int64_t)kRadix * ntiles, tsum, s);
      if (st != kOk) return st;
      scatter_kernel<<<(unsigned)ntiles, kThreads, 0, s>>>(ka, va, n, shift, hist, ntiles, kb, vb);
    }
    uint32_t* t = ka;
    ka = kb;
    kb = t;
    t = va;
    va = vb;
    vb = t;
  }
  PMB_CUDA_CHECK(cudaGetLastError());
  return kOk;
}

}  // namespace pmb
