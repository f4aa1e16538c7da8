// Particle-mesh FFT pipeline for power-of-two meshes.
//
// The force and its adjoint need, per evaluation, one real-to-complex 3D
// transform, the Green x gradient multiplier and three complex-to-real
// transforms (the adjoint the transpose of that).  cuFFT runs each 3D
// transform as three passes over the whole mesh plus a separate multiplier
// pass.  Here the passes are hand-written persistent kernels fed by TMA, and
// the multiplier is fused into the x pass, where all three wavenumbers of a
// column are known:
//
//   forward:  z R2C -> y -> [x, K(k) (i c_d), x^-1] -> y^-1 -> z C2R
//   adjoint:  z R2C -> y -> [x, K(k) sum_d (-i c_d), x^-1] -> y^-1 -> z C2R
//
// Linearity keeps the channel count down: c_y and c_z are constant along x,
// so the forward x pass writes only W = x^-1(i c_x phi) and Q = x^-1(phi);
// the inverse y pass makes F_y from i c_y Q and F_z = i c_z y^-1(Q).  The
// adjoint folds the y and z channels into one in its y pass the same way.
// Traffic per evaluation: 18 half-spectrum-sized reads/writes (about 28 for
// separate cuFFT transforms and multiplier).
//
// Half-spectrum layout ("y-blocked"): channel-major, then
//   ((y / BY) * nx + x) * BY + y % BY   rows of P complex values,
// P = nz/2 + 8 (columns nz/2+1 .. P-1 are zero padding), BY = 32.  Blocking
// y keeps the x pass's stride at BY * P * 8 bytes (133 KB at 1024^3) instead
// of a whole (y, kz) plane; with the plain layout the x pass touches a
// different 2 MB page per row and runs at half the bandwidth.
//
// Each column pass (y or x) is a four-step FFT of length L = R1 * R2 over a
// tile of KT = 8 adjacent columns (64-byte rows): the tile arrives in shared
// memory by TMA (a ring of S stages, one tile in flight while another is
// transformed), R1-point DFTs run in registers, twiddles, a transpose through
// shared memory, R2-point DFTs, and the results are stored from registers.
// The z passes work on KR = 16 contiguous rows with a bulk copy per tile; the
// real transform of length nz is a complex transform of length nz/2 plus the
// usual even/odd split.
//
// Semantics follow numpy's rfftn / irfftn (numerics/fft.py): forward
// unnormalised; the inverse is unnormalised (the multiplier's post scale
// carries 1/cells) and, like irfftn, drops the imaginary parts of the kz = 0
// and kz = nz/2 bins after the x and y inverse transforms.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <cmath>
#include <map>
#include <mutex>
#include <type_traits>

#include "pmb_common.cuh"
#include "pmb_kernels.cuh"
#include "pmb_spectral_device.cuh"
#include "pmb_tma.cuh"

namespace pmb {

namespace {

constexpr int KT = 8;   // columns per column tile
constexpr int BY = 32;  // y rows per block of the spectral layout
constexpr int KR = 16;  // rows per z-pass tile

__device__ unsigned int g_fft_timeouts;

// exp(-2 pi i k / 32) for k < 16, the float nearest to cos / sin of k pi / 16
// (k = 4 and 8 are never read: those butterflies are handled exactly).
__device__ __forceinline__ float2 w32(int k) {
  constexpr float re[16] = {1.0f,         0.98078525f,  0.9238795f,   0.8314696f,   0.70710677f,  0.55557024f,
                            0.38268343f,  0.19509032f,  0.0f,         -0.19509032f, -0.38268343f, -0.55557024f,
                            -0.70710677f, -0.8314696f,  -0.9238795f,  -0.98078525f};
  constexpr float im[16] = {-0.0f,        -0.19509032f, -0.38268343f, -0.55557024f, -0.70710677f, -0.8314696f,
                            -0.9238795f,  -0.98078525f, -1.0f,        -0.98078525f, -0.9238795f,  -0.8314696f,
                            -0.70710677f, -0.55557024f, -0.38268343f, -0.19509032f};
  return make_float2(re[k], im[k]);
}

// Twiddle tables W_L^k = exp(-2 pi i k / L) (k < L) of every L = 32 .. 2048,
// table L at offset L - 32, evaluated at compile time into a constant device
// array (no fill at run time, so no first-use ordering between streams).
// Each entry: the quadrant j = floor(4k / L) and the remainder are exact
// integers, the remainder is folded to an angle b in [0, pi/4], and sin b /
// cos b come from their Taylor series in double (13 terms; the first omitted
// term is below 1e-28), then rounded once to float.  Exact zeros carry the
// signs of sinpi / cospi of -2k/L: sine -0, cosine +0.
constexpr int kTwTotal = 2048 * 2 - 32;

struct TwiddleTable {
  float2 v[kTwTotal];
};

struct SinCos {
  double s, c;
};

constexpr SinCos sincos_taylor(double b) {
  const double b2 = b * b;
  double ts = b, s = b, tc = 1.0, c = 1.0;
  for (int k = 1; k <= 12; ++k) {
    ts *= -b2 / ((2.0 * k) * (2.0 * k + 1.0));
    tc *= -b2 / ((2.0 * k - 1.0) * (2.0 * k));
    s += ts;
    c += tc;
  }
  return SinCos{s, c};
}

constexpr float2 twiddle_entry(int k, int L) {
  constexpr double kPi = 3.14159265358979323846264338327950288;
  const int j = (4 * k) / L;
  int r = 4 * k - j * L;  // angle 2 pi k / L = (pi / 2) (j + r / L)
  const bool swap = 2 * r > L;
  if (swap) r = L - r;
  const SinCos t = sincos_taylor(0.5 * kPi * (double)r / (double)L);
  const double sb = swap ? t.c : t.s, cb = swap ? t.s : t.c;
  const double s = j == 0 ? sb : j == 1 ? cb : j == 2 ? -sb : -cb;
  const double c = j == 0 ? cb : j == 1 ? -sb : j == 2 ? -cb : sb;
  return float2{c == 0.0 ? 0.0f : (float)c, s == 0.0 ? -0.0f : (float)-s};
}

constexpr TwiddleTable make_twiddles() {
  TwiddleTable t{};
  int i = 0;
  for (int L = 32; L <= 2048; L *= 2)
    for (int k = 0; k < L; ++k) t.v[i++] = twiddle_entry(k, L);
  return t;
}

__device__ const TwiddleTable g_twiddles = make_twiddles();

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 conjf2(float2 a) { return make_float2(a.x, -a.y); }
// i * c * a
__device__ __forceinline__ float2 i_times(float c, float2 a) { return make_float2(-c * a.y, c * a.x); }

template <int R>
struct Log2 {
  static constexpr int v = 1 + Log2<R / 2>::v;
};
template <>
struct Log2<1> {
  static constexpr int v = 0;
};

__host__ __device__ constexpr int bit_reverse(int i, int bits) {
  int r = 0;
  for (int b = 0; b < bits; ++b) r |= ((i >> b) & 1) << (bits - 1 - b);
  return r;
}

// One radix-2 stage (butterfly span LEN) of an in-register R-point DFT on
// bit-reversed input; the stages recurse at compile time so every index is
// a constant and the array stays in registers.
template <int R, int LEN, bool INV>
__device__ __forceinline__ void dft_stage(float2 (&v)[R]) {
  constexpr int H = LEN / 2;
#pragma unroll
  for (int i = 0; i < R; i += LEN) {
#pragma unroll
    for (int k = 0; k < H; ++k) {
      float2 b = v[i + k + H];
      if (k == 0) {
      } else if (4 * k == LEN) {
        b = INV ? make_float2(-b.y, b.x) : make_float2(b.y, -b.x);
      } else {
        float2 w = w32(k * (32 / LEN));
        if (INV) w.y = -w.y;
        b = cmul(b, w);
      }
      const float2 a = v[i + k];
      v[i + k] = cadd(a, b);
      v[i + k + H] = csub(a, b);
    }
  }
  if constexpr (LEN < R) dft_stage<R, 2 * LEN, INV>(v);
}

// In-register R-point DFT (R <= 32), natural order in and out; INV uses the
// conjugate kernel (no scaling).
template <int R, bool INV>
__device__ __forceinline__ void reg_dft(float2 (&v)[R]) {
  constexpr int LB = Log2<R>::v;
#pragma unroll
  for (int i = 0; i < R; ++i) {
    const int j = bit_reverse(i, LB);
    if (j > i) {
      const float2 t = v[i];
      v[i] = v[j];
      v[j] = t;
    }
  }
  dft_stage<R, 2, INV>(v);
}

// Four-step FFT of length A1*A2 over KT columns, first half: the job (n2, c)
// holds x[A2*n1 + n2], n1 < A1; A1-point DFTs, twiddle W_L^(n2 k1), written
// transposed to buf[k1][n2][c] (rows padded by 8 values against bank conflicts).
template <int A1, int A2, bool INV>
__device__ __forceinline__ void four_step_a(float2 (&v)[A1], float2* buf, int n2, int c, const float2* tw) {
  constexpr int ROW = A2 * KT + 8;
  reg_dft<A1, INV>(v);
#pragma unroll
  for (int k1 = 0; k1 < A1; ++k1) {
    float2 r = v[k1];
    if (k1 != 0) {
      float2 w = tw[n2 * k1];
      if (INV) w.y = -w.y;
      r = cmul(r, w);
    }
    buf[k1 * ROW + n2 * KT + c] = r;
  }
}

// Second half: the job (k1, c) reads buf[k1][.][c] and does the A2-point DFT:
// u[k2] = X[k1 + A1*k2].
template <int A1, int A2, bool INV>
__device__ __forceinline__ void four_step_b(float2 (&u)[A2], const float2* buf, int k1, int c) {
  constexpr int ROW = A2 * KT + 8;
#pragma unroll
  for (int n2 = 0; n2 < A2; ++n2) u[n2] = buf[k1 * ROW + n2 * KT + c];
  reg_dft<A2, INV>(u);
}

template <int R1, int R2>
struct ColGeom {
  static constexpr int L = R1 * R2;
  static constexpr int T = (R1 > R2 ? R1 : R2) * KT;
  static constexpr int TILE = L * KT;
  static constexpr int XA = R1 * (R2 * KT + 8);
  static constexpr int XB = R2 * (R1 * KT + 8);
  static constexpr int BUF0 = TILE > XA ? TILE : XA;
  static constexpr int BUF = BUF0 > XB ? BUF0 : XB;  // float2 per stage
  static constexpr int BOX = L < 256 ? L : 256;      // rows per TMA box
};

// Column pass modes.
enum ColMode : int {
  kYFwd = 0,     // y forward, 1 -> 1
  kYInv = 1,     // y inverse, 1 -> 1
  kYInvYZ = 2,   // y inverse of i c_y Q and i c_z y^-1(Q): 1 -> 2
  kYFwdYZ = 3,   // (-i c_y) y(A_y) + (-i c_z) y(A_z): 2 -> 1
  kXFwd = 4,     // x forward, 1 -> 1
  kXInv = 5,     // x inverse, 1 -> 1
  kXGreen = 6,   // x, K(k), x^-1 of i c_x phi and phi: 1 -> 2
  kXGreenAdj = 7, // x of B_x and b, K(k) ((-i c_x) B_x + b), x^-1: 2 -> 1
  kXFwdAdjK = 8   // x of B_x and b, K(k) ((-i c_x) B_x + b) (no inverse): 2 -> 1
};

__host__ __device__ constexpr bool is_y(int mode) { return mode <= kYFwdYZ; }
__host__ __device__ constexpr int n_in(int mode) {
  return (mode == kYFwdYZ || mode == kXGreenAdj || mode == kXFwdAdjK) ? 2 : 1;
}

// floats of per-axis tables a column pass keeps in shared memory
__host__ __device__ constexpr int col_table_floats(int mode, int L) {
  return (mode == kXGreen || mode == kXGreenAdj || mode == kXFwdAdjK) ? 3 * L
                                                                     : ((mode == kYInvYZ || mode == kYFwdYZ) ? L : 0);
}

struct ColArgs {
  float2* out;
  int64_t ch;      // complex values per channel
  int64_t sb;      // values per y block (nx * BY * P)
  int P;           // row length
  int nx, ny, nz;  // mesh
  int ncolt;       // column tiles per (outer index)
  int nouter;      // x (y pass) or y blocks (x pass)
  int ntiles;      // ncolt * nouter * nbatch
  int ch_off;      // first input channel
  uint32_t polls;  // poll limit of the first wait on a stage (pmb_set_wait_limit)
  const float2* tw;
  SpecTables t;
  GreenParams g;
  // batches of equal-shape meshes with their own tables (ensembles): batch b
  // reads the table array at tab_base + b * tab_stride (null: t for all)
  const float* tab_base;
  int64_t tab_stride;
  int has_masks;
  // output channel of (batch, channel c): oofs + batch * ostride + c * cstride
  int oofs, ostride, cstride;
  // live-spectrum pruning inside a force chain (null: none): the masks of
  // prune_count table arrays at prune_base + b * prune_stride
  const float* prune_base;
  int64_t prune_stride;
  int prune_count;
};

// SpecTables of a table array [kx ky kz cx cy cz (mx my mz)] on the device
__device__ __forceinline__ SpecTables tables_at(const float* tb, int nx, int ny, int nz, int has_masks) {
  const int nzh = nz / 2 + 1;
  SpecTables r;
  r.kx = tb;
  r.ky = r.kx + nx;
  r.kz = r.ky + ny;
  r.cx = r.kz + nzh;
  r.cy = r.cx + nx;
  r.cz = r.cy + ny;
  r.mx = has_masks ? r.cz + nzh : nullptr;
  r.my = has_masks ? r.mx + nx : nullptr;
  r.mz = has_masks ? r.my + ny : nullptr;
  return r;
}

__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int c0, int c1, int c2, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];" ::"r"(smem_u32(dst)),
      "l"(map), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* map, int c0, int c1, int c2, int c3,
                                            uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
      "[%6];" ::"r"(smem_u32(dst)),
      "l"(map), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ bool kz_valid(int kz, int nz) { return kz <= nz / 2; }

// Live part of the spectrum inside a force chain.  The Green multiplier
// carries the particle-Nyquist masks (core/utils.py:15-37): on a mesh finer
// than the particle grid they keep ky in [0, ylo) u [ny - yhi, ny) and
// kz < zl (and the same box in kx), so on a mesh twice as fine 7/8 of the
// half spectrum is zero after it.  The passes on either side of the
// multiplier skip that part: the forward y pass runs only the kz < zs
// columns and stores only live ky rows, the x pass runs only live (ky, kz)
// columns, the inverse y pass runs only kz < zs and reads only live ky rows,
// and the z C2R takes kz >= zs as zeros.  Nothing skipped is ever read, and
// the values it would have carried are exact zeros, so the forward and
// adjoint results are the full chain's (up to the sign of exact zeros).  The
// z passes stay whole-row: they are bound by their transform work, and
// storing or loading only the live columns measured slower at 1024^3.
struct Live {
  int ylo, yhi;  // live ky: [0, ylo) u [ny - yhi, ny)
  int zs;        // kz columns kept: a multiple of KT, at most P
};

// Live extents of the masks of `count` table arrays (base + b * stride),
// their union over the arrays; masks of any other shape (or base null) keep
// the whole spectrum.  Block-wide: every thread calls it, every thread gets
// the result.
__device__ Live live_extents(const float* base, int64_t stride, int count, int nx, int ny, int nz) {
  __shared__ int s_first, s_last, s_fz;
  const int nzh = nz / 2 + 1, P = nz / 2 + 8;
  Live L{ny, 0, P};
  if (base == nullptr) return L;
  int ylo = 0, yhi = 0, zl = 0;
  bool bad = false;
  for (int b = 0; b < count && !bad; ++b) {
    const SpecTables T = tables_at(base + (int64_t)b * stride, nx, ny, nz, 1);
    if (threadIdx.x == 0) {
      s_first = ny;
      s_last = -1;
      s_fz = nzh;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < ny; i += blockDim.x)
      if (T.my[i] == 0.f) {
        atomicMin(&s_first, i);
        atomicMax(&s_last, i);
      }
    for (int i = threadIdx.x; i < nzh; i += blockDim.x)
      if (T.mz[i] == 0.f) atomicMin(&s_fz, i);
    __syncthreads();
    const int first = s_first, last = s_last, fz = s_fz;
    // the dead ky must be one run [first, last], the dead kz a tail [fz, nzh)
    int live_inside = 0;
    for (int i = first + (int)threadIdx.x; i <= last; i += blockDim.x) live_inside |= T.my[i] != 0.f;
    for (int i = fz + (int)threadIdx.x; i < nzh; i += blockDim.x) live_inside |= T.mz[i] != 0.f;
    bad = __syncthreads_or(live_inside) != 0;  // also orders the reads before the next member's reset
    if (last < 0) {
      ylo = ny;  // no dead ky
    } else {
      ylo = max(ylo, first);
      yhi = max(yhi, ny - 1 - last);
    }
    zl = max(zl, fz);
  }
  if (bad) return L;
  if (ylo + yhi < ny) {
    L.ylo = ylo;
    L.yhi = yhi;
  }
  const int zs = (zl + KT - 1) / KT * KT;
  L.zs = zs < P ? zs : P;
  return L;
}

__device__ __forceinline__ bool ky_live(const Live& L, int ky, int ny) { return ky < L.ylo || ky >= ny - L.yhi; }

// Green multiplier of the source value at (ix, iy, iz): phi = K(k) S, K =
// post * mask * T * (-1/k^2), zero at k = 0 (pmb_spectral_device.cuh has the
// reference citations).  kx2 / mx are the x-axis tables in shared memory; the
// column's constants are kyz2 = ky^2 + kz^2 and c0 = -post * my * mz (0 on
// the zero-padding columns); HAS_T: a transfer or radial table is present.
// The quotient uses the fast division (2 ulp), well inside the float32 bar
// of the force parity tests.
template <bool HAS_T>
__device__ __forceinline__ float green_scalar(const ColArgs& a, const float* kx2, const float* mx, float kyz2,
                                              float c0, int ix, int iy, int iz) {
  const float k2 = kx2[ix] + kyz2;
  float K = k2 == 0.f ? 0.f : __fdividef(c0 * mx[ix], k2);
  if constexpr (HAS_T) {
    const Mesh3 m{a.nx, a.ny, a.nz};
    const int64_t j = ((int64_t)ix * a.ny + iy) * (a.nz / 2 + 1) + iz;
    K *= transfer_of(a.g, a.t, j, ix, iy, iz, m);
  }
  return K;
}

// Persistent column pass: a ring of S stages, stage slot i holds input q =
// i % NIN of tile i / NIN of this CTA.
template <int R1, int R2, int S, int MODE, int CTAS, bool PR>
__global__ void __launch_bounds__(ColGeom<R1, R2>::T, CTAS)
    col_pass_kernel(const __grid_constant__ CUtensorMap tin, const ColArgs a) {
  using G = ColGeom<R1, R2>;
  constexpr int L = G::L;
  constexpr int NIN = n_in(MODE);
  constexpr bool YP = is_y(MODE);
  extern __shared__ __align__(128) float2 smem[];
  // [S stages][twiddles W_L^k][axis tables][barriers]
  float2* stw = smem + S * G::BUF;
  float* tab = reinterpret_cast<float*>(stw + L);
  uint64_t* bars = reinterpret_cast<uint64_t*>(tab + col_table_floats(MODE, L));
  const int t = threadIdx.x;
  const int c = t % KT;
  if (t == 0)
    for (int s = 0; s < S; ++s) mbar_init(&bars[s], 1);
  // live part of the spectrum (the whole of it outside a pruned chain):
  // y passes run the column tiles kz < zs; x passes the live (ky, kz tile)
  // columns; the forward y pass stores live ky rows only and the inverse y
  // pass loads them only (PIN / POUT)
  constexpr bool PIN = (MODE == kYInv || MODE == kYInvYZ);
  constexpr bool POUT = (MODE == kYFwd || MODE == kYFwdYZ);
  Live lv{a.ny, 0, a.P};
  if constexpr (PR) lv = live_extents(a.prune_base, a.prune_stride, a.prune_count, a.nx, a.ny, a.nz);
  const int nkt = lv.zs / KT;          // live kz tiles
  const int nly = lv.ylo + lv.yhi;     // live ky
  int ntiles = a.ntiles;
  if constexpr (PR) ntiles = (YP ? nkt * a.nouter : nly * nkt) * (a.ntiles / (a.ncolt * a.nouter));
  const int tiles_mine = ntiles > (int)blockIdx.x ? (ntiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
  const int slots = tiles_mine * NIN;
  // tile -> (column tile, outer, batch)
  auto decode = [&](int tile, int& ct, int& outer, int& batch) {
    if constexpr (!PR) {
      ct = tile % a.ncolt;
      const int r = tile / a.ncolt;
      outer = r % a.nouter;
      batch = r / a.nouter;
    } else if constexpr (YP) {
      ct = tile % nkt;
      const int r = tile / nkt;
      outer = r % a.nouter;
      batch = r / a.nouter;
    } else {
      const int kt = tile % nkt;
      const int r = tile / nkt;
      const int li = r % nly;
      batch = r / nly;
      const int iy = li < lv.ylo ? li : a.ny - nly + li;
      outer = iy / BY;
      ct = (iy % BY) * (a.P / KT) + kt;
    }
  };
  // tables of the current batch (the configuration's for unbatched passes)
  SpecTables T = a.t;
  int tab_batch = 0;
  auto load_tables = [&]() {
    for (int i = t; i < L; i += G::T) {
      if constexpr (MODE == kYInvYZ || MODE == kYFwdYZ) tab[i] = T.cy[i];
      if constexpr (MODE == kXGreen || MODE == kXGreenAdj || MODE == kXFwdAdjK) {
        const float kx = T.kx[i];
        tab[i] = kx * kx;                                  // kx^2
        tab[L + i] = T.cx[i];                              // c_x
        tab[2 * L + i] = T.mx != nullptr ? T.mx[i] : 1.f;  // particle-Nyquist mask
      }
    }
  };
  if (a.tab_base != nullptr && tiles_mine > 0) {
    if constexpr (PR) {
      int ct0, outer0;
      decode((int)blockIdx.x, ct0, outer0, tab_batch);
    } else {
      tab_batch = (int)(blockIdx.x / (a.ncolt * a.nouter));
    }
    T = tables_at(a.tab_base + (int64_t)tab_batch * a.tab_stride, a.nx, a.ny, a.nz, a.has_masks);
  }
  for (int i = t; i < L; i += G::T) stw[i] = a.tw[i];
  load_tables();
  __syncthreads();
  auto out_ch = [&](int batch, int chan) -> int64_t {
    return (int64_t)(a.oofs + batch * a.ostride + chan * a.cstride) * a.ch;
  };
  // TMA boxes (G::BOX rows) holding live ky rows: the pruned inverse y pass
  // loads only these (fewer, larger copies measured faster than one per y block)
  auto box_live = [&](int r0) { return r0 < lv.ylo || r0 + G::BOX > a.ny - lv.yhi; };
  int live_boxes = 0;
  if constexpr (PIN && PR)
    for (int r0 = 0; r0 < L; r0 += G::BOX) live_boxes += box_live(r0);

  auto issue = [&](int i) {
    if (i >= slots) return;
    const int tile = blockIdx.x + (i / NIN) * gridDim.x;
    int ct, outer, batch;
    decode(tile, ct, outer, batch);
    const int ch = a.ch_off + batch * NIN + i % NIN;
    const int s = i % S;
    float2* dst = smem + s * G::BUF;
    const int nyb = a.ny / BY;
    mbar_expect_tx(&bars[s], ((PIN && PR) ? live_boxes * G::BOX : L) * KT * 8);
#pragma unroll 1
    for (int r = 0; r < L; r += G::BOX) {
      if constexpr (PIN && PR)
        if (!box_live(r)) continue;
      if (YP)
        tma_load_4d(dst + r * KT, &tin, ct * KT, r % BY, outer, r / BY + ch * nyb, &bars[s]);
      else
        tma_load_3d(dst + r * KT, &tin, ct * KT, r, outer + ch * nyb, &bars[s]);
    }
  };
  if (t == 0)
    for (int i = 0; i < S; ++i) issue(i);

  // wait for slot i; false (uniformly across the CTA) on a timeout, after
  // draining every slot still in flight (i .. i + S - 1 were issued)
  auto acquire = [&](int i) -> bool {
    const int s = i % S;
    const bool ok = mbar_wait(&bars[s], (i / S) & 1, a.polls);
    if (__syncthreads_or(!ok)) {
      if (t == 0) atomicAdd(&g_fft_timeouts, 1u);
      mbar_drain(bars, S, i, slots);
      return false;
    }
    return true;
  };
  // slot i consumed: hand its stage to the copy engine for slot i + S
  auto release = [&](int i) {
    __syncthreads();
    if (t == 0) {
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      issue(i + S);
    }
  };

  // value of row r of this thread's column in a stage; a pruned inverse y
  // pass reads dead ky rows as zeros (they were never written)
  auto ld = [&](const float2* buf, int r) -> float2 {
    if constexpr (PIN && PR)
      if (!ky_live(lv, r, a.ny)) return make_float2(0.f, 0.f);
    return buf[r * KT + c];
  };
  const bool ja = t < R2 * KT;  // first-half jobs (n2 = t / KT)
  const bool jb = t < R1 * KT;  // second-half jobs (k1 = t / KT)
  const int q = t / KT;

  // forward or inverse transform of the tile in stage slot i; afterwards the
  // job (k1 = q, c) holds u[k2] = X[k1 + R1 k2].  Leaves the stage free to
  // reuse as scratch (not yet released).
  auto transform = [&](int i, float2 (&u)[R2], auto inv_tag) {
    constexpr bool INV = decltype(inv_tag)::value;
    float2* buf = smem + (i % S) * G::BUF;
    float2 v[R1];
    if (ja) {
#pragma unroll
      for (int n1 = 0; n1 < R1; ++n1) v[n1] = ld(buf, R2 * n1 + q);
    }
    __syncthreads();
    if (ja) four_step_a<R1, R2, INV>(v, buf, q, c, stw);
    __syncthreads();
    if (jb) four_step_b<R1, R2, INV>(u, buf, q, c);
  };

  // inverse transform of values held as u[k2] at index k1 + R1 k2 (k1 = q),
  // decomposition (R2, R1); result w[k2'] at index k1' + R2 k2' (k1' = q).
  auto inverse_held = [&](float2* buf, float2 (&u)[R2], float2 (&w)[R1]) {
    __syncthreads();
    if (jb) four_step_a<R2, R1, true>(u, buf, q, c, stw);
    __syncthreads();
    if (ja) four_step_b<R2, R1, true>(w, buf, q, c);
  };

  for (int it = 0; it < tiles_mine; ++it) {
    const int tile = blockIdx.x + it * gridDim.x;
    int ct, outer, batch;
    decode(tile, ct, outer, batch);
    if (a.tab_base != nullptr && batch != tab_batch) {
      // a new batch: its own tables (the previous tile released its stage
      // with a barrier, so no thread still reads them)
      __syncthreads();
      tab_batch = batch;
      T = tables_at(a.tab_base + (int64_t)batch * a.tab_stride, a.nx, a.ny, a.nz, a.has_masks);
      load_tables();
      __syncthreads();
    }
    const int i0 = it * NIN;
    float2 u[R2];
    if (!acquire(i0)) return;
    if constexpr (MODE == kYFwd || MODE == kYInv || MODE == kXFwd || MODE == kXInv) {
      constexpr bool INV = (MODE == kYInv || MODE == kXInv);
      transform(i0, u, std::integral_constant<bool, INV>{});
      const int64_t ob = out_ch(batch, 0);
      if (jb) {
#pragma unroll
        for (int k2 = 0; k2 < R2; ++k2) {
          const int r = q + R1 * k2;
          if constexpr (POUT && PR)
            if (!ky_live(lv, r, a.ny)) continue;
          int64_t off;
          if (YP)
            off = ob + (int64_t)(r / BY) * a.sb + ((int64_t)outer * BY + r % BY) * a.P + ct * KT + c;
          else
            off = ob + (int64_t)outer * a.sb + (int64_t)r * BY * a.P + ct * KT + c;
          a.out[off] = u[k2];
        }
      }
      release(i0);
    } else if constexpr (MODE == kYFwdYZ) {
      if constexpr (R1 == R2) {
        // one forward four-step call site run once per input (code stays small)
        const int kz = ct * KT + c;
        const bool kv = kz_valid(kz, a.nz);
        const float cz = kv ? T.cz[kz] : 0.f;
        float2 acc[R2];
#pragma unroll 1
        for (int ph = 0; ph < 2; ++ph) {
          if (ph == 1) {
            release(i0);
            if (!acquire(i0 + 1)) return;
          }
          float2* buf = smem + ((i0 + ph) % S) * G::BUF;
          float2 v[R1];
#pragma unroll
          for (int n1 = 0; n1 < R1; ++n1) v[n1] = buf[(R2 * n1 + q) * KT + c];
          __syncthreads();
          four_step_a<R1, R2, false>(v, buf, q, c, stw);
          __syncthreads();
          four_step_b<R1, R2, false>(u, buf, q, c);
          if (ph == 0) {
#pragma unroll
            for (int k2 = 0; k2 < R2; ++k2) acc[k2] = i_times(-tab[q + R1 * k2], u[k2]);
          } else {
#pragma unroll
            for (int k2 = 0; k2 < R2; ++k2) {
              const float2 r = kv ? cadd(acc[k2], i_times(-cz, u[k2])) : make_float2(0.f, 0.f);
              const int ky = q + R1 * k2;
              if constexpr (PR)
                if (!ky_live(lv, ky, a.ny)) continue;
              a.out[(int64_t)(ky / BY) * a.sb + ((int64_t)outer * BY + ky % BY) * a.P + kz] = r;
            }
          }
        }
        release(i0 + 1);
      } else {
        // acc = (-i c_y(ky)) y(A_y) + (-i c_z(kz)) y(A_z); rows are ky
        const int kz = ct * KT + c;
        const bool kv = kz_valid(kz, a.nz);
        const float cz = kv ? T.cz[kz] : 0.f;
        float2 acc[R2];
        transform(i0, u, std::false_type{});
        if (jb) {
  #pragma unroll
          for (int k2 = 0; k2 < R2; ++k2) acc[k2] = i_times(-tab[q + R1 * k2], u[k2]);
        }
        release(i0);
        if (!acquire(i0 + 1)) return;
        transform(i0 + 1, u, std::false_type{});
        if (jb) {
  #pragma unroll
          for (int k2 = 0; k2 < R2; ++k2) {
            const float2 z = i_times(-cz, u[k2]);
            const float2 r = kv ? cadd(acc[k2], z) : make_float2(0.f, 0.f);
            const int ky = q + R1 * k2;
            if constexpr (PR)
              if (!ky_live(lv, ky, a.ny)) continue;
            a.out[(int64_t)(ky / BY) * a.sb + ((int64_t)outer * BY + ky % BY) * a.P + kz] = r;
          }
        }
        release(i0 + 1);
      }
    } else if constexpr (MODE == kYInvYZ) {
      if constexpr (R1 == R2) {
        // inverses as conj(FFT(conj(.))): one forward four-step call site
        float2* buf = smem + (i0 % S) * G::BUF;
        const int kz = ct * KT + c;
        const bool kv = kz_valid(kz, a.nz);
        const float cz = kv ? T.cz[kz] : 0.f;
        float2 keep[R1];
#pragma unroll 1
        for (int ph = 0; ph < 2; ++ph) {
          float2 v[R1];
#pragma unroll
          for (int n1 = 0; n1 < R1; ++n1) {
            if (ph == 0) {
              keep[n1] = ld(buf, R2 * n1 + q);
              v[n1] = conjf2(i_times(tab[R2 * n1 + q], keep[n1]));
            } else {
              v[n1] = conjf2(keep[n1]);
            }
          }
          __syncthreads();
          four_step_a<R1, R2, false>(v, buf, q, c, stw);
          __syncthreads();
          four_step_b<R1, R2, false>(u, buf, q, c);
#pragma unroll
          for (int k2 = 0; k2 < R2; ++k2) {
            const int y = q + R1 * k2;
            const float2 r = conjf2(u[k2]);
            const float2 val = ph == 0 ? (kv ? r : make_float2(0.f, 0.f)) : i_times(cz, r);
            a.out[out_ch(batch, ph) + (int64_t)(y / BY) * a.sb + ((int64_t)outer * BY + y % BY) * a.P + kz] = val;
          }
        }
        release(i0);
      } else {
        // F_y = y^-1(i c_y(ky) Q), F_z = i c_z(kz) y^-1(Q); load rows are ky
        float2* buf = smem + (i0 % S) * G::BUF;
        const int kz = ct * KT + c;
        const bool kv = kz_valid(kz, a.nz);
        const float cz = kv ? T.cz[kz] : 0.f;
        float2 v[R1], vy[R1];
        if (ja) {
  #pragma unroll
          for (int n1 = 0; n1 < R1; ++n1) {
            v[n1] = ld(buf, R2 * n1 + q);
            vy[n1] = i_times(tab[R2 * n1 + q], v[n1]);
          }
        }
        __syncthreads();
        if (ja) four_step_a<R1, R2, true>(vy, buf, q, c, stw);
        __syncthreads();
        auto store = [&](int chan, int k2, float2 val) {
          const int y = q + R1 * k2;
          a.out[out_ch(batch, chan) + (int64_t)(y / BY) * a.sb + ((int64_t)outer * BY + y % BY) * a.P + kz] = val;
        };
        if (jb) {
          four_step_b<R1, R2, true>(u, buf, q, c);
  #pragma unroll
          for (int k2 = 0; k2 < R2; ++k2) store(0, k2, kv ? u[k2] : make_float2(0.f, 0.f));
        }
        __syncthreads();
        if (ja) four_step_a<R1, R2, true>(v, buf, q, c, stw);
        __syncthreads();
        if (jb) {
          four_step_b<R1, R2, true>(u, buf, q, c);
  #pragma unroll
          for (int k2 = 0; k2 < R2; ++k2) store(1, k2, i_times(cz, u[k2]));
        }
        release(i0);
      }
    } else if constexpr (MODE == kXGreen) {
      // column j = yi * P + kz of y block `outer`; rows are kx after the transform
      const int j = ct * KT + c;
      const int yi = j / a.P, kz = j - yi * a.P;
      const int iy = outer * BY + yi;
      const bool kv = kz_valid(kz, a.nz);
      float kyz2 = 0.f, c0 = 0.f;
      if (kv) {
        kyz2 = T.ky[iy] * T.ky[iy] + T.kz[kz] * T.kz[kz];
        c0 = -a.g.post_scale * (T.mx != nullptr ? T.my[iy] * T.mz[kz] : 1.f);
      }
      // the transfer tables cover kz <= nz/2 only: never read on padding columns
      const bool has_t = kv && (a.g.transfer != nullptr || a.g.radial != nullptr);
      float2* buf = smem + (i0 % S) * G::BUF;
      transform(i0, u, std::false_type{});
      float2 w[R2];
      auto multiply = [&](auto ht) {
#pragma unroll
        for (int k2 = 0; k2 < R2; ++k2) {
          const int kx = q + R1 * k2;
          const float K = green_scalar<decltype(ht)::value>(a, tab, tab + 2 * L, kyz2, c0, kx, iy, kz);
          u[k2] = make_float2(K * u[k2].x, K * u[k2].y);  // phi
          w[k2] = i_times(tab[L + kx], u[k2]);
        }
      };
      if (jb) {
        if (has_t)
          multiply(std::true_type{});
        else
          multiply(std::false_type{});
      }
      float2 o[R1];
      auto store = [&](int chan, float2 (&val)[R1]) {
        if (ja) {
#pragma unroll
          for (int k2 = 0; k2 < R1; ++k2) {
            const int x = q + R2 * k2;
            a.out[out_ch(batch, chan) + (int64_t)outer * a.sb + (int64_t)x * BY * a.P + j] = val[k2];
          }
        }
      };
      inverse_held(buf, w, o);
      store(0, o);
      inverse_held(buf, u, o);
      store(1, o);
      release(i0);
    } else if constexpr (MODE == kXGreenAdj) {
      const int j = ct * KT + c;
      const int yi = j / a.P, kz = j - yi * a.P;
      const int iy = outer * BY + yi;
      const bool kv = kz_valid(kz, a.nz);
      float kyz2 = 0.f, c0 = 0.f;
      if (kv) {
        kyz2 = T.ky[iy] * T.ky[iy] + T.kz[kz] * T.kz[kz];
        c0 = -a.g.post_scale * (T.mx != nullptr ? T.my[iy] * T.mz[kz] : 1.f);
      }
      // the transfer tables cover kz <= nz/2 only: never read on padding columns
      const bool has_t = kv && (a.g.transfer != nullptr || a.g.radial != nullptr);
      float2 acc[R2];
      transform(i0, u, std::false_type{});
      if (jb) {
#pragma unroll
        for (int k2 = 0; k2 < R2; ++k2) acc[k2] = i_times(-tab[L + q + R1 * k2], u[k2]);
      }
      release(i0);
      if (!acquire(i0 + 1)) return;
      float2* buf = smem + ((i0 + 1) % S) * G::BUF;
      transform(i0 + 1, u, std::false_type{});
      auto multiply = [&](auto ht) {
#pragma unroll
        for (int k2 = 0; k2 < R2; ++k2) {
          const int kx = q + R1 * k2;
          const float K = green_scalar<decltype(ht)::value>(a, tab, tab + 2 * L, kyz2, c0, kx, iy, kz);
          const float2 s = cadd(acc[k2], u[k2]);
          acc[k2] = make_float2(K * s.x, K * s.y);
        }
      };
      if (jb) {
        if (has_t)
          multiply(std::true_type{});
        else
          multiply(std::false_type{});
      }
      float2 o[R1];
      inverse_held(buf, acc, o);
      if (ja) {
#pragma unroll
        for (int k2 = 0; k2 < R1; ++k2) {
          const int x = q + R2 * k2;
          a.out[(int64_t)outer * a.sb + (int64_t)x * BY * a.P + j] = o[k2];
        }
      }
      release(i0 + 1);
    } else if constexpr (MODE == kXFwdAdjK) {
      // s = K(k) ((-i c_x) x(B_x) + x(b)); rows are kx
      const int j = ct * KT + c;
      const int yi = j / a.P, kz = j - yi * a.P;
      const int iy = outer * BY + yi;
      const bool kv = kz_valid(kz, a.nz);
      float kyz2 = 0.f, c0 = 0.f;
      if (kv) {
        kyz2 = T.ky[iy] * T.ky[iy] + T.kz[kz] * T.kz[kz];
        c0 = -a.g.post_scale * (T.mx != nullptr ? T.my[iy] * T.mz[kz] : 1.f);
      }
      // the transfer tables cover kz <= nz/2 only: never read on padding columns
      const bool has_t = kv && (a.g.transfer != nullptr || a.g.radial != nullptr);
      float2 acc[R2];
#pragma unroll 1
      for (int ph = 0; ph < 2; ++ph) {
        if (ph == 1) {
          release(i0);
          if (!acquire(i0 + 1)) return;
        }
        if constexpr (R1 == R2) {
          // square transform: every thread runs both halves, no job guards
          float2* buf = smem + ((i0 + ph) % S) * G::BUF;
          float2 v[R1];
#pragma unroll
          for (int n1 = 0; n1 < R1; ++n1) v[n1] = buf[(R2 * n1 + q) * KT + c];
          __syncthreads();
          four_step_a<R1, R2, false>(v, buf, q, c, stw);
          __syncthreads();
          four_step_b<R1, R2, false>(u, buf, q, c);
        } else {
          transform(i0 + ph, u, std::false_type{});
        }
        if (jb) {
          if (ph == 0) {
#pragma unroll
            for (int k2 = 0; k2 < R2; ++k2) acc[k2] = i_times(-tab[L + q + R1 * k2], u[k2]);
          } else {
            float2* orow = a.out + (int64_t)outer * a.sb + j;
            const int64_t rs = (int64_t)BY * a.P;
            auto multiply = [&](auto ht) {
#pragma unroll
              for (int k2 = 0; k2 < R2; ++k2) {
                const int kx = q + R1 * k2;
                const float K = green_scalar<decltype(ht)::value>(a, tab, tab + 2 * L, kyz2, c0, kx, iy, kz);
                const float2 sum = cadd(acc[k2], u[k2]);
                orow[kx * rs] = make_float2(K * sum.x, K * sum.y);
              }
            };
            if (has_t)
              multiply(std::true_type{});
            else
              multiply(std::false_type{});
          }
        }
      }
      release(i0 + 1);
    }
  }
}

// ---------------------------------------------------------------------------
// z passes (contiguous rows)
// ---------------------------------------------------------------------------
template <int R1, int R2>
struct ZGeom {
  static constexpr int M = R1 * R2;  // complex length = nz / 2
  static constexpr int P = M + 8;    // spectral row length
  static constexpr int T = 256;
  static constexpr int ROWZ = R2 + 1;
  static constexpr int XP = KR * R1 * ROWZ;  // transpose buffer (float2)
  static constexpr int TW = M + M + 8;       // W_M^k (k < M), W_N^k (k <= M), padded
};

struct ZArgs {
  const float* in_r;   // z R2C input (real rows)
  const float2* in_c;  // z C2R input (spectral rows)
  float* out_r;
  float2* out_c;
  int64_t ch;      // complex values per spectral channel
  int64_t cells;   // reals per real channel
  int64_t sb;      // nx * BY * P
  int nx, ny, nz;
  int tiles_per_ch, ntiles;
  uint32_t polls;      // poll limit of the first wait on a stage (pmb_set_wait_limit)
  const float2* tw_m;  // W_M^k, k < M
  const float2* tw_n;  // W_nz^k, k < nz
  // live-spectrum pruning inside a force chain (ColArgs): the C2R takes the
  // columns kz >= zs of each row as zeros
  const float* prune_base;
  int64_t prune_stride;
  int prune_count;
};

// spectral row offset of mesh row (x, y)
template <int P>
__device__ __forceinline__ int64_t spec_row(const ZArgs& a, int x, int y) {
  return (int64_t)(y / BY) * a.sb + ((int64_t)x * BY + y % BY) * P;
}

// twiddles of the z passes into shared memory: W_M^k then W_N^k (k <= M)
template <int M>
__device__ __forceinline__ void load_z_twiddles(const ZArgs& a, float2* tw) {
  for (int i = threadIdx.x; i < M; i += blockDim.x) tw[i] = a.tw_m[i];
  for (int i = threadIdx.x; i <= M; i += blockDim.x) tw[M + i] = a.tw_n[i];
}

// Real-to-complex along z: KR rows of nz reals -> KR rows of P complex.
template <int R1, int R2, int S>
__global__ void __launch_bounds__(256, 1) z_r2c_kernel(const ZArgs a) {
  using G = ZGeom<R1, R2>;
  constexpr int M = G::M, P = G::P;
  constexpr int STAGE = KR * M;  // float2
  extern __shared__ __align__(128) float2 smem[];
  float2* xp = smem + S * STAGE;
  float2* tw = xp + G::XP;
  uint64_t* bars = reinterpret_cast<uint64_t*>(tw + G::TW);
  const int t = threadIdx.x;
  const int tiles_mine = a.ntiles > (int)blockIdx.x ? (a.ntiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
  if (t == 0)
    for (int s = 0; s < S; ++s) mbar_init(&bars[s], 1);
  load_z_twiddles<M>(a, tw);
  __syncthreads();
  auto issue = [&](int i) {
    if (i >= tiles_mine) return;
    const int tile = blockIdx.x + i * gridDim.x;
    const int ch = tile / a.tiles_per_ch;
    const int64_t row0 = (int64_t)(tile % a.tiles_per_ch) * KR;
    const int s = i % S;
    mbar_expect_tx(&bars[s], KR * M * 8);
    bulk_copy_g2s(smem + s * STAGE, a.in_r + ch * a.cells + row0 * a.nz, KR * M * 8, &bars[s]);
  };
  if (t == 0)
    for (int i = 0; i < S; ++i) issue(i);
  for (int it = 0; it < tiles_mine; ++it) {
    const int s = it % S;
    const bool ok = mbar_wait(&bars[s], (it / S) & 1, a.polls);
    if (__syncthreads_or(!ok)) {
      if (t == 0) atomicAdd(&g_fft_timeouts, 1u);
      mbar_drain(bars, S, it, tiles_mine);
      return;
    }
    float2* st = smem + s * STAGE;
    const int tile = blockIdx.x + it * gridDim.x;
    const int ch = tile / a.tiles_per_ch;
    const int row0 = (tile % a.tiles_per_ch) * KR;
    // first half: job (n2, rho)
#pragma unroll 1
    for (int jbq = t; jbq < KR * R2; jbq += G::T) {
      const int n2 = jbq % R2, rho = jbq / R2;
      float2 v[R1];
#pragma unroll
      for (int n1 = 0; n1 < R1; ++n1) v[n1] = st[rho * M + R2 * n1 + n2];
      reg_dft<R1, false>(v);
#pragma unroll
      for (int k1 = 0; k1 < R1; ++k1) {
        float2 r = v[k1];
        if (k1 != 0) r = cmul(r, tw[n2 * k1]);
        xp[(rho * R1 + k1) * G::ROWZ + n2] = r;
      }
    }
    __syncthreads();
    if (t == 0) {  // the stage is consumed: start the copy of tile it + S
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      issue(it + S);
    }
    // second half: job (k1, rho) holds Z[k1 + R1 k2]; the even/odd split
    // X[k] = E[k] + W_N^k O[k] needs Z[M - k], held by the lane of job
    // ((R1 - k1) mod R1, rho) of the same warp (jobs run k1 fastest).
    const int x = row0 / a.ny, y0 = row0 % a.ny;
    float2* orow = a.out_c + ch * a.ch + spec_row<P>(a, x, y0);
    const int lane = t & 31;
    const int src = (lane & ~(R1 - 1)) | ((R1 - (lane & (R1 - 1))) & (R1 - 1));
#pragma unroll 1
    for (int jbq = t; jbq < KR * R1; jbq += G::T) {
      const int k1 = jbq % R1, rho = jbq / R1;
      float2 u[R2];
#pragma unroll
      for (int n2 = 0; n2 < R2; ++n2) u[n2] = xp[(rho * R1 + k1) * G::ROWZ + n2];
      reg_dft<R2, false>(u);
      float2* orr = orow + (int64_t)rho * P;
#pragma unroll
      for (int k2 = 0; k2 < R2; ++k2) {
        // partner value: Z[M - k] = Z[(R1 - k1) + R1 (R2 - 1 - k2)] for k1 > 0;
        // for k1 = 0 it is this lane's own Z[R1 ((R2 - k2) mod R2)]
        const float2 send = u[R2 - 1 - k2];
        float2 zm;
        zm.x = __shfl_sync(0xffffffffu, send.x, src);
        zm.y = __shfl_sync(0xffffffffu, send.y, src);
        if (k1 == 0) zm = u[(R2 - k2) % R2];
        zm = conjf2(zm);
        const float2 zk = u[k2];
        const float2 e = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y + zm.y));
        const float2 d = make_float2(0.5f * (zk.x - zm.x), 0.5f * (zk.y - zm.y));
        const float2 o = make_float2(d.y, -d.x);  // -i d
        const int k = k1 + R1 * k2;
        orr[k] = cadd(e, cmul(tw[M + k], o));
      }
      // X[M] = Re Z[0] - Im Z[0]; zero padding after it
      if (k1 < 8) orr[M + k1] = k1 == 0 ? make_float2(u[0].x - u[0].y, 0.f) : make_float2(0.f, 0.f);
    }
    __syncthreads();  // transpose buffer free
  }
}

// Complex-to-real along z: KR rows of P complex -> KR rows of nz reals.
template <int R1, int R2, int S, bool PR>
__global__ void __launch_bounds__(256, 1) z_c2r_kernel(const ZArgs a) {
  using G = ZGeom<R1, R2>;
  constexpr int M = G::M, P = G::P;
  constexpr int STAGE = KR * P;  // float2
  extern __shared__ __align__(128) float2 smem[];
  float2* xp = smem + S * STAGE;
  float2* tw = xp + G::XP;
  uint64_t* bars = reinterpret_cast<uint64_t*>(tw + G::TW);
  const int t = threadIdx.x;
  const int tiles_mine = a.ntiles > (int)blockIdx.x ? (a.ntiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
  if (t == 0)
    for (int s = 0; s < S; ++s) mbar_init(&bars[s], 1);
  load_z_twiddles<M>(a, tw);
  int zs = P;
  if constexpr (PR) zs = live_extents(a.prune_base, a.prune_stride, a.prune_count, a.nx, a.ny, a.nz).zs;
  __syncthreads();
  auto issue = [&](int i) {
    if (i >= tiles_mine) return;
    const int tile = blockIdx.x + i * gridDim.x;
    const int ch = tile / a.tiles_per_ch;
    const int row0 = (tile % a.tiles_per_ch) * KR;
    const int s = i % S;
    const int x = row0 / a.ny, y0 = row0 % a.ny;
    mbar_expect_tx(&bars[s], KR * P * 8);
    bulk_copy_g2s(smem + s * STAGE, a.in_c + ch * a.ch + spec_row<P>(a, x, y0), KR * P * 8, &bars[s]);
  };
  if (t == 0)
    for (int i = 0; i < S; ++i) issue(i);
  for (int it = 0; it < tiles_mine; ++it) {
    const int s = it % S;
    const bool ok = mbar_wait(&bars[s], (it / S) & 1, a.polls);
    if (__syncthreads_or(!ok)) {
      if (t == 0) atomicAdd(&g_fft_timeouts, 1u);
      mbar_drain(bars, S, it, tiles_mine);
      return;
    }
    const float2* st = smem + s * STAGE;
    const int tile = blockIdx.x + it * gridDim.x;
    const int ch = tile / a.tiles_per_ch;
    const int64_t row0 = (int64_t)(tile % a.tiles_per_ch) * KR;
    // first half with the even/odd merge:
    // Z[k] = (X[k] + conj X[M-k]) + i conj(W_N^k) (X[k] - conj X[M-k])
#pragma unroll 1
    for (int jbq = t; jbq < KR * R2; jbq += G::T) {
      const int n2 = jbq % R2, rho = jbq / R2;
      float2 v[R1];
#pragma unroll
      for (int n1 = 0; n1 < R1; ++n1) {
        const int k = R2 * n1 + n2;
        float2 xk = k < zs ? st[rho * P + k] : make_float2(0.f, 0.f);
        float2 xm = M - k < zs ? st[rho * P + M - k] : make_float2(0.f, 0.f);
        if (k == 0) {
          xk.y = 0.f;
          xm.y = 0.f;
        }
        xm = conjf2(xm);
        const float2 e = cadd(xk, xm);
        const float2 d = cmul(csub(xk, xm), conjf2(tw[M + k]));
        v[n1] = make_float2(e.x - d.y, e.y + d.x);  // e + i d
      }
      reg_dft<R1, true>(v);
#pragma unroll
      for (int k1 = 0; k1 < R1; ++k1) {
        float2 r = v[k1];
        if (k1 != 0) r = cmul(r, conjf2(tw[n2 * k1]));
        xp[(rho * R1 + k1) * G::ROWZ + n2] = r;
      }
    }
    __syncthreads();
    if (t == 0) {  // the stage is consumed: start the copy of tile it + S
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      issue(it + S);
    }
    float2* orow = reinterpret_cast<float2*>(a.out_r + ch * a.cells + row0 * a.nz);
#pragma unroll 1
    for (int jbq = t; jbq < KR * R1; jbq += G::T) {
      const int k1 = jbq % R1, rho = jbq / R1;
      float2 u[R2];
#pragma unroll
      for (int n2 = 0; n2 < R2; ++n2) u[n2] = xp[(rho * R1 + k1) * G::ROWZ + n2];
      reg_dft<R2, true>(u);
#pragma unroll
      for (int k2 = 0; k2 < R2; ++k2) orow[(int64_t)rho * M + k1 + R1 * k2] = u[k2];
    }
    __syncthreads();  // transpose buffer free
  }
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
bool pow2_in(int v, int lo, int hi) { return v >= lo && v <= hi && (v & (v - 1)) == 0; }

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    cudaDriverEntryPointQueryResult q;
    void* p = nullptr;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  return fn;
}

// Pointer to the twiddle table of length L on the current device.
struct TwiddleState {
  std::mutex mu;
  std::map<int, const float2*> base;  // device -> g_twiddles
};
TwiddleState& twiddles() {
  static TwiddleState* t = new TwiddleState();
  return *t;
}

int twiddle_table(int L, const float2** out) {
  if (L < 32 || L > 2048 || (L & (L - 1)) != 0) {
    set_last_error("pmfft: unsupported twiddle table length");
    return kUnsupported;
  }
  int dev = 0;
  PMB_CUDA_CHECK(cudaGetDevice(&dev));
  TwiddleState& t = twiddles();
  std::lock_guard<std::mutex> lock(t.mu);
  auto it = t.base.find(dev);
  if (it == t.base.end()) {
    void* p = nullptr;
    PMB_CUDA_CHECK(cudaGetSymbolAddress(&p, g_twiddles));
    it = t.base.emplace(dev, reinterpret_cast<const float2*>(p)).first;
  }
  *out = it->second + (L - 32);
  return kOk;
}

int sm_count() {
  int dev = 0, n = 148;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
  return n;
}

template <typename K>
int persistent_grid(K kernel, int threads, int smem, int ntiles) {
  int per_sm = 1;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem) != cudaSuccess || per_sm < 1)
    per_sm = 1;
  const int g = sm_count() * per_sm;
  return ntiles < g ? (ntiles > 0 ? ntiles : 1) : g;
}

constexpr int stages_for(int buf_bytes, int extra, int ctas) {
  const int s = ((224 * 1024) / ctas - extra - 1024) / buf_bytes;
  return s < 1 ? 1 : (s > 6 ? 6 : s);
}

// Resident CTAs per SM of the column passes (1: 255 registers and up to 3
// stages per CTA; 2: 128 registers and one or two stages each; 0: default).
int g_col_ctas = 0;

template <int R1, int R2, int MODE, int CTAS, bool PR>
int launch_col_ctas(const CUtensorMap& map, const ColArgs& a, cudaStream_t s) {
  using G = ColGeom<R1, R2>;
  constexpr int EXTRA = G::L * 8 + col_table_floats(MODE, G::L) * 4;
  constexpr int S = stages_for(G::BUF * 8, EXTRA, CTAS);
  const int smem = S * G::BUF * 8 + EXTRA + S * 8;
  auto k = col_pass_kernel<R1, R2, S, MODE, CTAS, PR>;
  PMB_CUDA_CHECK(smem_optin((const void*)k, smem));
  const int grid = persistent_grid(k, G::T, smem, a.ntiles);
  k<<<grid, G::T, smem, s>>>(map, a);
  PMB_CUDA_CHECK(cudaGetLastError());
  return kOk;
}

// One resident CTA per SM (255 registers, three stages) for every pass.  Two
// CTAs of 128 registers spill in the fused x passes; with the multiplier's
// tables in shared memory one CTA is faster (1024^3 on B200: x + multiplier
// 4.07 against 4.53 ms, adjoint 4.02 against 4.45 ms).
template <int R1, int R2, int MODE, bool PR>
int launch_col(const CUtensorMap& map, const ColArgs& a, cudaStream_t s) {
  return g_col_ctas == 2 ? launch_col_ctas<R1, R2, MODE, 2, PR>(map, a, s)
                         : launch_col_ctas<R1, R2, MODE, 1, PR>(map, a, s);
}

template <int MODE, bool PR = false>
int launch_col_len(int L, const CUtensorMap& map, const ColArgs& a, cudaStream_t s) {
  switch (L) {
    case 64: return launch_col<8, 8, MODE, PR>(map, a, s);
    case 128: return launch_col<16, 8, MODE, PR>(map, a, s);
    case 256: return launch_col<16, 16, MODE, PR>(map, a, s);
    case 512: return launch_col<32, 16, MODE, PR>(map, a, s);
    case 1024: return launch_col<32, 32, MODE, PR>(map, a, s);
    default: set_last_error("pmfft: unsupported transform length"); return kUnsupported;
  }
}

// the pruned instantiation of the modes a force chain runs pruned
template <int MODE>
int launch_col_len_pr(bool pr, int L, const CUtensorMap& map, const ColArgs& a, cudaStream_t s) {
  return pr ? launch_col_len<MODE, true>(L, map, a, s) : launch_col_len<MODE, false>(L, map, a, s);
}

template <int R1, int R2, bool C2R, bool PR>
int launch_z(const ZArgs& a, cudaStream_t s) {
  using G = ZGeom<R1, R2>;
  constexpr int stage = C2R ? KR * G::P * 8 : KR * G::M * 8;
  constexpr int S = 2;
  constexpr int smem = S * stage + G::XP * 8 + G::TW * 8 + S * 8;
  auto k = C2R ? z_c2r_kernel<R1, R2, S, PR> : z_r2c_kernel<R1, R2, S>;
  PMB_CUDA_CHECK(smem_optin((const void*)k, smem));
  const int grid = persistent_grid(k, G::T, smem, a.ntiles);
  k<<<grid, G::T, smem, s>>>(a);
  PMB_CUDA_CHECK(cudaGetLastError());
  return kOk;
}

template <bool C2R, bool PR>
int launch_z_len(int M, const ZArgs& a, cudaStream_t s) {
  switch (M) {
    case 64: return launch_z<8, 8, C2R, PR>(a, s);
    case 128: return launch_z<16, 8, C2R, PR>(a, s);
    case 256: return launch_z<16, 16, C2R, PR>(a, s);
    case 512: return launch_z<32, 16, C2R, PR>(a, s);
    default: set_last_error("pmfft: unsupported z length"); return kUnsupported;
  }
}

int encode(CUtensorMap* map, int rank, const void* base, const cuuint64_t* dims, const cuuint64_t* strides_bytes,
           const cuuint32_t* box) {
  auto fn = encode_fn();
  if (fn == nullptr) {
    set_last_error("pmfft: cuTensorMapEncodeTiled unavailable");
    return kCudaError;
  }
  cuuint32_t es[5] = {1, 1, 1, 1, 1};
  CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, rank, const_cast<void*>(base), dims, strides_bytes, box, es,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    set_last_error("pmfft: tensor map encoding failed");
    return kCudaError;
  }
  return kOk;
}

}  // namespace

bool pmfft_supported(Mesh3 m) {
  return pow2_in(m.nx, 64, 1024) && pow2_in(m.ny, 64, 1024) && pow2_in(m.nz, 128, 1024);
}

int pmfft_row_len(Mesh3 m) { return m.nz / 2 + 8; }

int64_t pmfft_channel_elems(Mesh3 m) { return (int64_t)m.nx * m.ny * pmfft_row_len(m); }

namespace {

// Masks that prune a force chain's passes: count table arrays at base +
// b * stride (base null: no pruning).
struct PruneSrc {
  const float* base;
  int64_t stride;
  int count;
};

PruneSrc prune_of(const SpecTables& t) { return PruneSrc{t.mx != nullptr ? t.kx : nullptr, 0, 1}; }

int z_pass(Mesh3 m, int inverse, int batch, const float* in_r, const float2* in_c, float* out_r, float2* out_c,
           PruneSrc pr, cudaStream_t s);
int col_pass(Mesh3 m, int mode, int nbatch, int ch_off, const float2* in, float2* out, SpecTables t, GreenParams g,
             const float* tab_base, int64_t tab_stride, int has_masks, int oofs, int ostride, int cstride, PruneSrc pr,
             cudaStream_t s);

}  // namespace

int pmfft_z(Mesh3 m, int inverse, int batch, const float* in_r, const float2* in_c, float* out_r, float2* out_c,
            cudaStream_t s) {
  return z_pass(m, inverse, batch, in_r, in_c, out_r, out_c, PruneSrc{nullptr, 0, 0}, s);
}

namespace {

int z_pass(Mesh3 m, int inverse, int batch, const float* in_r, const float2* in_c, float* out_r, float2* out_c,
           PruneSrc pr, cudaStream_t s) {
  if (!pmfft_supported(m) || batch < 1) {
    set_last_error("pmfft: unsupported mesh");
    return kUnsupported;
  }
  const int M = m.nz / 2;
  ZArgs a{};
  a.in_r = in_r;
  a.in_c = in_c;
  a.out_r = out_r;
  a.out_c = out_c;
  a.ch = pmfft_channel_elems(m);
  a.cells = m.cells();
  a.sb = (int64_t)m.nx * BY * pmfft_row_len(m);
  a.nx = m.nx;
  a.ny = m.ny;
  a.nz = m.nz;
  a.tiles_per_ch = (int)(m.rows() / KR);
  a.ntiles = a.tiles_per_ch * batch;
  a.polls = wait_polls();
  a.prune_base = pr.base;
  a.prune_stride = pr.stride;
  a.prune_count = pr.count;
  int st = twiddle_table(M, &a.tw_m);
  if (st != kOk) return st;
  st = twiddle_table(m.nz, &a.tw_n);
  if (st != kOk) return st;
  // only the inverse reads a pruned spectrum (the forward pass stores whole
  // rows: storing the live columns alone measured slower)
  if (inverse && pr.base != nullptr) return launch_z_len<true, true>(M, a, s);
  return inverse ? launch_z_len<true, false>(M, a, s) : launch_z_len<false, false>(M, a, s);
}

int col_pass(Mesh3 m, int mode, int nbatch, int ch_off, const float2* in, float2* out, SpecTables t, GreenParams g,
             const float* tab_base, int64_t tab_stride, int has_masks, int oofs, int ostride, int cstride, PruneSrc pr,
             cudaStream_t s) {
  if (!pmfft_supported(m) || nbatch < 1 || mode < kYFwd || mode > kXFwdAdjK) {
    set_last_error("pmfft: unsupported mesh or mode");
    return kUnsupported;
  }
  const int P = pmfft_row_len(m);
  const int nyb = m.ny / BY;
  const int nch = ch_off + nbatch * n_in(mode);
  ColArgs a{};
  a.out = out;
  a.ch = pmfft_channel_elems(m);
  a.sb = (int64_t)m.nx * BY * P;
  a.P = P;
  a.nx = m.nx;
  a.ny = m.ny;
  a.nz = m.nz;
  a.ch_off = ch_off;
  a.polls = wait_polls();
  a.t = t;
  a.g = g;
  a.tab_base = tab_base;
  a.tab_stride = tab_stride;
  a.has_masks = has_masks;
  a.oofs = oofs;
  a.ostride = ostride;
  a.cstride = cstride;
  if (mode == kXFwd || mode == kXInv || mode == kXFwdAdjK) pr = PruneSrc{nullptr, 0, 0};
  a.prune_base = pr.base;
  a.prune_stride = pr.stride;
  a.prune_count = pr.count;
  CUtensorMap map;
  int L, st;
  if (is_y(mode)) {
    L = m.ny;
    a.ncolt = P / KT;
    a.nouter = m.nx;
    const int box_rows = L < 256 ? L : 256;
    cuuint64_t dims[4] = {(cuuint64_t)P, (cuuint64_t)BY, (cuuint64_t)m.nx, (cuuint64_t)nyb * nch};
    cuuint64_t strides[3] = {(cuuint64_t)P * 8, (cuuint64_t)BY * P * 8, (cuuint64_t)a.sb * 8};
    cuuint32_t box[4] = {(cuuint32_t)KT, (cuuint32_t)BY, 1, (cuuint32_t)(box_rows / BY)};
    st = encode(&map, 4, in, dims, strides, box);
  } else {
    L = m.nx;
    a.ncolt = BY * P / KT;
    a.nouter = nyb;
    const int box_rows = L < 256 ? L : 256;
    cuuint64_t dims[3] = {(cuuint64_t)BY * P, (cuuint64_t)m.nx, (cuuint64_t)nyb * nch};
    cuuint64_t strides[2] = {(cuuint64_t)BY * P * 8, (cuuint64_t)a.sb * 8};
    cuuint32_t box[3] = {(cuuint32_t)KT, (cuuint32_t)box_rows, 1};
    st = encode(&map, 3, in, dims, strides, box);
  }
  if (st != kOk) return st;
  const int64_t ntiles = (int64_t)a.ncolt * a.nouter * nbatch;
  if (ntiles > 0x7fffffff) {
    set_last_error("pmfft: too many tiles");
    return kUnsupported;
  }
  a.ntiles = (int)ntiles;
  st = twiddle_table(L, &a.tw);
  if (st != kOk) return st;
  const bool pr_on = pr.base != nullptr;
  switch (mode) {
    case kYFwd: return launch_col_len_pr<kYFwd>(pr_on, L, map, a, s);
    case kYInv: return launch_col_len_pr<kYInv>(pr_on, L, map, a, s);
    case kYInvYZ: return launch_col_len_pr<kYInvYZ>(pr_on, L, map, a, s);
    case kYFwdYZ: return launch_col_len_pr<kYFwdYZ>(pr_on, L, map, a, s);
    case kXFwd: return launch_col_len<kXFwd>(L, map, a, s);
    case kXInv: return launch_col_len<kXInv>(L, map, a, s);
    case kXGreen: return launch_col_len_pr<kXGreen>(pr_on, L, map, a, s);
    case kXGreenAdj: return launch_col_len_pr<kXGreenAdj>(pr_on, L, map, a, s);
    default: return launch_col_len<kXFwdAdjK>(L, map, a, s);
  }
}

}  // namespace

int pmfft_col(Mesh3 m, int mode, int nbatch, int ch_off, const float2* in, float2* out, SpecTables t, GreenParams g,
              cudaStream_t s) {
  return col_pass(m, mode, nbatch, ch_off, in, out, t, g, nullptr, 0, 0, 0, 1, 1, PruneSrc{nullptr, 0, 0}, s);
}

int pmfft_col_batched(Mesh3 m, int mode, int nbatch, int ch_off, const float2* in, float2* out, SpecTables t,
                      GreenParams g, const float* tab_base, int64_t tab_stride, int has_masks, int oofs, int ostride,
                      int cstride, cudaStream_t s) {
  return col_pass(m, mode, nbatch, ch_off, in, out, t, g, tab_base, tab_stride, has_masks, oofs, ostride, cstride,
                  PruneSrc{nullptr, 0, 0}, s);
}

int pmfft_z_pruned(Mesh3 m, int inverse, int batch, const float* in_r, const float2* in_c, float* out_r, float2* out_c,
                   SpecTables prune_tables, cudaStream_t s) {
  return z_pass(m, inverse, batch, in_r, in_c, out_r, out_c, prune_of(prune_tables), s);
}

int pmfft_col_pruned(Mesh3 m, int mode, int nbatch, int ch_off, const float2* in, float2* out, SpecTables t,
                     GreenParams g, bool prune, cudaStream_t s) {
  return col_pass(m, mode, nbatch, ch_off, in, out, t, g, nullptr, 0, 0, 0, 1, 1,
                  prune ? prune_of(t) : PruneSrc{nullptr, 0, 0}, s);
}

int pmfft_set_col_ctas(int ctas) {
  if (ctas < 0 || ctas > 2) {
    set_last_error("pmfft: column-pass CTAs per SM must be 0 (per mode), 1 or 2");
    return kInvalidArgument;
  }
  g_col_ctas = ctas;
  return kOk;
}

int pmfft_timeouts(unsigned int* count) {
  PMB_CUDA_CHECK(cudaMemcpyFromSymbol(count, g_fft_timeouts, sizeof(unsigned int)));
  return kOk;
}

int pmfft_timeouts_clear() {
  const unsigned int zero = 0;
  PMB_CUDA_CHECK(cudaMemcpyToSymbol(g_fft_timeouts, &zero, sizeof(unsigned int)));
  return kOk;
}

// Forward force spectral chain: real source (1 channel) -> force meshes (3).
// work holds 5 channels of pmfft_channel_elems values.
int pmfft_force(Mesh3 m, const float* src, float* force_meshes, float2* work, SpecTables t, GreenParams g,
                cudaStream_t s) {
  const int64_t C = pmfft_channel_elems(m);
  float2* aq = work;       // A, then W (channel 0) and Q (channel 1)
  float2* fp = work + 2 * C;  // B (channel 0), then F'_x, F'_y, F'_z
  GreenParams none = g;
  const PruneSrc pr = prune_of(t);
  int st = z_pass(m, 0, 1, src, nullptr, nullptr, aq, pr, s);
  if (st != kOk) return st;
  if ((st = col_pass(m, kYFwd, 1, 0, aq, fp, t, none, nullptr, 0, 0, 0, 1, 1, pr, s)) != kOk) return st;
  if ((st = col_pass(m, kXGreen, 1, 0, fp, aq, t, g, nullptr, 0, 0, 0, 1, 1, pr, s)) != kOk) return st;
  if ((st = col_pass(m, kYInv, 1, 0, aq, fp, t, none, nullptr, 0, 0, 0, 1, 1, pr, s)) != kOk) return st;
  if ((st = col_pass(m, kYInvYZ, 1, 1, aq, fp + C, t, none, nullptr, 0, 0, 0, 1, 1, pr, s)) != kOk) return st;
  return z_pass(m, 1, 3, nullptr, fp, force_meshes, nullptr, pr, s);
}

// The forward chain for `count` equal-shape meshes in one launch per pass
// (ensembles): sources src[b], force meshes force_meshes[3 b + d], member b's
// tables at tab_base + b * tab_stride.  work holds 5 * count channels: the z
// pass and x pass outputs (W of every member, then Q), then the three force
// spectra of each member in order.
int pmfft_force_batched(Mesh3 m, int count, const float* src, float* force_meshes, float2* work,
                        const float* tab_base, int64_t tab_stride, int has_masks, GreenParams g, cudaStream_t s) {
  const int64_t C = pmfft_channel_elems(m);
  float2* aq = work;                  // A (count), then W (count) and Q (count)
  float2* fp = work + 2 * count * C;  // B (count), then F'_x, F'_y, F'_z per member
  GreenParams none = g;
  const SpecTables t0 = spec_tables_from(tab_base, m, has_masks);
  const PruneSrc pr{has_masks ? tab_base : nullptr, tab_stride, count};
  int st = z_pass(m, 0, count, src, nullptr, nullptr, aq, pr, s);
  if (st != kOk) return st;
  if ((st = col_pass(m, kYFwd, count, 0, aq, fp, t0, none, nullptr, 0, 0, 0, 1, 1, pr, s)) != kOk) return st;
  if ((st = col_pass(m, kXGreen, count, 0, fp, aq, t0, g, tab_base, tab_stride, has_masks, 0, 1, count, pr, s)) != kOk)
    return st;
  if ((st = col_pass(m, kYInv, count, 0, aq, fp, t0, none, nullptr, 0, 0, 0, 3, 1, pr, s)) != kOk) return st;
  if ((st = col_pass(m, kYInvYZ, count, count, aq, fp, t0, none, tab_base, tab_stride, has_masks, 1, 3, 1, pr, s)) !=
      kOk)
    return st;
  return z_pass(m, 1, 3 * count, nullptr, fp, force_meshes, nullptr, pr, s);
}

// Adjoint spectral chain: three mesh cotangents -> source cotangent.
int pmfft_force_adjoint(Mesh3 m, const float* mesh_cot, float* src_cot, float2* work, SpecTables t, GreenParams g,
                        cudaStream_t s) {
  const int64_t C = pmfft_channel_elems(m);
  float2* a3 = work;          // A_x, A_y, A_z; then S' (0) and S'' (1)
  float2* bb = work + 3 * C;  // B_x, b
  const PruneSrc pr = prune_of(t);
  int st = z_pass(m, 0, 3, mesh_cot, nullptr, nullptr, a3, pr, s);
  if (st != kOk) return st;
  if ((st = col_pass(m, kYFwd, 1, 0, a3, bb, t, g, nullptr, 0, 0, 0, 1, 1, pr, s)) != kOk) return st;
  if ((st = col_pass(m, kYFwdYZ, 1, 1, a3, bb + C, t, g, nullptr, 0, 0, 0, 1, 1, pr, s)) != kOk) return st;
  // fused x pass (4.45 ms at 1024^3) rather than the multiplier pass plus a
  // plain inverse x pass (3.45 + 1.49 ms)
  if ((st = col_pass(m, kXGreenAdj, 1, 0, bb, a3, t, g, nullptr, 0, 0, 0, 1, 1, pr, s)) != kOk) return st;
  if ((st = col_pass(m, kYInv, 1, 0, a3, a3 + C, t, g, nullptr, 0, 0, 0, 1, 1, pr, s)) != kOk) return st;
  return z_pass(m, 1, 1, nullptr, a3 + C, src_cot, nullptr, pr, s);
}

}  // namespace pmb
