// Ensembles of independent PM simulations of uneven sizes advanced together:
// one persistent launch per PM stage covers every simulation.
//
// The reference runs one simulation per call (nbody/solver.py:253-273); an
// ensemble there is a Python loop or a vmap over equal shapes.  Here the
// particles of all simulations are concatenated, the mesh rows of all
// simulations form one global row space (simulation s owns rows
// row0[s] .. row0[s] + nx*ny), so a single counting sort orders every
// particle of every simulation, and each stage kernel walks a flat work space
// (particles, scatter tiles or half-spectrum cells) and finds the owning
// simulation by binary search over a small prefix table.  Scatter tiles are
// handed out by an atomic work counter (largest simulations first), so
// uneven sizes and clustering balance across the SMs.  FFTs run as one
// batched cuFFT plan per distinct mesh shape (simulations of one shape are
// stored contiguously).  Per-simulation kick/drift factors live in a device
// table indexed by a device-side step counter, so one CUDA graph of a
// kick-drift-kick step replays for every step without host work.
//
// Every per-particle and per-cell operation is the single-simulation one
// (pmb_cic_device.cuh, pmb_spectral_device.cuh), so a simulation advanced in
// an ensemble gets the same arithmetic as when advanced alone.
#include <cufft.h>

#include <cmath>
#include <cstring>
#include <new>
#include <vector>

#include "../../include/pmb200.h"
#include "pmb_cic_device.cuh"
#include "pmb_common.cuh"
#include "pmb_kernels.cuh"
#include "pmb_spectral_device.cuh"

namespace pmb {

constexpr int kEnsMaxSims = 1024;

// Device descriptor of one member simulation.
struct EnsSim {
  int64_t p0, n;     // particle range in the concatenated particle arrays
  int64_t row0;      // first global mesh row
  Mesh3 m;
  int rx, ry;        // scatter tile shape
  float cell;        // mesh cell size
  float val;         // deposit per particle (mean density 1)
  float src_mul;     // 1.5 Omega_m, the Poisson source factor
  float post;        // 1 / cells, the inverse-FFT normalisation
  double scale;      // fixed-point scale of the density deposit
  float* rho;        // Poisson source mesh, (nx, ny, nz)
  float2* rho_hat;   // its half spectrum
  float2* grad_hat;  // three gradient spectra
  float* force;      // three force meshes
  SpecTables t;
  int pm;            // 1: the spectral stages run the hand-written pass chain
};

struct EnsDev {
  const EnsSim* sims;
  const int64_t* p_start;     // nsims + 1
  const int64_t* tile_start;  // nsims + 1
  const int64_t* spec_start;  // nsims + 1
  const float* fac;           // [steps][nsims][3]: opening kick, drift, closing kick
  const int* step;
  unsigned long long* work;   // scatter tile counter
  int nsims;
  int64_t ntot, ntiles, nspec;
  const int16_t* pmid;
  float* disp;
  float* vel;
  float* acc;
  Rec* rec;
  uint32_t* perm;
  uint32_t* offs;
  uint32_t* counts;
  uint32_t* row_of;
  uint32_t* rank_of;
};

// Largest s with start[s] <= x (start[0] == 0 <= x < start[nsims]).
__device__ __forceinline__ int find_sim(const int64_t* start, int nsims, int64_t x) {
  int lo = 0, hi = nsims - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (start[mid] <= x) lo = mid; else hi = mid - 1;
  }
  return lo;
}

__device__ __forceinline__ void load_starts(int64_t* sh, const int64_t* g, int nsims) {
  for (int i = threadIdx.x; i <= nsims; i += blockDim.x) sh[i] = g[i];
  __syncthreads();
}

// vel += acc * K_s  (integrator.py:512-538), K_s = opening kick of the step.
__global__ void ens_kick_kernel(EnsDev d) {
  __shared__ int64_t ps[kEnsMaxSims + 1];
  load_starts(ps, d.p_start, d.nsims);
  const float* f = d.fac + (int64_t)(*d.step) * d.nsims * 3;
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < d.ntot; p += (int64_t)gridDim.x * blockDim.x) {
    const float K = f[3 * find_sim(ps, d.nsims, p)];
#pragma unroll
    for (int c = 0; c < 3; ++c) d.vel[3 * p + c] = __fadd_rn(d.vel[3 * p + c], __fmul_rn(d.acc[3 * p + c], K));
  }
}

// Row counts over the global row space; with drift, disp += vel * D_s first
// (written back), as the single-simulation sort does.
__global__ void ens_bin_count_kernel(EnsDev d, int drift) {
  __shared__ int64_t ps[kEnsMaxSims + 1];
  load_starts(ps, d.p_start, d.nsims);
  const float* f = d.fac + (int64_t)(*d.step) * d.nsims * 3;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t base = (int64_t)blockIdx.x * blockDim.x; base < d.ntot; base += stride) {
    const int64_t i = base + threadIdx.x;
    const bool active = i < d.ntot;
    uint32_t row = 0xFFFFFFFFu;
    if (active) {
      const int s = find_sim(ps, d.nsims, i);
      const Mesh3 m = d.sims[s].m;
      float d0 = d.disp[3 * i], d1 = d.disp[3 * i + 1], d2 = d.disp[3 * i + 2];
      if (drift) {
        const float D = f[3 * s + 1];
        d0 = __fadd_rn(d0, __fmul_rn(d.vel[3 * i], D));
        d1 = __fadd_rn(d1, __fmul_rn(d.vel[3 * i + 1], D));
        d2 = __fadd_rn(d2, __fmul_rn(d.vel[3 * i + 2], D));
        d.disp[3 * i] = d0;
        d.disp[3 * i + 1] = d1;
        d.disp[3 * i + 2] = d2;
      }
      const Binned b = bin_particle(d.pmid, d0, d1, d2, i, m, d.sims[s].cell);
      row = (uint32_t)(d.sims[s].row0 + (int64_t)b.cx * m.ny + b.cy);
    }
    const unsigned full = __ballot_sync(0xFFFFFFFFu, active);
    if (active) {
      const unsigned peers = __match_any_sync(full, row);
      const int leader = __ffs(peers) - 1;
      const int lane = threadIdx.x & 31;
      uint32_t rb = 0;
      if (lane == leader) rb = atomicAdd(&d.counts[row], (uint32_t)__popc(peers));
      rb = __shfl_sync(peers, rb, leader);
      d.row_of[i] = row;
      d.rank_of[i] = rb + __popc(peers & ((1u << lane) - 1u));
    }
  }
}

__global__ void ens_bin_place_kernel(EnsDev d) {
  __shared__ int64_t ps[kEnsMaxSims + 1];
  load_starts(ps, d.p_start, d.nsims);
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < d.ntot; i += (int64_t)gridDim.x * blockDim.x) {
    const int s = find_sim(ps, d.nsims, i);
    const Mesh3 m = d.sims[s].m;
    const Binned b = bin_particle(d.pmid, d.disp[3 * i], d.disp[3 * i + 1], d.disp[3 * i + 2], i, m, d.sims[s].cell);
    const uint32_t dst = d.offs[d.row_of[i]] + d.rank_of[i];
    Rec r;
    r.fx = b.fx;
    r.fy = b.fy;
    r.fz = b.fz;
    r.key = (uint32_t)(((int64_t)b.cx * m.ny + b.cy) * m.nz + b.cz);
    d.rec[dst] = r;
    d.perm[dst] = (uint32_t)i;
  }
}

// Persistent deterministic scatter: CTAs pull scatter tiles from the work
// counter until every tile of every simulation is written.
__global__ void __launch_bounds__(256) ens_scatter_kernel(EnsDev d) {
  extern __shared__ __align__(16) unsigned int acc_smem[];
  __shared__ ScatterSmem sm;
  __shared__ long long item_sh;
  for (;;) {
    if (threadIdx.x == 0) item_sh = (long long)atomicAdd(d.work, 1ull);
    __syncthreads();
    const long long item = item_sh;
    if (item >= d.ntiles) break;
    const int s = find_sim(d.tile_start, d.nsims, item);
    const EnsSim& sim = d.sims[s];
    const Mesh3 m = sim.m;
    const int rx = sim.rx, ry = sim.ry;
    const int64_t local = item - d.tile_start[s];
    const int nby = (m.ny + ry - 1) / ry;
    const int x0 = (int)(local / nby) * rx, y0 = (int)(local % nby) * ry;
    scatter_tile<1>(d.rec, d.perm, d.offs + sim.row0, m, rx, ry, x0, y0, nullptr, 0, sim.val, sim.scale, 1,
                    sim.src_mul, sim.rho, acc_smem, sm);
  }
}

// Flat loop over the half spectra of all members; local cell coordinates
// from 32-bit index arithmetic (members have fewer than 2^31 half cells).
// odd_only: skip the members whose class the vector class kernel serves
// (half spectra of 4-divisible size at 4-aligned offsets).
__global__ void ens_green_kernel(EnsDev d, int odd_only) {
  __shared__ int64_t ss[kEnsMaxSims + 1];
  load_starts(ss, d.spec_start, d.nsims);
  for (int64_t jg = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; jg < d.nspec;
       jg += (int64_t)gridDim.x * blockDim.x) {
    const int s = find_sim(ss, d.nsims, jg);
    const EnsSim& sim = d.sims[s];
    if (sim.pm) continue;  // multiplier fused into the member's FFT pass chain
    if (odd_only && sim.m.half_cells() % 4 == 0 && (ss[s] & 3) == 0) continue;
    GreenParams g;
    g.green_kernel = 0;
    g.cell = 0.f;
    g.transfer = nullptr;
    g.radial = nullptr;
    g.radial_len = 0;
    g.post_scale = sim.post;
    const Mesh3 m = sim.m;
    const SpecTables t = sim.t;
    const uint32_t nzh = (uint32_t)(m.nz / 2 + 1), ny = (uint32_t)m.ny;
    const uint32_t j = (uint32_t)(jg - ss[s]);
    const uint32_t r = j / nzh, ix = r / ny;
    green_gradient_at(sim.rho_hat, sim.grad_hat, (int64_t)j, m.half_cells(), (int)ix, (int)(r - ix * ny),
                      (int)(j - r * nzh), m, t, g);
  }
}

// The multiplier of one mesh-shape class on the cuFFT route: blockIdx.y is
// the member (its own tables and post scale), the x blocks stride over its
// half spectrum four cells per thread with 32-byte vector loads and stores
// (members of one class have equal, 4-divisible half spectra, stored
// back to back).  The same per-cell arithmetic as ens_green_kernel, without
// its per-cell search over the members.
__global__ void ens_green_class_kernel(const EnsSim* __restrict__ sims, int first) {
  const EnsSim& sim = sims[first + blockIdx.y];
  GreenParams g;
  g.green_kernel = 0;
  g.cell = 0.f;
  g.transfer = nullptr;
  g.radial = nullptr;
  g.radial_len = 0;
  g.post_scale = sim.post;
  const Mesh3 m = sim.m;
  const SpecTables t = sim.t;
  const uint32_t nzh = (uint32_t)(m.nz / 2 + 1), ny = (uint32_t)m.ny;
  const uint32_t total = (uint32_t)m.half_cells(), groups = total / 4;
  const float4* s4 = reinterpret_cast<const float4*>(sim.rho_hat);
  for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < groups; q += gridDim.x * blockDim.x) {
    const uint32_t j = 4 * q, r = j / nzh, x = r / ny;
    int ix = (int)x, iy = (int)(r - x * ny), iz = (int)(j - r * nzh);
    const float4 a = s4[2 * q], b = s4[2 * q + 1];
    const float2 v[4] = {make_float2(a.x, a.y), make_float2(a.z, a.w), make_float2(b.x, b.y), make_float2(b.z, b.w)};
    float2 o[4][3];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      green_gradient_value(v[e], (int64_t)j + e, ix, iy, iz, m, t, g, o[e]);
      if (++iz == (int)nzh) {
        iz = 0;
        if (++iy == (int)ny) {
          iy = 0;
          ++ix;
        }
      }
    }
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      float4* g4 = reinterpret_cast<float4*>(sim.grad_hat + (int64_t)d * total);
      g4[2 * q] = make_float4(o[0][d].x, o[0][d].y, o[1][d].x, o[1][d].y);
      g4[2 * q + 1] = make_float4(o[2][d].x, o[2][d].y, o[3][d].x, o[3][d].y);
    }
  }
}

// acc = gather of the three force meshes; with kick, vel += acc * K_s (the
// closing half-kick of the step).
__global__ void ens_gather_kernel(EnsDev d, int kick) {
  __shared__ int64_t ps[kEnsMaxSims + 1];
  load_starts(ps, d.p_start, d.nsims);
  const float* f = d.fac + (int64_t)(*d.step) * d.nsims * 3;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < d.ntot; i += (int64_t)gridDim.x * blockDim.x) {
    // sorted positions of simulation s are [p0, p0 + n): its rows precede the next simulation's
    const int s = find_sim(ps, d.nsims, i);
    const EnsSim& sim = d.sims[s];
    gather_one<3>(d.rec[i], d.perm[i], sim.m, sim.force, d.acc, kick ? d.vel : nullptr, kick ? f[3 * s + 2] : 0.f);
  }
}

__global__ void ens_set_step_kernel(int* step, int v) { *step = v; }
__global__ void ens_advance_kernel(int* step) { *step += 1; }

struct EnsClass {
  Mesh3 m;
  int first, count;
  // pass-chain classes: the members' tables at a uniform stride (set at bind)
  const float* tab_base = nullptr;
  int64_t tab_stride = 0;
  int has_masks = 0;
  bool batched = false;
};

struct Ensemble {
  int nsims = 0;
  int max_steps = 0;
  int nsm = 148;
  std::vector<EnsSim> sims;
  std::vector<int> has_masks;
  std::vector<int64_t> p_start, tile_start, spec_start, mesh_start;
  std::vector<EnsClass> classes;
  int64_t ntot = 0, rows = 0, ntiles = 0, nspec = 0, ncells = 0;
  // launch shapes: threads and CTAs per SM of the particle / cell kernels
  int threads[8] = {256, 256, 256, 256, 256, 256, 256, 256};
  int ctas_per_sm[8] = {8, 8, 8, 8, 8, 8, 8, 8};
  bool bound = false;
  bool dirty = true;  // host descriptors changed since the last upload
  size_t scatter_smem = 0;
  int scatter_per_sm = 0;
  EnsDev dev{};
  EnsSim* d_sims = nullptr;
  uint32_t* tile_sums = nullptr;
  void* fft_work = nullptr;
  int64_t fft_bytes = 0;
  // the hand-written FFT pass chain (power-of-two member meshes): one work
  // area of five blocked spectral channels, reused member after member
  void* pm_work = nullptr;
  int64_t pm_bytes = 0;
  bool any_cufft = false;
  float* rho = nullptr;
  float2* rho_hat = nullptr;
  float2* grad_hat = nullptr;
  float* force = nullptr;
};

enum EnsStage { kStKick = 0, kStSort = 1, kStScatter = 2, kStR2C = 3, kStGreen = 4, kStC2R = 5, kStGather = 6 };

namespace {

#define ENS_REQUIRE(cond, msg) \
  do {                         \
    if (!(cond)) {             \
      set_last_error(msg);     \
      return kInvalidArgument; \
    }                          \
  } while (0)

#define ENS_TRY(expr)            \
  do {                           \
    int _st = (expr);            \
    if (_st != kOk) return _st;  \
  } while (0)

bool same_shape(Mesh3 a, Mesh3 b) { return a.nx == b.nx && a.ny == b.ny && a.nz == b.nz; }

int64_t tiles_of(const EnsSim& s) {
  return (int64_t)((s.m.nx + s.rx - 1) / s.rx) * ((s.m.ny + s.ry - 1) / s.ry);
}

void recount_tiles(Ensemble* e) {
  e->tile_start.assign(e->nsims + 1, 0);
  for (int s = 0; s < e->nsims; ++s) e->tile_start[s + 1] = e->tile_start[s] + tiles_of(e->sims[s]);
  e->ntiles = e->tile_start[e->nsims];
}

size_t scatter_smem_of(const Ensemble* e) {
  size_t mx = 0;
  for (const EnsSim& s : e->sims) {
    const size_t b = (size_t)ScatterSmem::acc_bytes(s.rx, s.ry, 1, s.m.nz);
    if (b > mx) mx = b;
  }
  return mx;
}

// Workspace: descriptors, prefix tables, factor table, step and work
// counters, sorted records, row offsets, sort scratch, cuFFT work area.
struct EnsLayout {
  int64_t sims, pst, tst, sst, fac, step, work, rec, perm, offs, counts, row_of, rank_of, tsums, fft, pm, total;
};

EnsLayout layout(const Ensemble* e) {
  EnsLayout L;
  int64_t off = 0;
  auto take = [&](int64_t b) {
    const int64_t o = off;
    off += align_up(b > 0 ? b : 1, 256);
    return o;
  };
  L.sims = take((int64_t)sizeof(EnsSim) * e->nsims);
  L.pst = take(8 * (int64_t)(e->nsims + 1));
  L.tst = take(8 * (int64_t)(e->nsims + 1));
  L.sst = take(8 * (int64_t)(e->nsims + 1));
  // one spare row: the step counter ends at max_steps after a full run
  L.fac = take(4 * 3 * (int64_t)e->nsims * (e->max_steps + 1));
  L.step = take(8);
  L.work = take(8);
  L.rec = take(16 * e->ntot);
  L.perm = take(4 * e->ntot);
  L.offs = take(4 * (e->rows + 1));
  L.counts = take(4 * (e->rows + 1));
  L.row_of = take(4 * e->ntot);
  L.rank_of = take(4 * e->ntot);
  L.tsums = take(4 * scan_tmp_elems(e->rows + 1));
  L.fft = take(e->fft_bytes);
  L.pm = take(e->pm_bytes);
  L.total = off;
  return L;
}

unsigned grid_of(const Ensemble* e, int stage, int64_t items) {
  const int th = e->threads[stage];
  int64_t b = (items + th - 1) / th;
  const int64_t cap = (int64_t)e->nsm * e->ctas_per_sm[stage];
  if (b > cap) b = cap;
  return (unsigned)(b > 0 ? b : 1);
}

// Uploads changed descriptors and sizes the persistent scatter launch.  Runs
// outside stream capture: every call after a descriptor change (bind,
// set_tiles) must precede a capture.
int upload(Ensemble* e, cudaStream_t s) {
  if (!e->dirty) return kOk;
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  PMB_CUDA_CHECK(cudaStreamIsCapturing(s, &cap));
  if (cap != cudaStreamCaptureStatusNone) {
    set_last_error("ensemble descriptors changed during stream capture; run one uncaptured call first");
    return kInvalidArgument;
  }
  // tile prefix table follows the (possibly retuned) tile shapes
  recount_tiles(e);
  e->dev.ntiles = e->ntiles;
  e->scatter_smem = scatter_smem_of(e);
  PMB_CUDA_CHECK(cudaFuncSetAttribute(ens_scatter_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)e->scatter_smem));
  PMB_CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&e->scatter_per_sm, ens_scatter_kernel, 256,
                                                               e->scatter_smem));
  PMB_CUDA_CHECK(cudaMemcpyAsync(e->d_sims, e->sims.data(), sizeof(EnsSim) * e->nsims, cudaMemcpyHostToDevice, s));
  PMB_CUDA_CHECK(cudaMemcpyAsync((void*)e->dev.tile_start, e->tile_start.data(), 8 * (e->nsims + 1),
                                 cudaMemcpyHostToDevice, s));
  e->dirty = false;
  return kOk;
}

int run_stage(Ensemble* e, int stage, int drift, int kick, cudaStream_t s) {
  const EnsDev& d = e->dev;
  switch (stage) {
    case kStKick:
      if (e->ntot > 0) ens_kick_kernel<<<grid_of(e, kStKick, e->ntot), e->threads[kStKick], 0, s>>>(d);
      break;
    case kStSort: {
      PMB_CUDA_CHECK(cudaMemsetAsync(d.counts, 0, 4 * (e->rows + 1), s));
      if (e->ntot > 0)
        ens_bin_count_kernel<<<grid_of(e, kStSort, e->ntot), e->threads[kStSort], 0, s>>>(d, drift);
      ENS_TRY(exclusive_scan_u32(d.counts, d.offs, e->rows + 1, e->tile_sums, s));
      if (e->ntot > 0) ens_bin_place_kernel<<<grid_of(e, kStSort, e->ntot), e->threads[kStSort], 0, s>>>(d);
      break;
    }
    case kStScatter: {
      const size_t smem = e->scatter_smem;
      const int per_sm = e->scatter_per_sm;
      if (per_sm < 1) {
        set_last_error("ensemble scatter: tile shape does not fit in shared memory");
        return kUnsupported;
      }
      int64_t grid = (int64_t)e->nsm * per_sm;
      if (grid > e->ntiles) grid = e->ntiles;
      PMB_CUDA_CHECK(cudaMemsetAsync(d.work, 0, 8, s));
      if (grid > 0) ens_scatter_kernel<<<(unsigned)grid, 256, smem, s>>>(d);
      break;
    }
    case kStR2C:
      // members on the pass chain run their whole spectral chain here (the
      // same kernels as a single run's pmb_force); the others R2C by class
      for (const EnsClass& c : e->classes) {
        if (e->sims[c.first].pm && c.batched) {
          // the whole class in one launch per pass, each member with its tables
          GreenParams g;
          g.green_kernel = 0;
          g.cell = 0.f;
          g.transfer = nullptr;
          g.radial = nullptr;
          g.radial_len = 0;
          g.post_scale = e->sims[c.first].post;
          ENS_TRY(pmfft_force_batched(c.m, c.count, e->sims[c.first].rho, e->sims[c.first].force,
                                      (float2*)e->pm_work, c.tab_base, c.tab_stride, c.has_masks, g, s));
        } else if (e->sims[c.first].pm) {
          for (int i = c.first; i < c.first + c.count; ++i) {
            const EnsSim& q = e->sims[i];
            GreenParams g;
            g.green_kernel = 0;
            g.cell = 0.f;
            g.transfer = nullptr;
            g.radial = nullptr;
            g.radial_len = 0;
            g.post_scale = q.post;
            ENS_TRY(pmfft_force(q.m, q.rho, q.force, (float2*)e->pm_work, q.t, g, s));
          }
        } else {
          ENS_TRY(fft_r2c(c.m, c.count, e->sims[c.first].rho, e->sims[c.first].rho_hat, e->fft_work, s));
        }
      }
      break;
    case kStGreen:
      if (e->nspec > 0 && e->any_cufft) {
        // classes whose half spectra split into aligned groups of four run the
        // class kernel; any other cuFFT member takes the flat kernel
        bool flat = false;
        for (const EnsClass& c : e->classes) {
          if (e->sims[c.first].pm) continue;
          const int64_t hc = c.m.half_cells();
          if (hc % 4 != 0 || (e->spec_start[c.first] & 3) != 0) {
            flat = true;
            continue;
          }
          const int th = e->threads[kStGreen];
          int64_t bx = (hc / 4 + th - 1) / th;
          const int64_t cap = ((int64_t)e->nsm * e->ctas_per_sm[kStGreen] + c.count - 1) / c.count;
          if (bx > cap) bx = cap;
          ens_green_class_kernel<<<dim3((unsigned)(bx > 0 ? bx : 1), (unsigned)c.count), th, 0, s>>>(e->d_sims,
                                                                                                  c.first);
        }
        if (flat) ens_green_kernel<<<grid_of(e, kStGreen, e->nspec), e->threads[kStGreen], 0, s>>>(d, 1);
      }
      break;
    case kStC2R:
      for (const EnsClass& c : e->classes)
        if (!e->sims[c.first].pm)
          ENS_TRY(fft_c2r(c.m, 3 * c.count, e->sims[c.first].grad_hat, e->sims[c.first].force, e->fft_work, s));
      break;
    case kStGather:
      if (e->ntot > 0) ens_gather_kernel<<<grid_of(e, kStGather, e->ntot), e->threads[kStGather], 0, s>>>(d, kick);
      break;
    default:
      set_last_error("unknown ensemble stage");
      return kInvalidArgument;
  }
  PMB_CUDA_CHECK(cudaGetLastError());
  return kOk;
}

}  // namespace
}  // namespace pmb

using namespace pmb;

extern "C" {

int pmb_ens_create(int nsims, const int64_t* counts, const int32_t* mesh_shapes, const float* cells,
                   const float* vals, const float* src_muls, const int32_t* has_masks, int max_steps,
                   void** handle) {
  ENS_REQUIRE(handle != nullptr, "pmb_ens_create: null handle");
  *handle = nullptr;
  ENS_REQUIRE(nsims >= 1 && nsims <= kEnsMaxSims, "pmb_ens_create: 1..1024 simulations supported");
  ENS_REQUIRE(max_steps >= 0 && max_steps <= 1 << 20, "pmb_ens_create: max_steps out of range");
  ENS_REQUIRE(counts && mesh_shapes && cells && vals && src_muls && has_masks, "pmb_ens_create: null array");
  Ensemble* e = new (std::nothrow) Ensemble();
  ENS_REQUIRE(e != nullptr, "pmb_ens_create: out of host memory");
  e->nsims = nsims;
  e->max_steps = max_steps;
  e->sims.resize(nsims);
  e->has_masks.assign(has_masks, has_masks + nsims);
  e->p_start.assign(nsims + 1, 0);
  e->spec_start.assign(nsims + 1, 0);
  e->mesh_start.assign(nsims + 1, 0);
  int64_t row0 = 0;
  for (int s = 0; s < nsims; ++s) {
    EnsSim& q = e->sims[s];
    std::memset(&q, 0, sizeof(q));
    q.m = Mesh3{mesh_shapes[3 * s], mesh_shapes[3 * s + 1], mesh_shapes[3 * s + 2]};
    const bool ok_mesh = q.m.nx >= 1 && q.m.ny >= 1 && q.m.nz >= 1 && q.m.nz <= 4096 &&
                         (double)q.m.nx * q.m.ny * q.m.nz < 4294967296.0 &&
                         (double)q.m.nx * q.m.ny * (q.m.nz / 2 + 1) < 2147483648.0;
    if (!ok_mesh || counts[s] < 0 || !(cells[s] > 0.f) || !std::isfinite(vals[s])) {
      delete e;
      set_last_error("pmb_ens_create: invalid simulation description");
      return kInvalidArgument;
    }
    // simulations of one mesh shape must be contiguous (one batched FFT per shape)
    if (s > 0 && !same_shape(q.m, e->sims[s - 1].m)) {
      for (const EnsClass& c : e->classes)
        if (same_shape(c.m, q.m)) {
          delete e;
          set_last_error("pmb_ens_create: simulations of equal mesh shape must be consecutive");
          return kInvalidArgument;
        }
    }
    if (s == 0 || !same_shape(q.m, e->sims[s - 1].m)) e->classes.push_back(EnsClass{q.m, s, 0});
    e->classes.back().count += 1;
    q.p0 = e->p_start[s];
    q.n = counts[s];
    q.row0 = row0;
    row0 += q.m.rows();
    q.cell = cells[s];
    q.val = vals[s];
    q.src_mul = src_muls[s];
    q.post = (float)(1.0 / (double)q.m.cells());
    const float a = fabsf(vals[s]);
    q.scale = fixed_point_scale(fixed_point_pow2(q.n), a);
    q.rx = 2;
    q.ry = 2;
    if (q.rx > q.m.nx) q.rx = q.m.nx;
    if (q.ry > q.m.ny) q.ry = q.m.ny;
    e->p_start[s + 1] = e->p_start[s] + counts[s];
    e->spec_start[s + 1] = e->spec_start[s] + q.m.half_cells();
    e->mesh_start[s + 1] = e->mesh_start[s] + q.m.cells();
  }
  e->ntot = e->p_start[nsims];
  e->rows = row0;
  e->nspec = e->spec_start[nsims];
  e->ncells = e->mesh_start[nsims];
  if (e->ntot >= 4294967295ll || e->rows >= 4294967295ll) {
    delete e;
    set_last_error("pmb_ens_create: more than 2^32-1 particles or rows");
    return kInvalidArgument;
  }
  recount_tiles(e);
  int64_t fb = 0;
  for (const EnsClass& c : e->classes) {
    if (pmfft_enabled() && pmfft_supported(c.m)) {
      for (int i = c.first; i < c.first + c.count; ++i) e->sims[i].pm = 1;
      const int64_t pb = 5 * 8 * pmfft_channel_elems(c.m) * c.count;
      e->pm_bytes = e->pm_bytes > pb ? e->pm_bytes : pb;
      continue;
    }
    e->any_cufft = true;
    const int64_t w1 = fft_work_bytes(c.m, c.count), w3 = fft_work_bytes(c.m, 3 * c.count);
    if (w1 < 0 || w3 < 0) {
      delete e;
      return kCufftError;
    }
    fb = fb > w1 ? fb : w1;
    fb = fb > w3 ? fb : w3;
  }
  e->fft_bytes = fb;
  int dev = 0;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&e->nsm, cudaDevAttrMultiProcessorCount, dev);
  *handle = e;
  return kOk;
}

int pmb_ens_destroy(void* handle) {
  delete (Ensemble*)handle;
  return kOk;
}

int64_t pmb_ens_workspace_bytes(const void* handle) {
  if (handle == nullptr) return -1;
  return layout((const Ensemble*)handle).total;
}

int64_t pmb_ens_size(const void* handle, int which) {
  const Ensemble* e = (const Ensemble*)handle;
  if (e == nullptr) return -1;
  switch (which) {
    case 0: return e->ntot;
    case 1: return e->ncells;
    case 2: return e->nspec;
    case 3: return e->ntiles;
    case 4: return (int64_t)e->classes.size();
    default: return -1;
  }
}

int pmb_ens_bind(void* handle, const int16_t* pmid, float* disp, float* vel, float* acc, float* rho, void* rho_hat,
                 void* grad_hat, float* force, const float* tables, const int64_t* table_offsets, void* workspace,
                 int64_t workspace_bytes, void* stream) {
  Ensemble* e = (Ensemble*)handle;
  ENS_REQUIRE(e != nullptr, "pmb_ens_bind: null handle");
  const EnsLayout L = layout(e);
  ENS_REQUIRE(workspace != nullptr && workspace_bytes >= L.total, "pmb_ens_bind: workspace too small");
  ENS_REQUIRE(((uintptr_t)workspace & 255) == 0, "pmb_ens_bind: workspace must be 256-byte aligned");
  cudaStream_t s = (cudaStream_t)stream;
  char* w = (char*)workspace;
  e->rho = rho;
  e->rho_hat = (float2*)rho_hat;
  e->grad_hat = (float2*)grad_hat;
  e->force = force;
  for (int i = 0; i < e->nsims; ++i) {
    EnsSim& q = e->sims[i];
    q.rho = rho + e->mesh_start[i];
    q.rho_hat = (float2*)rho_hat + e->spec_start[i];
    q.grad_hat = (float2*)grad_hat + 3 * e->spec_start[i];
    q.force = force + 3 * e->mesh_start[i];
    q.t = spec_tables_from(tables + table_offsets[i], q.m, e->has_masks[i]);
  }
  for (EnsClass& c : e->classes) {
    // one batched pass chain per class when the members' tables sit at a
    // uniform stride with the same masks (the layout the host builds)
    c.tab_base = tables + table_offsets[c.first];
    c.has_masks = e->has_masks[c.first];
    c.tab_stride = c.count > 1 ? table_offsets[c.first + 1] - table_offsets[c.first] : 0;
    bool ok = true;
    for (int i = c.first; i < c.first + c.count; ++i)
      ok = ok && e->has_masks[i] == c.has_masks &&
           table_offsets[i] == table_offsets[c.first] + (int64_t)(i - c.first) * c.tab_stride;
    c.batched = ok;
  }
  e->d_sims = (EnsSim*)(w + L.sims);
  e->tile_sums = (uint32_t*)(w + L.tsums);
  e->fft_work = w + L.fft;
  e->pm_work = w + L.pm;
  EnsDev& d = e->dev;
  d.sims = e->d_sims;
  d.p_start = (const int64_t*)(w + L.pst);
  d.tile_start = (const int64_t*)(w + L.tst);
  d.spec_start = (const int64_t*)(w + L.sst);
  d.fac = (const float*)(w + L.fac);
  d.step = (const int*)(w + L.step);
  d.work = (unsigned long long*)(w + L.work);
  d.nsims = e->nsims;
  d.ntot = e->ntot;
  d.ntiles = e->ntiles;
  d.nspec = e->nspec;
  d.pmid = pmid;
  d.disp = disp;
  d.vel = vel;
  d.acc = acc;
  d.rec = (Rec*)(w + L.rec);
  d.perm = (uint32_t*)(w + L.perm);
  d.offs = (uint32_t*)(w + L.offs);
  d.counts = (uint32_t*)(w + L.counts);
  d.row_of = (uint32_t*)(w + L.row_of);
  d.rank_of = (uint32_t*)(w + L.rank_of);
  PMB_CUDA_CHECK(cudaMemcpyAsync((void*)d.p_start, e->p_start.data(), 8 * (e->nsims + 1), cudaMemcpyHostToDevice, s));
  PMB_CUDA_CHECK(
      cudaMemcpyAsync((void*)d.spec_start, e->spec_start.data(), 8 * (e->nsims + 1), cudaMemcpyHostToDevice, s));

  PMB_CUDA_CHECK(cudaMemsetAsync((void*)d.fac, 0, 4 * 3 * (int64_t)e->nsims * (e->max_steps + 1), s));
  ens_set_step_kernel<<<1, 1, 0, s>>>((int*)d.step, 0);
  PMB_CUDA_CHECK(cudaGetLastError());
  e->dirty = true;
  e->bound = true;
  return upload(e, s);
}

int pmb_ens_set_tiles(void* handle, const int32_t* rx, const int32_t* ry) {
  Ensemble* e = (Ensemble*)handle;
  ENS_REQUIRE(e != nullptr, "pmb_ens_set_tiles: null handle");
  for (int i = 0; i < e->nsims; ++i) {
    const EnsSim& q = e->sims[i];
    ENS_REQUIRE(rx[i] >= 1 && ry[i] >= 1 && (rx[i] + 1) * (ry[i] + 1) <= kMaxSrcRows && rx[i] <= q.m.nx &&
                    ry[i] <= q.m.ny && ScatterSmem::acc_bytes(rx[i], ry[i], 1, q.m.nz) <= 200 * 1024,
                "pmb_ens_set_tiles: tile shape out of range");
  }
  for (int i = 0; i < e->nsims; ++i) {
    e->sims[i].rx = rx[i];
    e->sims[i].ry = ry[i];
  }
  e->dirty = true;
  return kOk;
}

int pmb_ens_set_launch(void* handle, int stage, int threads, int ctas_per_sm) {
  Ensemble* e = (Ensemble*)handle;
  ENS_REQUIRE(e != nullptr, "pmb_ens_set_launch: null handle");
  ENS_REQUIRE(stage >= 0 && stage < 8 && stage != kStScatter, "pmb_ens_set_launch: stage has no launch shape");
  ENS_REQUIRE(threads >= 64 && threads <= 1024 && threads % 32 == 0, "pmb_ens_set_launch: threads out of range");
  ENS_REQUIRE(ctas_per_sm >= 1 && ctas_per_sm <= 32, "pmb_ens_set_launch: CTAs per SM out of range");
  e->threads[stage] = threads;
  e->ctas_per_sm[stage] = ctas_per_sm;
  return kOk;
}

int pmb_ens_set_factors(void* handle, int nsteps, const float* factors, void* stream) {
  Ensemble* e = (Ensemble*)handle;
  ENS_REQUIRE(e != nullptr && e->bound, "pmb_ens_set_factors: ensemble not bound");
  ENS_REQUIRE(nsteps >= 0 && nsteps <= e->max_steps, "pmb_ens_set_factors: more steps than max_steps");
  if (nsteps > 0)
    PMB_CUDA_CHECK(cudaMemcpyAsync((void*)e->dev.fac, factors, 4 * 3 * (int64_t)e->nsims * nsteps,
                                   cudaMemcpyHostToDevice, (cudaStream_t)stream));
  return kOk;
}

int pmb_ens_set_step(void* handle, int step, void* stream) {
  Ensemble* e = (Ensemble*)handle;
  ENS_REQUIRE(e != nullptr && e->bound, "pmb_ens_set_step: ensemble not bound");
  ENS_REQUIRE(step >= 0 && step < (e->max_steps > 0 ? e->max_steps : 1), "pmb_ens_set_step: step out of range");
  ens_set_step_kernel<<<1, 1, 0, (cudaStream_t)stream>>>((int*)e->dev.step, step);
  PMB_CUDA_CHECK(cudaGetLastError());
  return kOk;
}

int pmb_ens_stage(void* handle, int stage, int drift, int kick, void* stream) {
  Ensemble* e = (Ensemble*)handle;
  ENS_REQUIRE(e != nullptr && e->bound, "pmb_ens_stage: ensemble not bound");
  cudaStream_t s = (cudaStream_t)stream;
  ENS_TRY(upload(e, s));
  return run_stage(e, stage, drift, kick, s);
}

int pmb_ens_force(void* handle, int drift, int kick, void* stream) {
  Ensemble* e = (Ensemble*)handle;
  ENS_REQUIRE(e != nullptr && e->bound, "pmb_ens_force: ensemble not bound");
  cudaStream_t s = (cudaStream_t)stream;
  ENS_TRY(upload(e, s));
  ENS_TRY(run_stage(e, kStSort, drift, 0, s));
  ENS_TRY(run_stage(e, kStScatter, 0, 0, s));
  ENS_TRY(run_stage(e, kStR2C, 0, 0, s));
  ENS_TRY(run_stage(e, kStGreen, 0, 0, s));
  ENS_TRY(run_stage(e, kStC2R, 0, 0, s));
  return run_stage(e, kStGather, 0, kick, s);
}

int pmb_ens_step(void* handle, void* stream) {
  Ensemble* e = (Ensemble*)handle;
  ENS_REQUIRE(e != nullptr && e->bound, "pmb_ens_step: ensemble not bound");
  cudaStream_t s = (cudaStream_t)stream;
  ENS_TRY(upload(e, s));
  ENS_TRY(run_stage(e, kStKick, 0, 0, s));
  ENS_TRY(pmb_ens_force(handle, 1, 1, stream));
  ens_advance_kernel<<<1, 1, 0, s>>>((int*)e->dev.step);
  PMB_CUDA_CHECK(cudaGetLastError());
  return kOk;
}

}  // extern "C"
