// Density scatter for callers that cannot allocate device memory.
//
// Some callers of this library are not allowed to allocate: a framework
// plugin (for example an XLA custom-call handler) runs inside a host program
// that owns every device allocation, may be handed no scratch buffer at all,
// and must not call cudaMalloc behind the framework's back -- the rule the
// reference states for its own native handlers (cuda/route_kernels.cu:1-7).
// pmb_scatter_density_noalloc serves them: it runs the same cell sort and
// deterministic pull scatter as pmb_sort_rows + pmb_scatter_rows, but takes
// its scratch (sorted records, permutation, row counts and offsets, scan
// partials, fixed-point scale) from one file-scope device array of fixed size
// instead of from a caller workspace.
//
// Costs and limits:
//  * the array is kNoAllocScratchBytes (32 MiB) of device memory that every
//    GPU which loads this library holds until the process exits;
//  * a call needs 28 bytes per particle plus 12 bytes per mesh row (and a few
//    hundred bytes of alignment); larger problems, like invalid arguments, are
//    rejected with an error before any work is queued (use the workspace entry
//    points instead);
//  * every call on a device shares the same array and leaves its contents
//    behind, so calls whose execution overlaps on the GPU (different streams,
//    or host threads) race and corrupt each other: serialise them;
//  * the first call on each device looks up the array's device address with
//    cudaGetSymbolAddress (with that device current); make that first call
//    before any stream capture.
#include <cmath>
#include <mutex>

#include "../../include/pmb200.h"
#include "pmb_common.cuh"
#include "pmb_integrate.cuh"
#include "pmb_kernels.cuh"

namespace {

constexpr int64_t kNoAllocScratchBytes = int64_t(32) << 20;

// The scratch itself.  Host code must not use this name as an address (on
// the host it is only a stand-in for the symbol); it passes the address from
// cudaGetSymbolAddress to the kernels instead.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void* g_scratch_addr[kMaxDevices] = {nullptr};

// Per-device set-up: resolve the device address of the array once, with the
// device current.
int scratch_address(void** out) {
  int dev = 0;
  PMB_CUDA_CHECK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) {
    pmb::set_last_error("pmb_scatter_density_noalloc: device index out of range");
    return pmb::kUnsupported;
  }
  std::lock_guard<std::mutex> lk(g_mu);
  if (g_scratch_addr[dev] == nullptr) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr) {
      pmb::set_last_error(e != cudaSuccess ? cudaGetErrorString(e) : "cudaGetSymbolAddress returned null");
      return pmb::kCudaError;
    }
    g_scratch_addr[dev] = p;
  }
  *out = g_scratch_addr[dev];
  return pmb::kOk;
}

}  // namespace

extern "C" int pmb_scatter_density_noalloc(const int16_t* pmid, const float* disp, int64_t n, int nx, int ny, int nz,
                                           float cell, float val, float* out, void* stream) {
  using namespace pmb;
  if (nx < 1 || ny < 1 || nz < 1 || nz > 4096 || (double)nx * ny * nz >= 4294967296.0) {
    set_last_error("pmb_scatter_density_noalloc: unsupported mesh shape");
    return kInvalidArgument;
  }
  if (n < 0 || n >= 4294967295ll || !(cell > 0.f) || pmid == nullptr || disp == nullptr || out == nullptr) {
    set_last_error("pmb_scatter_density_noalloc: invalid argument");
    return kInvalidArgument;
  }
  if (!(fabsf(val) < INFINITY)) {
    set_last_error("pmb_scatter_density_noalloc: non-finite value");
    return kInvalidArgument;
  }
  Mesh3 m{nx, ny, nz};
  const int64_t rec_bytes = align_up(16 * n, 256), perm_bytes = align_up(4 * n, 256);
  const int64_t offs_bytes = align_up(4 * (m.rows() + 1), 256);
  const int64_t bins_bytes = bin_scratch_bytes(n, m);
  const int64_t need = rec_bytes + perm_bytes + offs_bytes + bins_bytes + 256 + 256;
  if (need > kNoAllocScratchBytes) {
    set_last_error("pmb_scatter_density_noalloc: problem needs more than the fixed 32 MiB scratch "
                   "(28 B per particle + 12 B per mesh row); use pmb_sort_rows + pmb_scatter_rows");
    return kInvalidArgument;
  }
  void* base = nullptr;
  int st = scratch_address(&base);
  if (st != kOk) return st;
  char* p = (char*)base;
  Rec* rec = (Rec*)p;
  uint32_t* perm = (uint32_t*)(p + rec_bytes);
  uint32_t* offs = (uint32_t*)(p + rec_bytes + perm_bytes);
  void* bins = p + rec_bytes + perm_bytes + offs_bytes;
  double* scale = (double*)(p + rec_bytes + perm_bytes + offs_bytes + bins_bytes);
  uint32_t* status = (uint32_t*)(p + rec_bytes + perm_bytes + offs_bytes + bins_bytes + 256);
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  // bin_particles zeroes the row counts itself; the scale word is rewritten
  // below, so nothing left over from an earlier call is read.
  st = bin_particles(pmid, const_cast<float*>(disp), nullptr, 0.f, n, m, cell, rec, perm, offs, bins, s, nullptr,
                     nullptr, status);
  if (st != kOk) return st;
  st = set_double(scale, fixed_point_scale(fixed_point_pow2(n), fabsf(val)), s);
  if (st != kOk) return st;
  return scatter_sorted(rec, perm, offs, m, 1, nullptr, 0, val, scale, 0, 1.f, out, s, n, status);
}
