// Bulk asynchronous copies (global -> shared, cp.async.bulk) completed through
// an mbarrier transaction count, with bounded waits.
//
// Every copy reads this GPU's own memory into the issuing CTA's shared memory
// only (no copies into other CTAs of a cluster).  Copies need 16-byte aligned
// source and destination and a size that is a multiple of 16 bytes.
#pragma once

#include <cstdint>

namespace pmb {

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

// Default poll limit of a bounded wait (pmb_set_wait_limit changes the limit
// of the first wait; the drain after a timeout always uses this one).
constexpr uint32_t kWaitPolls = 1u << 22;

// Waits for the given phase parity of the barrier; gives up after `polls`
// polls (each poll may suspend the thread for a short, hardware-defined time;
// 0 polls gives up at once) and returns false.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, uint32_t polls = kWaitPolls) {
  for (uint32_t it = 0; it < polls; ++it) {
    uint32_t done;
    asm volatile(
        "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// After a timed-out wait on ring slot `first` of an S-stage ring whose slots
// [first, end) were issued: waits (kWaitPolls each) for every copy still in
// flight, so that none lands in shared memory after the CTA has moved on.  If
// one of these waits gives up as well, the launch's results are undefined;
// the timeout is reported either way.
__device__ __forceinline__ void mbar_drain(uint64_t* bars, int S, int first, int end) {
  for (int j = first; j < end && j < first + S; ++j) mbar_wait(&bars[j % S], (uint32_t)((j / S) & 1));
}

// Wait used by every thread of a CTA after issuing bulk copies on one
// barrier: on a timeout the counter (a device variable of the calling file,
// reported by pmb_wait_timeouts and pmb_device_status) is raised and the
// copies still in flight get the drain wait before the caller returns without
// touching the staged data.
__device__ __forceinline__ bool mbar_wait_or_flag(uint64_t* bar, uint32_t parity, unsigned int* timeouts,
                                                  uint32_t polls = kWaitPolls) {
  if (__syncthreads_or(!mbar_wait(bar, parity, polls)) == 0) return true;
  if (threadIdx.x == 0) atomicAdd(timeouts, 1u);
  mbar_wait(bar, parity);
  return false;
}

}  // namespace pmb
