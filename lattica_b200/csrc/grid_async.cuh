// Thin inline-PTX wrappers for the sm_100a asynchronous copy engine (TMA bulk
// copies, mbarriers) used by the streaming kernels. Every wait is bounded:
// after kMaxSpins failed polls the caller records GRID_DEV_TIMEOUT in the
// device error word and abandons the work item instead of spinning forever.
#pragma once
#include <stdint.h>

namespace grid {

constexpr uint32_t kMaxSpins = 1u << 22;

enum DeviceError : int {
  GRID_DEV_OK = 0,
  GRID_DEV_TIMEOUT = 1,
  GRID_DEV_SAMPLE_SHORT = 2,  // the uniform sampler ran out of candidates
};

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count)
               : "memory");
}

__device__ __forceinline__ void mbar_inval(uint64_t* bar) {
  asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_addr(bar)) : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
               "r"(bytes)
               : "memory");
}

// Plain arrive (release semantics, shared::cta).
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait on an mbarrier phase. Returns false (and records a timeout in
// *err) if the phase did not complete within max_spins polls.
__device__ __forceinline__ bool mbar_wait_budget(uint64_t* bar, uint32_t parity,
                                                 uint32_t max_spins, int* err) {
  for (uint32_t i = 0; i < max_spins; ++i) {
    if (mbar_try_wait(bar, parity)) return true;
  }
  atomicExch(err, GRID_DEV_TIMEOUT);
  return false;
}

// The kernels' wait: kMaxSpins polls.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int* err) {
  return mbar_wait_budget(bar, parity, kMaxSpins, err);
}

// Bounded wait that lets the thread sleep in the barrier between polls
// (suspend-time hint of 20 us; the thread resumes as soon as the phase
// completes), so waiting warps take no issue slots from working ones. Gives
// up after kMaxSleeps polls (about 1.3 s at most).
constexpr uint32_t kMaxSleeps = 1u << 16;

__device__ __forceinline__ bool mbar_wait_sleep(uint64_t* bar, uint32_t parity, int* err) {
  for (uint32_t i = 0; i < kMaxSleeps; ++i) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity), "r"(20000u)
        : "memory");
    if (ok) return true;
  }
  atomicExch(err, GRID_DEV_TIMEOUT);
  return false;
}

// Global -> shared bulk copy completing on an mbarrier (bytes multiple of 16,
// both addresses 16-byte aligned).
__device__ __forceinline__ void bulk_load(void* dst_smem, const void* src_gmem, uint32_t bytes,
                                          uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(smem_addr(dst_smem)),
      "l"(src_gmem), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}

// Shared -> global bulk copy tracked by the issuing thread's bulk group.
__device__ __forceinline__ void bulk_store(void* dst_gmem, const void* src_smem, uint32_t bytes) {
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst_gmem),
               "r"(smem_addr(src_smem)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ void bulk_commit() {
  asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}

// Wait until this thread's committed bulk stores have finished reading shared memory.
__device__ __forceinline__ void bulk_wait_read_all() {
  asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
}

// Wait until this thread's committed bulk stores are complete.
__device__ __forceinline__ void bulk_wait_all() {
  asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
}

// Per-thread 16-byte global -> shared copy (L2 only); src_bytes < 16 zero-fills
// the rest (0 reads nothing). Both addresses 16-byte aligned.
__device__ __forceinline__ void cp_async16(void* dst_smem, const void* src_gmem,
                                           uint32_t src_bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(smem_addr(dst_smem)),
               "l"(src_gmem), "r"(src_bytes)
               : "memory");
}

// Per-thread 8-byte global -> shared copy (through L1); src_bytes < 8 zero-fills
// the rest. Both addresses 8-byte aligned.
__device__ __forceinline__ void cp_async8(void* dst_smem, const void* src_gmem,
                                          uint32_t src_bytes) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(smem_addr(dst_smem)),
               "l"(src_gmem), "r"(src_bytes)
               : "memory");
}

__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;" ::: "memory");
}

// Wait until at most N of this thread's committed copy groups are pending.
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Order generic-proxy shared-memory accesses before later async-proxy (TMA) accesses.
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

}  // namespace grid
