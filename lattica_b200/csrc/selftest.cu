// Test support for the failure path of the bounded device waits.
//
// Every wait of the library's kernels on an mbarrier phase gives up after a
// fixed number of polls, records GRID_DEV_TIMEOUT in the plan's device error
// word and lets the kernel finish, so the context stays usable and
// grid_gpu_plan_check reports GRID_ERR_TIMEOUT. This entry point exercises that
// path without a real stall: one warp waits on an mbarrier that nothing
// arrives at (no copy, no MMA, no other thread is involved), with a poll budget
// the caller chooses, then returns.
#include <cuda_runtime.h>

#include "grid_async.cuh"
#include "grid_internal.h"

namespace {

constexpr uint32_t kMaxProbeSpins = 1u << 22;  // the library's own wait budget

__global__ void wait_probe_kernel(uint32_t max_spins, int* err) {
  __shared__ uint64_t bar;
  if (threadIdx.x == 0) {
    grid::mbar_init(&bar, 1);
    grid::fence_mbar_init();
  }
  __syncwarp();
  // phase 0 never completes: the wait runs out after max_spins polls
  if (threadIdx.x == 0) grid::mbar_wait_budget(&bar, 0, max_spins, err);
  __syncwarp();
}

}  // namespace

extern "C" {

int grid_gpu_selftest_wait_timeout_dev(const grid_gpu_plan* p, uint32_t max_spins, void* stream) {
  if (!p) return GRID_ERR_NULL_POINTER;
  if (max_spins == 0 || max_spins > kMaxProbeSpins) return GRID_ERR_INVALID_PARAMETERS;
  wait_probe_kernel<<<1, 32, 0, (cudaStream_t)stream>>>(max_spins, p->d_err);
  return grid::cuda_status(cudaGetLastError());
}

}  // extern "C"
