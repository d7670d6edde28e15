// Gram matrix entry point that allocates nothing.
//
// Some callers cannot allocate device memory: a prover loop with a latency
// budget (cudaMalloc / cudaFree synchronise the device and stall every stream
// in flight), or a plugin embedded in a host runtime that owns the device
// memory pool and forbids allocations behind its back. grid_gpu_gram_dev
// already takes its scratch from the caller; this variant takes it from a
// fixed buffer compiled into the library instead, so the caller passes only
// inputs and outputs.
//
// The buffer is a file-scope __device__ array of kNoAllocScratchBytes. Every
// GPU that loads the library holds it until the process exits. All calls
// share it and it keeps the last call's contents; nothing in it needs to start
// at zero (each word the Gram path reads was written earlier in the same call).
// Two calls whose work overlaps on the GPU — different streams, or different
// host threads — race on it; callers must order them (e.g. one stream).
#include <cuda_runtime.h>

#include <mutex>

#include "grid_internal.h"

namespace {

constexpr size_t kNoAllocScratchBytes = 48ull << 20;  // 48 MiB

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// Device address of the buffer, looked up once per device. In host code the
// array's name is only a host-side stand-in, so the address must come from
// cudaGetSymbolAddress with that device current. The cached address lives as
// long as the process's context on that device: like every plan and matrix of
// this library, it does not survive cudaDeviceReset.
std::mutex g_setup_mu;
void* g_scratch_addr[grid::kMaxDevices] = {};

int scratch_for_device(int device, void** out) {
  if (device < 0 || device >= grid::kMaxDevices) return GRID_ERR_INVALID_PARAMETERS;
  std::lock_guard<std::mutex> lk(g_setup_mu);
  if (!g_scratch_addr[device]) {
    int prev = -1;
    cudaError_t e = cudaGetDevice(&prev);
    if (e != cudaSuccess) return grid::cuda_status(e);
    if (prev != device && (e = cudaSetDevice(device)) != cudaSuccess) return grid::cuda_status(e);
    void* ptr = nullptr;
    e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
    if (prev != device) cudaSetDevice(prev);
    if (e != cudaSuccess) return grid::cuda_status(e);
    g_scratch_addr[device] = ptr;
  }
  *out = g_scratch_addr[device];
  return GRID_OK;
}

}  // namespace

extern "C" {

size_t grid_gpu_noalloc_scratch_bytes(void) { return kNoAllocScratchBytes; }

int grid_gpu_gram_noalloc_dev(const grid_gpu_plan* plan, const uint32_t* S, size_t r, size_t n,
                              uint32_t* G, void* stream) {
  if (!plan || !S || !G) return GRID_ERR_NULL_POINTER;
  if (r == 0 || n == 0) return GRID_ERR_INVALID_PARAMETERS;
  // The witness's evaluations alone take r * n * d words of the buffer: reject
  // sizes beyond it before any product that could wrap is formed.
  const size_t max_polys = kNoAllocScratchBytes / (4 * (size_t)plan->d);
  if (r > max_polys || n > max_polys / r) return GRID_ERR_SCRATCH_LIMIT;
  size_t need = 0;
  int st = grid_gpu_gram_workspace(plan, r, n, &need);
  if (st) return st;
  if (need > kNoAllocScratchBytes) return GRID_ERR_SCRATCH_LIMIT;
  // The buffer's address is per device: the launches go to the current device,
  // which must be the plan's.
  int cur = -1;
  cudaError_t e = cudaGetDevice(&cur);
  if (e != cudaSuccess) return grid::cuda_status(e);
  if (cur != plan->device) return GRID_ERR_INVALID_PARAMETERS;
  void* scratch = nullptr;
  st = scratch_for_device(plan->device, &scratch);
  if (st) return st;
  return grid_gpu_gram_dev(plan, S, r, n, G, scratch, kNoAllocScratchBytes, stream);
}

}  // extern "C"
