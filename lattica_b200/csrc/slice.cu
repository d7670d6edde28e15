// Elementwise slice hooks of Ring for PrimeField<Q, u32> words
// (algebra/src/arith/prime.rs:433-491, over the simd/montgomery.rs kernels):
//   add_assign_slice         dst += src
//   sub_assign_slice         dst -= src
//   scalar_mul_slice         dst *= scalar
//   add_assign_scaled_slice  dst += src * scalar
//   dot_product              sum_i lhs_i * rhs_i
// Words are canonical Montgomery words; products are Montgomery products
// (a * b * 2^-32 mod q), the reference's field multiplication. Every kernel is
// a grid-stride loop over 16-byte vectors when the buffers allow it (HBM-bound),
// with a scalar tail.
#include <cuda_runtime.h>

#include "grid_field.cuh"
#include "grid_internal.h"

using namespace grid;

namespace {

enum SliceOp : int { OP_ADD = 0, OP_SUB = 1, OP_SCALE = 2, OP_ADD_SCALED = 3 };

template <int OP>
__device__ __forceinline__ uint32_t apply(uint32_t d, uint32_t s, uint32_t c, const FieldParams& f) {
  if (OP == OP_ADD) return add_mod(d, s, f.q);
  if (OP == OP_SUB) return sub_mod(d, s, f.q);
  if (OP == OP_SCALE) return mont_mul(d, c, f.q, f.qinv);
  return add_mod(d, mont_mul(s, c, f.q, f.qinv), f.q);
}

template <int OP>
__global__ void slice_kernel(uint32_t* __restrict__ dst, const uint32_t* __restrict__ src,
                             uint32_t c, size_t n, bool vec, FieldParams f) {
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  size_t i0 = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  size_t head = 0;
  if (vec) {
    const size_t nv = n / 4;
    uint4* d4 = reinterpret_cast<uint4*>(dst);
    const uint4* s4 = reinterpret_cast<const uint4*>(src);
    for (size_t i = i0; i < nv; i += stride) {
      uint4 d = d4[i];
      const uint4 s = OP == OP_SCALE ? make_uint4(0, 0, 0, 0) : s4[i];
      d.x = apply<OP>(d.x, s.x, c, f);
      d.y = apply<OP>(d.y, s.y, c, f);
      d.z = apply<OP>(d.z, s.z, c, f);
      d.w = apply<OP>(d.w, s.w, c, f);
      d4[i] = d;
    }
    head = nv * 4;
  }
  for (size_t i = head + i0; i < n; i += stride)
    dst[i] = apply<OP>(dst[i], OP == OP_SCALE ? 0u : src[i], c, f);
}

// One CTA: sum of Montgomery products, 96-bit exact per thread, then a
// modular tree over the CTA. Dot products on this path are short (a row of a
// ring matrix); long contractions use the evaluation-domain product kernels.
constexpr int kDotThreads = 1024;

__global__ void __launch_bounds__(kDotThreads)
    dot_kernel(const uint32_t* __restrict__ lhs, const uint32_t* __restrict__ rhs, size_t n,
               uint32_t* __restrict__ out, FieldParams f) {
  __shared__ uint32_t part[kDotThreads];
  Acc96 acc;
  acc96_zero(acc);
  for (size_t i = threadIdx.x; i < n; i += kDotThreads) acc96_mad(acc, lhs[i], rhs[i]);
  part[threadIdx.x] = acc96_reduce(acc, f);
  __syncthreads();
  for (int w = kDotThreads / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) part[threadIdx.x] = add_mod(part[threadIdx.x], part[threadIdx.x + w], f.q);
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = part[0];
}

// PrimeField<Q, u64> words (value * 2^64 mod q, the reference's default limb,
// algebra/src/arith/prime.rs:24-29) <-> the u32 words of this library
// (value * 2^32 mod q): one Montgomery product by 1, or by 2^64 mod q.
__global__ void from_u64_kernel(const uint64_t* __restrict__ in, size_t n,
                                uint32_t* __restrict__ out, int* __restrict__ bad, FieldParams f) {
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const uint64_t w = in[i];
    if (bad && w >= f.q) atomicExch(bad, 1);  // not a canonical word: its output is meaningless
    out[i] = mont_mul((uint32_t)w, 1u, f.q, f.qinv);
  }
}

__global__ void to_u64_kernel(const uint32_t* __restrict__ in, size_t n,
                              uint64_t* __restrict__ out, FieldParams f) {
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
    out[i] = mont_mul(in[i], f.r2, f.q, f.qinv);
}

template <int OP>
int launch_slice(const grid_gpu_plan* p, uint32_t* dst, const uint32_t* src, uint32_t c,
                 size_t n, cudaStream_t s) {
  if (n == 0) return GRID_OK;
  const bool vec = ((uintptr_t)dst & 15u) == 0 && (OP == OP_SCALE || ((uintptr_t)src & 15u) == 0);
  const int threads = 256;
  const size_t units = vec ? (n + 3) / 4 : n;
  size_t blocks = (units + threads - 1) / threads;
  const size_t cap = (size_t)p->num_sms * 8;
  if (blocks > cap) blocks = cap;
  slice_kernel<OP><<<(unsigned)blocks, threads, 0, s>>>(dst, src, c, n, vec, p->f);
  return cuda_status(cudaGetLastError());
}

bool words_ok(size_t n) { return n < ((size_t)1 << 40); }

}  // namespace

extern "C" {

int grid_gpu_add_assign_dev(const grid_gpu_plan* p, uint32_t* dst, const uint32_t* src,
                            size_t nwords, void* stream) {
  if (!p || ((!dst || !src) && nwords)) return GRID_ERR_NULL_POINTER;
  if (!words_ok(nwords)) return GRID_ERR_INVALID_PARAMETERS;
  return launch_slice<OP_ADD>(p, dst, src, 0, nwords, (cudaStream_t)stream);
}

int grid_gpu_sub_assign_dev(const grid_gpu_plan* p, uint32_t* dst, const uint32_t* src,
                            size_t nwords, void* stream) {
  if (!p || ((!dst || !src) && nwords)) return GRID_ERR_NULL_POINTER;
  if (!words_ok(nwords)) return GRID_ERR_INVALID_PARAMETERS;
  return launch_slice<OP_SUB>(p, dst, src, 0, nwords, (cudaStream_t)stream);
}

int grid_gpu_scalar_mul_dev(const grid_gpu_plan* p, uint32_t* dst, uint32_t scalar,
                            size_t nwords, void* stream) {
  if (!p || (!dst && nwords)) return GRID_ERR_NULL_POINTER;
  if (!words_ok(nwords) || scalar >= p->f.q) return GRID_ERR_INVALID_PARAMETERS;
  return launch_slice<OP_SCALE>(p, dst, nullptr, scalar, nwords, (cudaStream_t)stream);
}

int grid_gpu_add_assign_scaled_dev(const grid_gpu_plan* p, uint32_t* dst, const uint32_t* src,
                                   uint32_t scalar, size_t nwords, void* stream) {
  if (!p || ((!dst || !src) && nwords)) return GRID_ERR_NULL_POINTER;
  if (!words_ok(nwords) || scalar >= p->f.q) return GRID_ERR_INVALID_PARAMETERS;
  return launch_slice<OP_ADD_SCALED>(p, dst, src, scalar, nwords, (cudaStream_t)stream);
}

int grid_gpu_dot_product_dev(const grid_gpu_plan* p, const uint32_t* lhs, const uint32_t* rhs,
                             size_t nwords, uint32_t* out, void* stream) {
  if (!p || !out || ((!lhs || !rhs) && nwords)) return GRID_ERR_NULL_POINTER;
  // each thread's 96-bit accumulator holds at most 2^32 products
  if (nwords > (size_t)kDotThreads << 32) return GRID_ERR_INVALID_PARAMETERS;
  dot_kernel<<<1, kDotThreads, 0, (cudaStream_t)stream>>>(lhs, rhs, nwords, out, p->f);
  return cuda_status(cudaGetLastError());
}

int grid_gpu_words_from_u64_dev(const grid_gpu_plan* p, const uint64_t* in, size_t nwords,
                                uint32_t* out, int* noncanonical, void* stream) {
  if (!p || ((!in || !out) && nwords)) return GRID_ERR_NULL_POINTER;
  if (!words_ok(nwords)) return GRID_ERR_INVALID_PARAMETERS;
  if (nwords == 0) return GRID_OK;
  if (noncanonical) {
    const cudaError_t e = cudaMemsetAsync(noncanonical, 0, sizeof(int), (cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_status(e);
  }
  size_t blocks = (nwords + 255) / 256;
  const size_t cap = (size_t)p->num_sms * 8;
  if (blocks > cap) blocks = cap;
  from_u64_kernel<<<(unsigned)blocks, 256, 0, (cudaStream_t)stream>>>(
      in, nwords, out, noncanonical, p->f);
  return cuda_status(cudaGetLastError());
}

int grid_gpu_words_to_u64_dev(const grid_gpu_plan* p, const uint32_t* in, size_t nwords,
                              uint64_t* out, void* stream) {
  if (!p || ((!in || !out) && nwords)) return GRID_ERR_NULL_POINTER;
  if (!words_ok(nwords)) return GRID_ERR_INVALID_PARAMETERS;
  if (nwords == 0) return GRID_OK;
  size_t blocks = (nwords + 255) / 256;
  const size_t cap = (size_t)p->num_sms * 8;
  if (blocks > cap) blocks = cap;
  to_u64_kernel<<<(unsigned)blocks, 256, 0, (cudaStream_t)stream>>>(in, nwords, out, p->f);
  return cuda_status(cudaGetLastError());
}

}  // extern "C"
