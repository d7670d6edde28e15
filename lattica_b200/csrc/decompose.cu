// Digit decompositions of R_q coefficients.
//
// Balanced (centered) base-b limbs: decompose_coeff_balanced / centered_mod /
// decompose_poly_balanced / decompose_polys
// (labrador/src/main_protocol/mod.rs:258-323, 731-747): the canonical
// coefficient is centered into (-q/2, q/2], then limb = centered_mod(carry, b)
// in [-b/2, b/2] and carry = (carry - limb) / b, num_limbs times (a carry left
// after the last limb is dropped, as in the reference). Limb v is stored as the
// Montgomery word of v mod q. Output layout [poly][limb][coeff].
//
// Unsigned gadget digits: gadget_decompose / GadgetRing::decompose_element
// (algebra/src/poly/decomposition.rs:47-61, commit/src/gadget/mod.rs:151-162):
// digit = value % base, value /= base, k = #digits(q - 1) times.
#include <cuda_runtime.h>

#include "grid_field.cuh"
#include "grid_internal.h"

namespace grid {
namespace {

__device__ __forceinline__ long long centered_mod(long long v, long long base) {
  const long long half = base / 2;
  const long long r = v % base;  // truncating, like Rust's %
  if (r > half) return r - base;
  if (r < -half) return r + base;
  return r;
}

__global__ void balanced_kernel(const uint32_t* __restrict__ in, size_t npolys, int d,
                                long long base, int num_limbs, uint32_t* __restrict__ out,
                                FieldParams f) {
  const size_t total = npolys * (size_t)d;
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  const long long q = f.q;
  const long long half_q = q / 2;
  for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total; idx += stride) {
    const size_t poly = idx / d;
    const int i = (int)(idx % d);
    long long carry = (long long)from_mont(in[idx], f);
    if (carry > half_q) carry -= q;
    uint32_t* dst = out + poly * (size_t)num_limbs * d + i;
    for (int k = 0; k < num_limbs; ++k) {
      const long long limb = centered_mod(carry, base);
      const long long u = limb >= 0 ? limb : q + limb;  // q - |limb|
      dst[(size_t)k * d] = to_mont((uint32_t)(u % q), f);
      carry = (carry - limb) / base;
    }
  }
}

// digit_major = 1: out[digit][len] (gadget_decompose); 0: out[poly][digit][coeff]
// (decompose_element per polynomial, concatenated).
__global__ void gadget_kernel(const uint32_t* __restrict__ in, size_t len, int d,
                              unsigned long long base, int digits, int digit_major,
                              uint32_t* __restrict__ out, FieldParams f) {
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < len; idx += stride) {
    unsigned long long v = from_mont(in[idx], f);
    for (int k = 0; k < digits; ++k) {
      const uint32_t digit = (uint32_t)((v % base) % f.q);
      v /= base;
      const size_t o = digit_major ? (size_t)k * len + idx
                                   : ((idx / d) * (size_t)digits + k) * d + (idx % d);
      out[o] = to_mont(digit, f);
    }
  }
}

unsigned blocks_for(size_t n, int num_sms) {
  size_t b = (n + 255) / 256;
  const size_t cap = (size_t)num_sms * 16;
  if (b > cap) b = cap;
  return (unsigned)(b < 1 ? 1 : b);
}

}  // namespace

int launch_decompose_balanced(const grid_gpu_plan* p, const uint32_t* polys, size_t npolys,
                              uint64_t base, size_t num_limbs, uint32_t* out, cudaStream_t s) {
  if (base < 2 || base > (1ull << 32) || num_limbs == 0 || num_limbs > 64)
    return GRID_ERR_INVALID_PARAMETERS;
  if (npolys == 0) return GRID_OK;
  balanced_kernel<<<blocks_for(npolys * p->d, p->num_sms), 256, 0, s>>>(
      polys, npolys, (int)p->d, (long long)base, (int)num_limbs, out, p->f);
  return cuda_status(cudaGetLastError());
}

int launch_gadget_decompose(const grid_gpu_plan* p, const uint32_t* x, size_t len, uint64_t base,
                            size_t digits, int digit_major, uint32_t* out, cudaStream_t s) {
  if (base < 2 || digits == 0) return GRID_ERR_INVALID_PARAMETERS;
  if (len == 0) return GRID_OK;
  gadget_kernel<<<blocks_for(len, p->num_sms), 256, 0, s>>>(x, len, (int)p->d, base, (int)digits,
                                                             digit_major, out, p->f);
  return cuda_status(cudaGetLastError());
}

size_t gadget_digit_count(uint64_t q, uint64_t base) {
  uint64_t m = q - 1;
  size_t digits = 0;
  while (m > 0) {
    ++digits;
    m /= base;
  }
  return digits ? digits : 1;
}

}  // namespace grid
