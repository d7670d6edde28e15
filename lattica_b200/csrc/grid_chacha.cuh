// ChaCha20 block function (RFC 8439) for device code: the JL keystream
// (IETF ChaCha20, nonce = part index) and the CRS sampler's ChaCha20Rng
// (64-bit block counter in words 12-13, stream 0 in words 14-15, which is the
// same block with the counter's high word in the nonce slot).
#pragma once
#include <stdint.h>

namespace grid {
namespace chacha {

struct ChachaKey {
  uint32_t k[8];
};

__device__ __forceinline__ uint32_t rotl(uint32_t x, int r) { return __funnelshift_l(x, x, r); }

// a + b as an integer multiply-add by a multiplier the compiler cannot fold
// (a constant-bank word equal to 1): it issues on the FMA pipe, not the ALU
// pipe that carries the XORs and rotations.
static __constant__ uint32_t kChachaOne = 1;
__device__ __forceinline__ uint32_t add_on_fma(uint32_t a, uint32_t b) {
  uint32_t r;
  asm("mad.lo.u32 %0, %1, %2, %3;" : "=r"(r) : "r"(b), "r"(kChachaOne), "r"(a));
  return r;
}

// One quarter round. FMA_ADDS of its four additions (0, 2 or 4) go to the FMA
// pipe: a kernel whose FMA pipe is idle balances its two integer pipes.
template <int FMA_ADDS>
__device__ __forceinline__ void quarter_round(uint32_t& a, uint32_t& b, uint32_t& c, uint32_t& d) {
  a = FMA_ADDS >= 2 ? add_on_fma(a, b) : a + b;
  d ^= a;
  d = rotl(d, 16);
  c = FMA_ADDS >= 4 ? add_on_fma(c, d) : c + d;
  b ^= c;
  b = rotl(b, 12);
  a = FMA_ADDS >= 2 ? add_on_fma(a, b) : a + b;
  d ^= a;
  d = rotl(d, 8);
  c = FMA_ADDS >= 4 ? add_on_fma(c, d) : c + d;
  b ^= c;
  b = rotl(b, 7);
}

// RFC 8439 block function: out[16] = keystream words of block `counter`.
template <int FMA_ADDS = 0>
__device__ __forceinline__ void chacha20_block(const ChachaKey& key, uint32_t counter,
                                               uint32_t nonce0, uint32_t (&out)[16]) {
  uint32_t x0 = 0x61707865u, x1 = 0x3320646eu, x2 = 0x79622d32u, x3 = 0x6b206574u;
  uint32_t x4 = key.k[0], x5 = key.k[1], x6 = key.k[2], x7 = key.k[3];
  uint32_t x8 = key.k[4], x9 = key.k[5], x10 = key.k[6], x11 = key.k[7];
  uint32_t x12 = counter, x13 = nonce0, x14 = 0, x15 = 0;
#pragma unroll
  for (int i = 0; i < 10; ++i) {
    quarter_round<FMA_ADDS>(x0, x4, x8, x12);
    quarter_round<FMA_ADDS>(x1, x5, x9, x13);
    quarter_round<FMA_ADDS>(x2, x6, x10, x14);
    quarter_round<FMA_ADDS>(x3, x7, x11, x15);
    quarter_round<FMA_ADDS>(x0, x5, x10, x15);
    quarter_round<FMA_ADDS>(x1, x6, x11, x12);
    quarter_round<FMA_ADDS>(x2, x7, x8, x13);
    quarter_round<FMA_ADDS>(x3, x4, x9, x14);
  }
  out[0] = x0 + 0x61707865u; out[1] = x1 + 0x3320646eu;
  out[2] = x2 + 0x79622d32u; out[3] = x3 + 0x6b206574u;
  out[4] = x4 + key.k[0]; out[5] = x5 + key.k[1]; out[6] = x6 + key.k[2]; out[7] = x7 + key.k[3];
  out[8] = x8 + key.k[4]; out[9] = x9 + key.k[5]; out[10] = x10 + key.k[6];
  out[11] = x11 + key.k[7];
  out[12] = x12 + counter; out[13] = x13 + nonce0; out[14] = x14; out[15] = x15;
}

}  // namespace chacha
}  // namespace grid
