// Device-side arithmetic in Z_q for PrimeField<Q, u32> Montgomery words
// (value * 2^32 mod q, canonical in [0, q)), q an odd prime < 2^32.
//
// Reference semantics: algebra/src/arith/prime.rs:110-183 (add_raw_words,
// sub_raw_words, montgomery_reduce_wide). The GPU uses the "positive inverse"
// form of Montgomery reduction, (a*b - m*q) / 2^32 with m = lo(a*b) * q^-1,
// which yields the same canonical residue a*b*2^-32 mod q as the reference's
// (a*b + m*q) / 2^32 with m = lo(a*b) * (-q^-1), without a 33-bit carry.
#pragma once
#include <stdint.h>

namespace grid {

struct FieldParams {
  uint32_t q;     // modulus
  uint32_t qinv;  // q^-1 mod 2^32 (positive inverse)
  uint32_t r1;    // 2^32 mod q  (Montgomery one)
  uint32_t r2;    // 2^64 mod q  (to-Montgomery factor)
};

// a*b*2^-32 mod q. Canonical output whenever min(a, b) < q.
__device__ __forceinline__ uint32_t mont_mul(uint32_t a, uint32_t b, uint32_t q, uint32_t qinv) {
  const uint32_t lo = a * b;
  const uint32_t hi = __umulhi(a, b);
  const uint32_t m = lo * qinv;
  const uint32_t u = __umulhi(m, q);
  const uint32_t r = hi - u;
  return hi < u ? r + q : r;
}

// Multiply by a fixed constant w < q with precomputed wq = w * q^-1 mod 2^32
// (saves the low product: m = a*w*q^-1 = a*wq mod 2^32).
__device__ __forceinline__ uint32_t mont_mul_c(uint32_t a, uint32_t w, uint32_t wq, uint32_t q) {
  const uint32_t hi = __umulhi(a, w);
  const uint32_t m = a * wq;
  const uint32_t u = __umulhi(m, q);
  const uint32_t r = hi - u;
  return hi < u ? r + q : r;
}

// (a + b) mod q for canonical a, b (works for q up to 2^32 - 1: computes
// a - (q - b) and adds q back on borrow).
__device__ __forceinline__ uint32_t add_mod(uint32_t a, uint32_t b, uint32_t q) {
  const uint32_t nb = q - b;
  const uint32_t r = a - nb;
  return a < nb ? r + q : r;
}

__device__ __forceinline__ uint32_t sub_mod(uint32_t a, uint32_t b, uint32_t q) {
  const uint32_t r = a - b;
  return a < b ? r + q : r;
}

// ---------------------------------------------------------------------------
// Lazy words: any 32-bit word congruent to the value mod q. r1 = 2^32 mod q.
//
// Carries and borrows are taken from unsigned compares. (Taking the borrow
// from the high word of a 64-bit difference, or from a sub.cc / subc pair,
// was measured on sm_100a to report a borrow for 0 - 0 when fed by __umulhi
// results inside the unrolled transforms, so those forms are not used.)
// ---------------------------------------------------------------------------

// a - t (mod q) for t < q and any word a; result in [0, 2^32).
// Borrow: a - t + 2^32 + q wraps to a - t + q, which lies in (0, q).
__device__ __forceinline__ uint32_t sub_lazy(uint32_t a, uint32_t t, uint32_t q) {
  const uint32_t r = a - t;
  return a < t ? r + q : r;
}

// a + t (mod q) for t < q and any word a; result in [0, 2^32).
// Carry: a + t - 2^32 <= q - 2, plus r1 < q stays below 2^32 for every q < 2^32.
__device__ __forceinline__ uint32_t add_lazy(uint32_t a, uint32_t t, uint32_t r1) {
  const uint32_t s = a + t;
  return s < t ? s + r1 : s;
}

// (a + b) mod q, canonical, for canonical a, b: a - (q - b), + q on borrow.
__device__ __forceinline__ uint32_t add_canon(uint32_t a, uint32_t b, uint32_t q) {
  return sub_lazy(a, q - b, q);
}

// Montgomery product by a constant w < q (Shoup companion wq): canonical for any word a.
__device__ __forceinline__ uint32_t mont_c(uint32_t a, uint32_t w, uint32_t wq, uint32_t q) {
  const uint32_t hi = __umulhi(a, w);
  const uint32_t m = a * wq;
  const uint32_t u = __umulhi(m, q);
  return sub_lazy(hi, u, q);
}

// Montgomery product a*b*2^-32 for any word a and canonical b: canonical.
__device__ __forceinline__ uint32_t mont_v(uint32_t a, uint32_t b, uint32_t q, uint32_t qinv) {
  const uint32_t lo = a * b;
  const uint32_t hi = __umulhi(a, b);
  const uint32_t m = lo * qinv;
  const uint32_t u = __umulhi(m, q);
  return sub_lazy(hi, u, q);
}

// Any 32-bit word x -> x mod q, by one Montgomery multiply with 2^32 mod q.
__device__ __forceinline__ uint32_t reduce_word(uint32_t x, const FieldParams& f) {
  return mont_mul(x, f.r1, f.q, f.qinv);
}

// Montgomery word -> canonical integer value.
__device__ __forceinline__ uint32_t from_mont(uint32_t x, const FieldParams& f) {
  return mont_mul(x, 1u, f.q, f.qinv);
}

// Canonical integer v < q -> Montgomery word.
__device__ __forceinline__ uint32_t to_mont(uint32_t v, const FieldParams& f) {
  return mont_mul(v, f.r2, f.q, f.qinv);
}

// 96-bit accumulator for sums of 64-bit products: acc += a*b.
struct Acc96 {
  uint32_t w0, w1, w2;  // bits 0..31, 32..63, 64..95
};

__device__ __forceinline__ void acc96_zero(Acc96& a) {
  a.w0 = 0;
  a.w1 = 0;
  a.w2 = 0;
}

// One carry chain: w0 += lo(a*b), w1 += hi(a*b) + carry, w2 += carry.
__device__ __forceinline__ void acc96_mad(Acc96& acc, uint32_t a, uint32_t b) {
  asm("mad.lo.cc.u32 %0, %3, %4, %0;\n\t"
      "madc.hi.cc.u32 %1, %3, %4, %1;\n\t"
      "addc.u32 %2, %2, 0;"
      : "+r"(acc.w0), "+r"(acc.w1), "+r"(acc.w2)
      : "r"(a), "r"(b));
}

// Reduce V = w2*2^64 + w1*2^32 + w0 to V * 2^-32 mod q (canonical).
// This is the Montgomery-domain sum of the accumulated products:
// sum(a_k*b_k) * 2^-32 = sum(mont_mul(a_k, b_k)) mod q.
// Requires w2 < 2^32 (at most 2^32 products of words < 2^32).
__device__ __forceinline__ uint32_t acc96_reduce(const Acc96& acc, const FieldParams& f) {
  const uint32_t w0 = acc.w0, w1 = acc.w1;
  // Low 64 bits: (w1*2^32 + w0) * 2^-32 = w1 - hi(m*q) with m = w0*q^-1.
  const uint32_t m = w0 * f.qinv;
  const uint32_t u = __umulhi(m, f.q);
  uint32_t lo_part = w1 - u;     // in (-q, 2^32): fix the negative case
  if (w1 < u) lo_part += f.q;    // now any word in [0, 2^32)
  lo_part = reduce_word(lo_part, f);  // canonical
  // High word: w2 * 2^64 * 2^-32 = w2 * 2^32 = mont_mul(w2, 2^64 mod q).
  const uint32_t hi_part = mont_mul(acc.w2, f.r2, f.q, f.qinv);
  return add_mod(lo_part, hi_part, f.q);
}

}  // namespace grid
