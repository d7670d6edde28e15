// Ring products for moduli without a 2d-th root of unity.
//
// The reference multiplies in R_q = Z_q[X]/(X^d + 1) through the twisted NTT
// when q has a primitive 2d-th root of unity and by the schoolbook rule
// otherwise (NegacyclicMulRing::negacyclic_mul_coeffs falling back to
// naive_negacyclic_mul_coeffs, algebra/src/poly/ring.rs:60-100). Its own
// LaBRADOR moduli, 2^32 - 5 and 12281, have no 128th root, so every ring
// product on its prover path takes the schoolbook branch. A ring product is a
// field computation, so any exact method yields the same canonical words.
//
// A ring plan for such a q computes every contraction (commitments, Gram,
// garbage h, amortization, single products) exactly over the integers:
//  * input words x < q are lifted to residues modulo three auxiliary primes
//    p_j = 1 (mod 512) just below 2^32 (x mod p_j is one conditional
//    subtraction, since p_j > 2^31);
//  * each residue problem runs on the NTT kernels of an ordinary plan for p_j,
//    with the lifted words read as Montgomery words: its output words are
//    w_j = V * 2^-32 mod p_j, where V is the exact integer sum of the word
//    products with the negacyclic signs;
//  * Garner's mixed-radix reconstruction x1 + p0 x2 + p0 p1 x3 recovers V in
//    (-P/2, P/2), P = p0 p1 p2 > 2^95, whenever |V| < 2^93 (the callers bound
//    terms * d * (q - 1)^2 below 2^93); the sign is read from x3, which then
//    lies below p2/2 exactly when V >= 0;
//  * the output word is V * 2^-32 mod q: the Montgomery word of the sum of the
//    word products, the same word as the reference's schoolbook sum of
//    Montgomery products.
#include <cuda_runtime.h>

#include <new>

#include "grid_field.cuh"
#include "grid_internal.h"

namespace grid {
namespace {

// The three largest primes below 2^32 that are 1 mod 512 (NTTs up to 512
// points, so every compiled degree d <= 256 has its 2d-th root).
constexpr uint32_t kAux[3] = {4294962689u, 4294957057u, 4294955009u};

uint64_t mulmod(uint64_t a, uint64_t b, uint64_t m) {
  return (uint64_t)((unsigned __int128)a * b % m);
}

uint64_t powmod(uint64_t b, uint64_t e, uint64_t m) {
  uint64_t r = 1 % m;
  b %= m;
  while (e) {
    if (e & 1) r = mulmod(r, b, m);
    b = mulmod(b, b, m);
    e >>= 1;
  }
  return r;
}

uint64_t invmod(uint64_t a, uint64_t p) { return powmod(a, p - 2, p); }  // p prime

uint32_t neg_inv32(uint32_t q) {  // q^-1 mod 2^32 (positive inverse, grid_field.cuh)
  uint32_t x = 1;
  for (int i = 0; i < 5; ++i) x *= 2u - q * x;
  return x;
}

__global__ void crt_lift_kernel(const uint4* __restrict__ x, size_t n4, uint4* __restrict__ o0,
                                uint4* __restrict__ o1, uint4* __restrict__ o2, uint3 p) {
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n4; i += stride) {
    const uint4 v = x[i];
    auto lift = [](uint4 w, uint32_t m) {
      return make_uint4(w.x >= m ? w.x - m : w.x, w.y >= m ? w.y - m : w.y,
                        w.z >= m ? w.z - m : w.z, w.w >= m ? w.w - m : w.w);
    };
    if (o0) o0[i] = lift(v, p.x);
    if (o1) o1[i] = lift(v, p.y);
    if (o2) o2[i] = lift(v, p.z);
  }
}

__device__ __forceinline__ uint32_t crt_word(uint32_t w0, uint32_t w1, uint32_t w2,
                                             const CrtConsts& c) {
  const uint32_t p0 = c.p[0], p1 = c.p[1], p2 = c.p[2];
  // x1 = V mod p0 = w0 * 2^32 mod p0
  const uint32_t x1 = mont_mul(w0, c.r2_0, p0, c.pinv[0]);
  // x2 = (V - x1) p0^-1 mod p1
  const uint32_t x2 = sub_mod(mont_mul(w1, c.c1a, p1, c.pinv[1]),
                              mont_mul(x1, c.c1b, p1, c.pinv[1]), p1);
  // x3 = ((V - x1) p0^-1 - x2) p1^-1 mod p2
  const uint32_t t3 = sub_mod(mont_mul(w2, c.c2a, p2, c.pinv[2]),
                              mont_mul(x1, c.c2b, p2, c.pinv[2]), p2);
  const uint32_t x3 = sub_mod(t3, mont_mul(x2, c.c2c, p2, c.pinv[2]), p2);
  // V * 2^-32 mod q = (x1 + p0 x2 + p0 p1 x3 [- P]) * 2^-32
  const FieldParams& f = c.fq;
  uint32_t r = add_mod(mont_mul(x1, 1u, f.q, f.qinv), mont_mul(x2, c.m1, f.q, f.qinv), f.q);
  r = add_mod(r, mont_mul(x3, c.m2, f.q, f.qinv), f.q);
  return x3 > c.half_p2 ? sub_mod(r, c.p_rinv, f.q) : r;
}

__global__ void crt_combine_kernel(const uint4* __restrict__ w0, const uint4* __restrict__ w1,
                                   const uint4* __restrict__ w2, size_t n4,
                                   uint4* __restrict__ out, CrtConsts c) {
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n4; i += stride) {
    const uint4 a = w0[i], b = w1[i], e = w2[i];
    out[i] = make_uint4(crt_word(a.x, b.x, e.x, c), crt_word(a.y, b.y, e.y, c),
                        crt_word(a.z, b.z, e.z, c), crt_word(a.w, b.w, e.w, c));
  }
}

unsigned grid_for(const grid_gpu_plan* p, size_t n4) {
  size_t blocks = (n4 + 255) / 256;
  const size_t cap = (size_t)(p->num_sms > 0 ? p->num_sms : 1) * 8;
  if (blocks > cap) blocks = cap;
  return (unsigned)(blocks ? blocks : 1);
}

}  // namespace

const uint32_t* crt_moduli() { return kAux; }

void crt_consts(uint32_t q, CrtConsts* c) {
  const uint64_t p0 = kAux[0], p1 = kAux[1], p2 = kAux[2];
  const uint64_t R = (1ull << 32);
  for (int j = 0; j < 3; ++j) {
    c->p[j] = kAux[j];
    c->pinv[j] = neg_inv32(kAux[j]);
  }
  c->r2_0 = (uint32_t)mulmod(R % p0, R % p0, p0);
  const uint64_t i0 = invmod(p0 % p1, p1);
  c->c1a = (uint32_t)mulmod(mulmod(R % p1, R % p1, p1), i0, p1);
  c->c1b = (uint32_t)mulmod(R % p1, i0, p1);
  const uint64_t i01 = invmod(mulmod(p0 % p2, p1 % p2, p2), p2);
  const uint64_t i1 = invmod(p1 % p2, p2);
  c->c2a = (uint32_t)mulmod(mulmod(R % p2, R % p2, p2), i01, p2);
  c->c2b = (uint32_t)mulmod(R % p2, i01, p2);
  c->c2c = (uint32_t)mulmod(R % p2, i1, p2);
  c->half_p2 = (uint32_t)(p2 / 2);
  c->fq.q = q;
  c->fq.qinv = neg_inv32(q);
  c->fq.r1 = (uint32_t)(R % q);
  c->fq.r2 = (uint32_t)(((unsigned __int128)1 << 64) % q);
  c->m1 = (uint32_t)(p0 % q);
  c->m2 = (uint32_t)mulmod(p0 % q, p1 % q, q);
  const uint64_t Pq = mulmod(c->m2, p2 % q, q);
  c->p_rinv = (uint32_t)mulmod(Pq, invmod(R % q, q), q);  // P * 2^-32 mod q
}

bool crt_bound_ok(const grid_gpu_plan* p, size_t terms) {
  // terms * d * (q - 1)^2 < 2^93: V fits the reconstruction's signed range
  const unsigned __int128 q1 = p->q - 1;
  const unsigned __int128 t = (unsigned __int128)terms * p->d;
  if (terms == 0) return true;
  if (t >> 40) return false;
  return t * q1 * q1 < ((unsigned __int128)1 << 93);
}

int crt_lift(const grid_gpu_plan* p, const uint32_t* x, size_t words, uint32_t* o0, uint32_t* o1,
             uint32_t* o2, cudaStream_t s) {
  if (words == 0) return GRID_OK;
  if (words % 4) return GRID_ERR_INVALID_PARAMETERS;  // whole polynomials of d >= 8 words
  const size_t n4 = words / 4;
  crt_lift_kernel<<<grid_for(p, n4), 256, 0, s>>>(
      reinterpret_cast<const uint4*>(x), n4, reinterpret_cast<uint4*>(o0),
      reinterpret_cast<uint4*>(o1), reinterpret_cast<uint4*>(o2),
      make_uint3(kAux[0], kAux[1], kAux[2]));
  return cuda_status(cudaGetLastError());
}

int crt_combine(const grid_gpu_plan* p, const uint32_t* w0, const uint32_t* w1,
                const uint32_t* w2, size_t words, uint32_t* out, cudaStream_t s) {
  if (words == 0) return GRID_OK;
  if (words % 4) return GRID_ERR_INVALID_PARAMETERS;
  const size_t n4 = words / 4;
  crt_combine_kernel<<<grid_for(p, n4), 256, 0, s>>>(
      reinterpret_cast<const uint4*>(w0), reinterpret_cast<const uint4*>(w1),
      reinterpret_cast<const uint4*>(w2), n4, reinterpret_cast<uint4*>(out), p->crt_c);
  return cuda_status(cudaGetLastError());
}

}  // namespace grid
