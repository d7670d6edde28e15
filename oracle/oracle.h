/*
 * CPU oracle for the Gridland ring-arithmetic hot path.
 *
 * TEST INFRASTRUCTURE ONLY. This is a plain-C restatement of the reference
 * (mrain/lattica, Rust) CPU algorithms, used as the bit-exact checker for the
 * CUDA library and as the timed CPU baseline. Nothing in the product path
 * (lattica_b200/, include/) links, loads or calls it.
 *
 * Words are PrimeField<Q, u32> Montgomery words: value * 2^32 mod q, canonical
 * in [0, q).  Every function cites the reference file:line it restates.
 */
#ifndef GRID_ORACLE_H
#define GRID_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes mirror the C-ABI in include/grid_gpu.h. */
enum {
    ORC_OK = 0,
    ORC_ERR_LENGTH_MISMATCH = 1,
    ORC_ERR_LENGTH_NOT_POW2 = 2,
    ORC_ERR_UNSUPPORTED_SIZE = 3,
    ORC_ERR_UNSUPPORTED_TWIST = 4,
    ORC_ERR_INVALID_PARAMETERS = 5,
    ORC_ERR_DIMENSION_MISMATCH = 6,
    ORC_ERR_INVALID_MODULUS = 7,
    ORC_ERR_NULL = 8,
    ORC_ERR_OOM = 9
};

typedef struct {
    uint32_t q;
    uint32_t r_mod_q;   /* 2^32 mod q   (Montgomery one)   prime.rs:60-71  */
    uint32_t r2_mod_q;  /* 2^64 mod q                      prime.rs:73-78  */
    uint32_t q_inv;     /* -q^-1 mod 2^32                  prime.rs:80-91  */
} orc_field;

int orc_field_init(orc_field *f, uint64_t q);
uint32_t orc_to_mont(const orc_field *f, uint64_t v);
uint32_t orc_from_mont(const orc_field *f, uint32_t w);
uint32_t orc_add(const orc_field *f, uint32_t a, uint32_t b);
uint32_t orc_sub(const orc_field *f, uint32_t a, uint32_t b);
uint32_t orc_mul(const orc_field *f, uint32_t a, uint32_t b);
uint32_t orc_neg(const orc_field *f, uint32_t a);
uint32_t orc_pow(const orc_field *f, uint32_t base, uint64_t exp);
uint32_t orc_inv(const orc_field *f, uint32_t a);
int orc_is_prime_u64(uint64_t n);

/* Twisted negacyclic NTT plan (poly/ntt.rs:25-154 over arith/ntt.rs:397-500). */
typedef struct {
    orc_field f;
    uint32_t n;
    uint32_t generator;   /* Montgomery word of the smallest generator */
    uint32_t omega;       /* root_of_unity(n), Montgomery */
    uint32_t psi;         /* root_of_unity(2n), Montgomery */
    uint32_t inv_scale;   /* n^-1, Montgomery */
    uint32_t *fwd_tw;     /* stage twiddles, stage s has 2^s entries, concatenated */
    uint32_t *inv_tw;     /* inverse stage twiddles, stage order len = n, n/2, ..., 2 */
    uint32_t *twists;     /* psi^i */
    uint32_t *untwists;   /* psi^-i */
} orc_plan;

/* Returns ORC_OK or the NttError code the reference build would raise. */
int orc_plan_create(orc_plan *p, uint64_t q, uint64_t n);
void orc_plan_destroy(orc_plan *p);
uint64_t orc_max_ntt_size(uint64_t q);
uint32_t orc_find_generator(const orc_field *f);

/* Cyclic NTT on one length-n vector (arith/ntt.rs:207-340). */
void orc_ntt_forward(const orc_plan *p, uint32_t *v);
void orc_ntt_inverse(const orc_plan *p, uint32_t *v);
/* Twisted transforms applied to `count` consecutive polys of length n. */
void orc_twisted_forward(const orc_plan *p, uint32_t *polys, size_t count);
void orc_twisted_inverse(const orc_plan *p, uint32_t *polys, size_t count);
/* out = INTT_tw( NTT_tw(a) (.) b ) for `count` polys; b is already in the twisted domain. */
void orc_ntt_mul_inverse(const orc_plan *p, const uint32_t *a, const uint32_t *b_evals,
                         uint32_t *out, size_t count);
/* Same, split over `threads` OpenMP threads (independent polys). */
void orc_ntt_mul_inverse_mt(const orc_plan *p, const uint32_t *a, const uint32_t *b_evals,
                            uint32_t *out, size_t count, int threads);
/* The same product through the AVX2 restatement of the reference's x86 path
 * (oracle_avx2.c): identical words, for the timed CPU baseline. */
void orc_ntt_mul_inverse_avx2(const orc_plan *p, const uint32_t *a, const uint32_t *b_evals,
                              uint32_t *out, size_t count);
void orc_ntt_mul_inverse_avx2_mt(const orc_plan *p, const uint32_t *a, const uint32_t *b_evals,
                                 uint32_t *out, size_t count, int threads);
/* The prepared commitment through the same AVX2 pieces (matvec's words). */
int orc_matvec_avx2(const orc_plan *p, const uint32_t *A, size_t rows, size_t cols,
                    int a_is_eval, const uint32_t *s, size_t batch, uint32_t *t, int threads);
/* Negacyclic product via twisted NTT (poly/ntt.rs:110-126). */
void orc_poly_mul_ntt(const orc_plan *p, const uint32_t *a, const uint32_t *b, uint32_t *out);
/* Schoolbook negacyclic product (poly/ring.rs:60-77). */
void orc_naive_negacyclic(const orc_field *f, uint32_t n, const uint32_t *a, const uint32_t *b,
                          uint32_t *out);
void orc_pointwise_mul(const orc_field *f, uint32_t *dst, const uint32_t *rhs, size_t len);

/* Slice hooks of Ring for PrimeField (arith/prime.rs:433-491). */
void orc_add_assign_slice(const orc_field *f, uint32_t *dst, const uint32_t *src, size_t len);
void orc_sub_assign_slice(const orc_field *f, uint32_t *dst, const uint32_t *src, size_t len);
void orc_scalar_mul_slice(const orc_field *f, uint32_t *dst, uint32_t scalar, size_t len);
void orc_add_assign_scaled_slice(const orc_field *f, uint32_t *dst, const uint32_t *src,
                                 uint32_t scalar, size_t len);
uint32_t orc_dot_product(const orc_field *f, const uint32_t *lhs, const uint32_t *rhs, size_t len);

/* Ring contractions with schoolbook negacyclic products, for any odd prime
 * q < 2^32 (the reference's path when q has no 2d-th root, poly/ring.rs:60-100):
 * RingMat::mul_slice per witness, compute_garbage_g / compute_garbage_h, and the
 * amortized witness z[k] = sum_i c_i s_i[k]. */
int orc_ring_matvec(const orc_field *f, uint32_t d, const uint32_t *A, size_t rows, size_t cols,
                    const uint32_t *s, size_t batch, uint32_t *t, int threads);
int orc_ring_gram(const orc_field *f, uint32_t d, const uint32_t *S, size_t r, size_t n,
                  uint32_t *G, int threads);
int orc_ring_garbage_h(const orc_field *f, uint32_t d, const uint32_t *S, const uint32_t *Phi,
                       size_t r, size_t n, uint32_t *H, int threads);
int orc_ring_amortize(const orc_field *f, uint32_t d, const uint32_t *S, const uint32_t *c,
                      size_t r, size_t n, uint32_t *Z, int threads);

/* t[b][row] = sum_k A[row][k] * s[b][k] in R_q (commit/src/linear.rs:459-506,
 * poly/twisted_ntt.rs:378-408). A is coefficient-domain unless a_is_eval. */
int orc_matvec(const orc_plan *p, const uint32_t *A, size_t rows, size_t cols, int a_is_eval,
               const uint32_t *s, size_t batch, uint32_t *t);
int orc_matvec_mt(const orc_plan *p, const uint32_t *A, size_t rows, size_t cols, int a_is_eval,
                  const uint32_t *s, size_t batch, uint32_t *t, int threads);
/* Linear commitment t = A_msg*m + A_open*r (commit/src/linear.rs:476-506). */
int orc_linear_commit(const orc_plan *p, const uint32_t *a_msg, size_t rows, size_t msg_cols,
                      const uint32_t *a_open, size_t open_cols, const uint32_t *m,
                      const uint32_t *r, uint32_t *t);

/* Gram g_ij = <s_i, s_j>, i <= j, row-major upper triangle
 * (labrador/src/main_protocol/garbage.rs:76-93, mod.rs:664-670). */
int orc_gram(const orc_plan *p, const uint32_t *S, size_t r, size_t n, uint32_t *G, int threads);
int orc_garbage_h(const orc_plan *p, const uint32_t *S, const uint32_t *Phi, size_t r, size_t n,
                  uint32_t *H);
int orc_amortize(const orc_plan *p, const uint32_t *S, const uint32_t *c, size_t r, size_t n,
                 uint32_t *Z);
/* Slow faithful path: one full negacyclic product per term (poly/ring.rs:226-228). */
int orc_gram_naive(const orc_plan *p, const uint32_t *S, size_t r, size_t n, uint32_t *G);
size_t orc_garbage_index(size_t r, size_t i, size_t j);

/* Balanced decomposition (labrador/src/main_protocol/mod.rs:258-323,731-747). */
void orc_decompose_coeff_balanced(uint64_t c, uint64_t base, size_t num_limbs, uint64_t q,
                                  int64_t *limbs_out);
int64_t orc_centered_mod(int64_t v, int64_t base);
int orc_decompose_polys(const orc_field *f, uint32_t d, const uint32_t *polys, size_t npolys,
                        uint64_t base, size_t num_limbs, uint32_t *out);
int orc_reconstruct_from_limbs(const orc_field *f, uint32_t d, const uint32_t *limbs,
                               size_t num_limbs, uint64_t base, uint32_t *out);
/* Unsigned gadget decomposition (algebra/src/poly/decomposition.rs:47-61). */
size_t orc_gadget_digits(uint64_t q, uint64_t base);
int orc_gadget_decompose(const orc_field *f, const uint32_t *x, size_t len, uint64_t base,
                         uint32_t *out /* [k][len] */);

/* ChaCha20 (IETF, RFC 8439) block function: 64 output bytes. */
void orc_chacha20_block(const uint8_t key[32], uint32_t counter, const uint8_t nonce[12],
                        uint8_t out[64]);
void orc_chacha20_quarter(uint32_t *a, uint32_t *b, uint32_t *c, uint32_t *d);
/* JL projection + extraction (labrador/src/jl.rs:267-303,388-508).
 * parts: num_parts x cols words. p_out: rows words. flat_out may be NULL. */
int orc_jl_project(const orc_field *f, const uint8_t seed[32], size_t rows, size_t cols,
                   const uint32_t *parts, size_t num_parts, size_t d, uint32_t *p_out,
                   int8_t *flat_out, int threads);

/* jl_rows_flat_to_conjugated_polys + jl_evals (main_protocol/mod.rs:885-923,
 * step_prover.rs:185-206): evals[m] = sum conj(pi_{m,i,j}) * s_{i,j}. */
int orc_jl_evals(const orc_plan *p, const int8_t *flat, size_t rows, const uint32_t *parts,
                 size_t num_parts, size_t n, uint32_t *evals);

/* Uniform ring elements from ChaCha20Rng(seed), CommitKey::from_seed order
 * (labrador/src/crs.rs:136-198, 308-326; prime.rs:730-743). */
int orc_sample_uniform_polys(const orc_field *f, const uint8_t seed[32], size_t npolys,
                             uint32_t d, uint64_t accept_max, uint32_t *out);

#ifdef __cplusplus
}
#endif
#endif
