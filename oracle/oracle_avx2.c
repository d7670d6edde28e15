/* AVX2 restatement of the reference's u32 Montgomery NTT path, for the timed
 * CPU baseline (test infrastructure; the library never loads it).
 *
 * The reference's x86 backend (algebra/src/simd/montgomery.rs:636-890) runs
 * the same plan as the scalar path: bit reversal, then per stage the
 * butterflies of each block, eight at a time with AVX2 when the block's half
 * length is at least 8 and one at a time below that (the scalar tail of
 * butterfly_{forward,inverse}_prime_montgomery_u32, avx2/u32_arith.rs:212-315);
 * pointwise products (twist, the config-1 multiply, untwist) run eight lanes
 * at a time (mul_assign_prime_montgomery_u32_avx2, u32_arith.rs:101-120).
 * Here each lane follows the scalar word rules of oracle.c exactly:
 * mont_reduce (prime.rs:141-183, including the carry case for q >= 2^31),
 * add_raw_words and sub_raw_words (prime.rs:110-137). The products are formed
 * on 64-bit half-lanes (even lanes, then the odd lanes shifted down), so every
 * output word equals the scalar oracle's (checked in tests/test_oracle_avx2.py). */
#include <immintrin.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "oracle.h"

typedef struct {
    __m256i q32, qm1_32, bias32;   /* q, q - 1, 2^31 in 32-bit lanes */
    __m256i q64, qm1_64, qinv64;   /* q, q - 1, -q^-1 in 64-bit lanes */
    __m256i bias64, two32;         /* 2^63, 2^32 in 64-bit lanes */
} vfield;

static vfield vfield_of(const orc_field *f) {
    vfield v;
    v.q32 = _mm256_set1_epi32((int)f->q);
    v.qm1_32 = _mm256_set1_epi32((int)(f->q - 1));
    v.bias32 = _mm256_set1_epi32((int)0x80000000u);
    v.q64 = _mm256_set1_epi64x((long long)f->q);
    v.qm1_64 = _mm256_set1_epi64x((long long)f->q - 1);
    v.qinv64 = _mm256_set1_epi64x((long long)f->q_inv);
    v.bias64 = _mm256_set1_epi64x((long long)0x8000000000000000ull);
    v.two32 = _mm256_set1_epi64x(1ll << 32);
    return v;
}

/* unsigned a > b on 32-bit lanes: all-ones where true */
static inline __m256i gt_u32(const vfield *v, __m256i a, __m256i b) {
    return _mm256_cmpgt_epi32(_mm256_xor_si256(a, v->bias32), _mm256_xor_si256(b, v->bias32));
}

/* mont_reduce on 64-bit lanes holding t = a b: the result in the low word */
static inline __m256i redc64(const vfield *v, __m256i t) {
    const __m256i m = _mm256_mul_epu32(t, v->qinv64);   /* low word used below */
    const __m256i mq = _mm256_mul_epu32(m, v->q64);
    const __m256i s = _mm256_add_epi64(t, mq);
    /* carry out of 64 bits: s < t unsigned */
    const __m256i carry =
        _mm256_cmpgt_epi64(_mm256_xor_si256(t, v->bias64), _mm256_xor_si256(s, v->bias64));
    __m256i r = _mm256_or_si256(_mm256_srli_epi64(s, 32), _mm256_and_si256(carry, v->two32));
    const __m256i ge = _mm256_cmpgt_epi64(r, v->qm1_64);  /* r < 2^33: signed compare */
    return _mm256_sub_epi64(r, _mm256_and_si256(ge, v->q64));
}

/* eight Montgomery products a b 2^-32 mod q, canonical */
static inline __m256i mont8(const vfield *v, __m256i a, __m256i b) {
    const __m256i re = redc64(v, _mm256_mul_epu32(a, b));
    const __m256i ro = redc64(v, _mm256_mul_epu32(_mm256_srli_epi64(a, 32),
                                                  _mm256_srli_epi64(b, 32)));
    return _mm256_blend_epi32(re, _mm256_slli_epi64(ro, 32), 0xAA);
}

static inline __m256i add8(const vfield *v, __m256i a, __m256i b) {
    const __m256i s = _mm256_add_epi32(a, b);
    const __m256i reduce = _mm256_or_si256(gt_u32(v, a, s), gt_u32(v, s, v->qm1_32));
    return _mm256_sub_epi32(s, _mm256_and_si256(reduce, v->q32));
}

static inline __m256i sub8(const vfield *v, __m256i a, __m256i b) {
    const __m256i borrow = gt_u32(v, b, a);
    return _mm256_add_epi32(_mm256_sub_epi32(a, b), _mm256_and_si256(borrow, v->q32));
}

#define LD(p) _mm256_loadu_si256((const __m256i *)(p))
#define ST(p, x) _mm256_storeu_si256((__m256i *)(p), (x))

static void pointwise(const orc_field *f, const vfield *v, uint32_t *dst, const uint32_t *rhs,
                      uint32_t n) {
    uint32_t i = 0;
    for (; i + 8 <= n; i += 8) ST(dst + i, mont8(v, LD(dst + i), LD(rhs + i)));
    for (; i < n; i++) dst[i] = orc_mul(f, dst[i], rhs[i]);
}

static void bit_reverse(uint32_t *x, uint32_t n) {
    for (uint32_t i = 1, j = 0; i < n; i++) {
        uint32_t bit = n >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) { const uint32_t t = x[i]; x[i] = x[j]; x[j] = t; }
    }
}

static void forward(const orc_plan *p, const vfield *v, uint32_t *x) {
    const orc_field *f = &p->f;
    const uint32_t n = p->n;
    bit_reverse(x, n);
    size_t off = 0;
    for (uint32_t len = 2; len <= n; len <<= 1) {
        const uint32_t half = len / 2;
        const uint32_t *tw = p->fwd_tw + off;
        for (uint32_t start = 0; start < n; start += len) {
            uint32_t *even = x + start, *odd = x + start + half;
            uint32_t i = 0;
            for (; i + 8 <= half; i += 8) {
                const __m256i e = LD(even + i);
                const __m256i t = mont8(v, LD(odd + i), LD(tw + i));
                ST(even + i, add8(v, e, t));
                ST(odd + i, sub8(v, e, t));
            }
            for (; i < half; i++) {
                const uint32_t t = orc_mul(f, odd[i], tw[i]);
                odd[i] = orc_sub(f, even[i], t);
                even[i] = orc_add(f, even[i], t);
            }
        }
        off += half;
    }
}

static void inverse(const orc_plan *p, const vfield *v, uint32_t *x) {
    const orc_field *f = &p->f;
    const uint32_t n = p->n;
    size_t off = 0;
    for (uint32_t len = n; len > 1; len >>= 1) {
        const uint32_t half = len / 2;
        const uint32_t *tw = p->inv_tw + off;
        const int final_stage = len == 2;
        for (uint32_t start = 0; start < n; start += len) {
            uint32_t *even = x + start, *odd = x + start + half;
            uint32_t i = 0;
            for (; !final_stage && i + 8 <= half; i += 8) {
                const __m256i e = LD(even + i), o = LD(odd + i);
                ST(odd + i, mont8(v, sub8(v, e, o), LD(tw + i)));
                ST(even + i, add8(v, e, o));
            }
            for (; i < half; i++) {
                const uint32_t diff = orc_sub(f, even[i], odd[i]);
                uint32_t ev = orc_add(f, even[i], odd[i]);
                uint32_t od = orc_mul(f, diff, tw[i]);
                if (final_stage) {
                    ev = orc_mul(f, ev, p->inv_scale);
                    od = orc_mul(f, od, p->inv_scale);
                }
                even[i] = ev;
                odd[i] = od;
            }
        }
        off += half;
    }
    bit_reverse(x, n);
}

void orc_ntt_mul_inverse_avx2(const orc_plan *p, const uint32_t *a, const uint32_t *b_evals,
                              uint32_t *out, size_t count) {
    const vfield v = vfield_of(&p->f);
    const uint32_t n = p->n;
    for (size_t c = 0; c < count; c++) {
        uint32_t *x = out + c * n;
        memcpy(x, a + c * n, sizeof(uint32_t) * n);
        pointwise(&p->f, &v, x, p->twists, n);
        forward(p, &v, x);
        pointwise(&p->f, &v, x, b_evals + c * n, n);
        inverse(p, &v, x);
        pointwise(&p->f, &v, x, p->untwists, n);
    }
}

void orc_ntt_mul_inverse_avx2_mt(const orc_plan *p, const uint32_t *a, const uint32_t *b_evals,
                                 uint32_t *out, size_t count, int threads) {
#ifdef _OPENMP
    if (threads < 1) threads = omp_get_max_threads();
    const long long cnt = (long long)count;
#pragma omp parallel for num_threads(threads) schedule(static)
    for (long long c = 0; c < cnt; c++)
        orc_ntt_mul_inverse_avx2(p, a + (size_t)c * p->n, b_evals + (size_t)c * p->n,
                                 out + (size_t)c * p->n, 1);
#else
    (void)threads;
    orc_ntt_mul_inverse_avx2(p, a, b_evals, out, count);
#endif
}

/* The prepared commitment t_b[row] = INTT(sum_k A_hat[row][k] * s_hat_b[k]),
 * the reference's mul_matrix_vector_trusted over cached A_hat evaluations
 * (commit/src/linear.rs:717-742, TwistedNttPoly::dot_product,
 * poly/twisted_ntt.rs:378-408, whose pointwise products and additions run
 * eight lanes at a time in the x86 backend): per witness, the twisted
 * forward transforms of its columns, one eight-lane multiply-accumulate pass
 * per row, the twisted inverse. a_is_eval = 0 transforms A first. */
int orc_matvec_avx2(const orc_plan *p, const uint32_t *A, size_t rows, size_t cols,
                    int a_is_eval, const uint32_t *s, size_t batch, uint32_t *t, int threads) {
    const vfield v = vfield_of(&p->f);
    const orc_field *f = &p->f;
    const uint32_t n = p->n;
    uint32_t *own = NULL;
    const uint32_t *ahat = A;
    if (!a_is_eval) {
        own = (uint32_t *)malloc(sizeof(uint32_t) * rows * cols * n);
        if (!own) return ORC_ERR_OOM;
        memcpy(own, A, sizeof(uint32_t) * rows * cols * n);
        for (size_t i = 0; i < rows * cols; i++) {
            pointwise(f, &v, own + i * n, p->twists, n);
            forward(p, &v, own + i * n);
        }
        ahat = own;
    }
    int err = 0;
    const long long nb = (long long)batch;
#ifdef _OPENMP
    if (threads < 1) threads = omp_get_max_threads();
#pragma omp parallel for num_threads(threads) schedule(dynamic)
#endif
    for (long long b = 0; b < nb; b++) {
        uint32_t *shat = (uint32_t *)malloc(sizeof(uint32_t) * cols * n);
        if (!shat) { err = 1; continue; }
        memcpy(shat, s + (size_t)b * cols * n, sizeof(uint32_t) * cols * n);
        for (size_t k = 0; k < cols; k++) {
            pointwise(f, &v, shat + k * n, p->twists, n);
            forward(p, &v, shat + k * n);
        }
        for (size_t row = 0; row < rows; row++) {
            uint32_t *out = t + ((size_t)b * rows + row) * n;
            const uint32_t *arow = ahat + row * cols * n;
            uint32_t e = 0;
            for (; e + 8 <= n; e += 8) {
                __m256i acc = _mm256_setzero_si256();
                for (size_t k = 0; k < cols; k++)
                    acc = add8(&v, acc, mont8(&v, LD(arow + k * n + e), LD(shat + k * n + e)));
                ST(out + e, acc);
            }
            for (; e < n; e++) {
                uint32_t acc = 0;
                for (size_t k = 0; k < cols; k++)
                    acc = orc_add(f, acc, orc_mul(f, arow[k * n + e], shat[k * n + e]));
                out[e] = acc;
            }
            inverse(p, &v, out);
            pointwise(f, &v, out, p->untwists, n);
        }
        free(shat);
    }
    (void)threads;
    free(own);
    return err ? ORC_ERR_OOM : ORC_OK;
}
