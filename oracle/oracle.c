/*
 * CPU oracle for the Gridland ring-arithmetic hot path — TEST INFRASTRUCTURE.
 *
 * Plain-C restatement of the reference's Rust CPU algorithms (mrain/lattica),
 * used only by tests/, __graft_entry__.smoke() and bench.py's CPU baseline as
 * the bit-exact checker. The CUDA library never links or calls this code.
 *
 * The reference is Rust and no Rust toolchain exists where this runs, so the
 * reference itself cannot be built; this restatement is pinned against the
 * known-answer tests held in the reference's own test modules (see
 * tests/golden/reference_kats.json and tests/test_oracle_kats.py).
 */
#include "oracle.h"

#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ------------------------------------------------------------------------ */
/* Prime field, PrimeField<Q, u32> (algebra/src/arith/prime.rs)              */
/* ------------------------------------------------------------------------ */

static uint64_t mulmod64(uint64_t a, uint64_t b, uint64_t m) {
    return (uint64_t)(((unsigned __int128)a * b) % m);
}

static uint64_t powmod64(uint64_t b, uint64_t e, uint64_t m) {
    /* pow_mod_const, prime.rs:807-819 */
    uint64_t acc = 1 % m;
    b %= m;
    while (e > 0) {
        if (e & 1) acc = mulmod64(acc, b, m);
        e >>= 1;
        if (e > 0) b = mulmod64(b, b, m);
    }
    return acc;
}

/* is_prime_const, prime.rs:776-800: trial division by small primes, then
 * Miller-Rabin with the deterministic 64-bit base set. */
int orc_is_prime_u64(uint64_t n) {
    static const uint64_t small[12] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37};
    static const uint64_t bases[7] = {2, 325, 9375, 28178, 450775, 9780504, 1795265022};
    if (n < 2) return 0;
    for (int i = 0; i < 12; i++) {
        if (n == small[i]) return 1;
        if (n % small[i] == 0) return 0;
    }
    uint64_t d = n - 1;
    int s = 0;
    while ((d & 1) == 0) { d >>= 1; s++; }
    for (int i = 0; i < 7; i++) {
        uint64_t a = bases[i] % n;
        if (a == 0) continue;
        uint64_t x = powmod64(a, d, n);
        if (x == 1 || x == n - 1) continue;
        int composite = 1;
        for (int r = 1; r < s; r++) {
            x = mulmod64(x, x, n);
            if (x == n - 1) { composite = 0; break; }
        }
        if (composite) return 0;
    }
    return 1;
}

int orc_field_init(orc_field *f, uint64_t q) {
    /* PrimeField::MODULUS const-asserts, prime.rs:31-46 (u32 limb). */
    if (q < 3 || (q & 1) == 0 || q >= (1ull << 32) || !orc_is_prime_u64(q))
        return ORC_ERR_INVALID_MODULUS;
    f->q = (uint32_t)q;
    f->r_mod_q = (uint32_t)((1ull << 32) % q);                         /* prime.rs:60-67 */
    f->r2_mod_q = (uint32_t)(((uint64_t)f->r_mod_q * f->r_mod_q) % q); /* prime.rs:73-78 */
    uint64_t inv = 1; /* Newton iteration, prime.rs:81-91 */
    for (int i = 0; i < 6; i++) inv = inv * (2 - q * inv);
    f->q_inv = (uint32_t)(0 - inv); /* -q^-1 mod 2^32 */
    return ORC_OK;
}

/* montgomery_reduce / montgomery_reduce_wide, prime.rs:141-183. */
static uint32_t mont_reduce(const orc_field *f, uint64_t t) {
    const uint32_t q = f->q;
    if (q >= (1u << 31)) {
        uint32_t t_lo = (uint32_t)t;
        uint32_t m = t_lo * f->q_inv;
        uint64_t product = (uint64_t)m * q;
        uint32_t t_hi = (uint32_t)(t >> 32);
        uint32_t prod_lo = (uint32_t)product;
        uint32_t prod_hi = (uint32_t)(product >> 32);
        uint32_t sum_lo = t_lo + prod_lo;
        int carry_lo = sum_lo < t_lo;
        uint32_t sum_hi = t_hi + prod_hi;
        int carry_a = sum_hi < t_hi;
        uint32_t sum_hi2 = sum_hi + (uint32_t)carry_lo;
        int carry_b = sum_hi2 < sum_hi;
        if (carry_a || carry_b) return sum_hi2 + (0u - q);
        if (sum_hi2 >= q) return sum_hi2 - q;
        return sum_hi2;
    }
    uint32_t m = (uint32_t)t * f->q_inv;
    uint64_t s = t + (uint64_t)m * q;
    uint32_t r = (uint32_t)(s >> 32);
    return r >= q ? r - q : r;
}

uint32_t orc_to_mont(const orc_field *f, uint64_t v) {
    /* to_montgomery, prime.rs:186-195 (value reduced mod q first) */
    uint32_t val = (uint32_t)(v % f->q);
    return mont_reduce(f, (uint64_t)val * f->r2_mod_q);
}

uint32_t orc_from_mont(const orc_field *f, uint32_t w) { return mont_reduce(f, w); }

uint32_t orc_add(const orc_field *f, uint32_t a, uint32_t b) {
    /* add_raw_words, prime.rs:110-126 */
    const uint32_t q = f->q;
    if (q < (1u << 31)) {
        uint32_t s = a + b;
        return s >= q ? s - q : s;
    }
    uint32_t s = a + b;
    int carry = s < a;
    return (carry || s >= q) ? s - q : s;
}

uint32_t orc_sub(const orc_field *f, uint32_t a, uint32_t b) {
    /* sub_raw_words, prime.rs:129-137 */
    return a >= b ? a - b : f->q - b + a;
}

uint32_t orc_mul(const orc_field *f, uint32_t a, uint32_t b) {
    /* mul_raw_words, prime.rs:223-226 */
    return mont_reduce(f, (uint64_t)a * b);
}

uint32_t orc_neg(const orc_field *f, uint32_t a) { return a == 0 ? 0 : f->q - a; }

uint32_t orc_pow(const orc_field *f, uint32_t base, uint64_t exp) {
    uint32_t result = f->r_mod_q;
    while (exp > 0) {
        if (exp & 1) result = orc_mul(f, result, base);
        base = orc_mul(f, base, base);
        exp >>= 1;
    }
    return result;
}

uint32_t orc_inv(const orc_field *f, uint32_t a) { return orc_pow(f, a, (uint64_t)f->q - 2); }

/* find_generator, prime.rs:645-687: factor q-1 by trial division, then the
 * smallest g >= 2 with g^((q-1)/p) != 1 for every prime factor p. */
uint32_t orc_find_generator(const orc_field *f) {
    uint64_t factors[64];
    int nf = 0;
    uint64_t n = (uint64_t)f->q - 1;
    for (uint64_t d = 2; d <= n / d; d++) {
        if (n % d == 0) {
            factors[nf++] = d;
            while (n % d == 0) n /= d;
        }
    }
    if (n > 1) factors[nf++] = n;
    for (uint64_t g = 2; g < f->q; g++) {
        uint32_t gm = orc_to_mont(f, g);
        int ok = 1;
        for (int i = 0; i < nf; i++) {
            if (orc_pow(f, gm, ((uint64_t)f->q - 1) / factors[i]) == f->r_mod_q) { ok = 0; break; }
        }
        if (ok) return gm;
    }
    return 0;
}

/* root_of_unity, prime.rs:566-586. Returns 0 (not a field unit) for None. */
static uint32_t root_of_unity(const orc_field *f, uint64_t n) {
    if (n == 0 || ((uint64_t)f->q - 1) % n != 0) return 0;
    uint32_t g = orc_find_generator(f);
    if (g == 0) return 0;
    uint32_t root = orc_pow(f, g, ((uint64_t)f->q - 1) / n);
    if (orc_pow(f, root, n) != f->r_mod_q) return 0;
    if (n > 1 && orc_pow(f, root, n / 2) == f->r_mod_q) return 0;
    return root;
}

uint64_t orc_max_ntt_size(uint64_t q) {
    /* max_ntt_size, prime.rs:598-607 */
    uint64_t v = q - 1, m = 1;
    while ((v & 1) == 0) { v >>= 1; m <<= 1; }
    return m;
}

/* ------------------------------------------------------------------------ */
/* NTT plans and transforms (algebra/src/arith/ntt.rs, poly/ntt.rs)          */
/* ------------------------------------------------------------------------ */

int orc_plan_create(orc_plan *p, uint64_t q, uint64_t n) {
    memset(p, 0, sizeof(*p));
    int st = orc_field_init(&p->f, q);
    if (st) return st;
    const orc_field *f = &p->f;
    /* NttPlan::build, ntt.rs:124-154 */
    if (n == 0 || (n & (n - 1)) != 0) return ORC_ERR_LENGTH_NOT_POW2;
    uint32_t root = root_of_unity(f, n);
    if (root == 0) return ORC_ERR_UNSUPPORTED_SIZE;
    uint32_t inv_root = orc_inv(f, root);
    /* TwistedNttPlan::build, poly/ntt.rs:139-154 */
    uint32_t psi = root_of_unity(f, 2 * n);
    if (psi == 0) return ORC_ERR_UNSUPPORTED_TWIST;
    uint32_t inv_psi = orc_inv(f, psi);

    p->n = (uint32_t)n;
    p->generator = orc_find_generator(f);
    p->omega = root;
    p->psi = psi;
    p->inv_scale = orc_inv(f, orc_to_mont(f, n)); /* inverse_ntt_scale, prime.rs:592-596 */
    p->fwd_tw = (uint32_t *)malloc(sizeof(uint32_t) * (n > 1 ? n - 1 : 1));
    p->inv_tw = (uint32_t *)malloc(sizeof(uint32_t) * (n > 1 ? n - 1 : 1));
    p->twists = (uint32_t *)malloc(sizeof(uint32_t) * n);
    p->untwists = (uint32_t *)malloc(sizeof(uint32_t) * n);
    if (!p->fwd_tw || !p->inv_tw || !p->twists || !p->untwists) {
        orc_plan_destroy(p);
        return ORC_ERR_OOM;
    }
    /* forward stages: stage_len = 2, 4, ..., n; w_len = root^(n/stage_len); stage_twiddles (ntt.rs:196-205) */
    size_t off = 0;
    for (uint64_t stage_len = 2; stage_len <= n; stage_len <<= 1) {
        uint64_t half = stage_len / 2;
        uint32_t w = orc_pow(f, root, n / stage_len);
        uint32_t cur = f->r_mod_q;
        for (uint64_t i = 0; i < half; i++) { p->fwd_tw[off++] = cur; cur = orc_mul(f, cur, w); }
    }
    /* inverse stages: stage_len = n, n/2, ..., 2 with inv_root */
    off = 0;
    for (uint64_t stage_len = n; stage_len > 1; stage_len >>= 1) {
        uint64_t half = stage_len / 2;
        uint32_t w = orc_pow(f, inv_root, n / stage_len);
        uint32_t cur = f->r_mod_q;
        for (uint64_t i = 0; i < half; i++) { p->inv_tw[off++] = cur; cur = orc_mul(f, cur, w); }
    }
    /* powers(psi, n), powers(inv_psi, n): poly/ntt.rs:128-137 */
    uint32_t cur = f->r_mod_q, cur_i = f->r_mod_q;
    for (uint64_t i = 0; i < n; i++) {
        p->twists[i] = cur;
        p->untwists[i] = cur_i;
        cur = orc_mul(f, cur, psi);
        cur_i = orc_mul(f, cur_i, inv_psi);
    }
    return ORC_OK;
}

void orc_plan_destroy(orc_plan *p) {
    free(p->fwd_tw);
    free(p->inv_tw);
    free(p->twists);
    free(p->untwists);
    p->fwd_tw = p->inv_tw = p->twists = p->untwists = NULL;
}

/* bit_reverse_permute, ntt.rs:180-194 */
static void bit_reverse_permute(uint32_t *v, uint32_t n) {
    uint32_t j = 0;
    for (uint32_t i = 1; i < n; i++) {
        uint32_t bit = n >> 1;
        while (j & bit) { j ^= bit; bit >>= 1; }
        j ^= bit;
        if (i < j) { uint32_t t = v[i]; v[i] = v[j]; v[j] = t; }
    }
}

/* scalar_ntt_forward_with_plan + apply_forward_chunk, ntt.rs:292-312,207-234 */
void orc_ntt_forward(const orc_plan *p, uint32_t *v) {
    const orc_field *f = &p->f;
    const uint32_t n = p->n;
    bit_reverse_permute(v, n);
    size_t off = 0;
    for (uint32_t len = 2; len <= n; len <<= 1) {
        const uint32_t half = len / 2;
        const uint32_t *tw = p->fwd_tw + off;
        for (uint32_t start = 0; start < n; start += len) {
            uint32_t *even = v + start, *odd = v + start + half;
            for (uint32_t i = 0; i < half; i++) {
                uint32_t t = orc_mul(f, odd[i], tw[i]);
                odd[i] = orc_sub(f, even[i], t);
                even[i] = orc_add(f, even[i], t);
            }
        }
        off += half;
    }
}

/* scalar_ntt_inverse_with_plan + apply_inverse_chunk, ntt.rs:314-340,236-280:
 * GS stages from len = n down to 2, n^-1 applied inside the last stage, then
 * bit reversal. */
void orc_ntt_inverse(const orc_plan *p, uint32_t *v) {
    const orc_field *f = &p->f;
    const uint32_t n = p->n;
    size_t off = 0;
    for (uint32_t len = n; len > 1; len >>= 1) {
        const uint32_t half = len / 2;
        const uint32_t *tw = p->inv_tw + off;
        const int final_stage = (len == 2);
        for (uint32_t start = 0; start < n; start += len) {
            uint32_t *even = v + start, *odd = v + start + half;
            for (uint32_t i = 0; i < half; i++) {
                uint32_t diff = orc_sub(f, even[i], odd[i]);
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
    bit_reverse_permute(v, n);
}

void orc_pointwise_mul(const orc_field *f, uint32_t *dst, const uint32_t *rhs, size_t len) {
    for (size_t i = 0; i < len; i++) dst[i] = orc_mul(f, dst[i], rhs[i]);
}

/* forward_in_place_trusted / inverse_in_place_trusted, poly/ntt.rs:75-104 */
void orc_twisted_forward(const orc_plan *p, uint32_t *polys, size_t count) {
    for (size_t c = 0; c < count; c++) {
        uint32_t *v = polys + c * p->n;
        orc_pointwise_mul(&p->f, v, p->twists, p->n);
        orc_ntt_forward(p, v);
    }
}

void orc_twisted_inverse(const orc_plan *p, uint32_t *polys, size_t count) {
    for (size_t c = 0; c < count; c++) {
        uint32_t *v = polys + c * p->n;
        orc_ntt_inverse(p, v);
        orc_pointwise_mul(&p->f, v, p->untwists, p->n);
    }
}

void orc_ntt_mul_inverse(const orc_plan *p, const uint32_t *a, const uint32_t *b_evals,
                         uint32_t *out, size_t count) {
    const uint32_t n = p->n;
    for (size_t c = 0; c < count; c++) {
        uint32_t *v = out + c * n;
        memcpy(v, a + c * n, sizeof(uint32_t) * n);
        orc_twisted_forward(p, v, 1);
        orc_pointwise_mul(&p->f, v, b_evals + c * n, n);
        orc_twisted_inverse(p, v, 1);
    }
}

void orc_ntt_mul_inverse_mt(const orc_plan *p, const uint32_t *a, const uint32_t *b_evals,
                            uint32_t *out, size_t count, int threads) {
#ifdef _OPENMP
    if (threads < 1) threads = omp_get_max_threads();
    const long long cnt = (long long)count;
#pragma omp parallel for num_threads(threads) schedule(static)
    for (long long c = 0; c < cnt; c++)
        orc_ntt_mul_inverse(p, a + (size_t)c * p->n, b_evals + (size_t)c * p->n,
                            out + (size_t)c * p->n, 1);
#else
    (void)threads;
    orc_ntt_mul_inverse(p, a, b_evals, out, count);
#endif
}

/* multiply_in_place, poly/ntt.rs:110-126 */
void orc_poly_mul_ntt(const orc_plan *p, const uint32_t *a, const uint32_t *b, uint32_t *out) {
    const uint32_t n = p->n;
    uint32_t *tmp = (uint32_t *)malloc(sizeof(uint32_t) * n);
    memcpy(out, a, sizeof(uint32_t) * n);
    memcpy(tmp, b, sizeof(uint32_t) * n);
    orc_twisted_forward(p, out, 1);
    orc_twisted_forward(p, tmp, 1);
    orc_pointwise_mul(&p->f, out, tmp, n);
    orc_twisted_inverse(p, out, 1);
    free(tmp);
}

/* neg_cyclic_mul, poly/ring.rs:60-77 */
void orc_naive_negacyclic(const orc_field *f, uint32_t n, const uint32_t *a, const uint32_t *b,
                          uint32_t *out) {
    for (uint32_t i = 0; i < n; i++) out[i] = 0;
    for (uint32_t i = 0; i < n; i++)
        for (uint32_t j = 0; j < n; j++) {
            uint32_t prod = orc_mul(f, a[i], b[j]);
            if (i + j < n) out[i + j] = orc_add(f, out[i + j], prod);
            else out[i + j - n] = orc_sub(f, out[i + j - n], prod);
        }
}

/* Slice hooks of Ring for PrimeField (arith/prime.rs:433-491, over
 * simd/montgomery.rs add_assign / sub_assign / scalar_mul): elementwise field
 * operations on Montgomery words. dot_product (prime.rs:467-491) sums the
 * Montgomery products; its CHUNK = 64 split changes no value. */
void orc_add_assign_slice(const orc_field *f, uint32_t *dst, const uint32_t *src, size_t len) {
    for (size_t i = 0; i < len; i++) dst[i] = orc_add(f, dst[i], src[i]);
}

void orc_sub_assign_slice(const orc_field *f, uint32_t *dst, const uint32_t *src, size_t len) {
    for (size_t i = 0; i < len; i++) dst[i] = orc_sub(f, dst[i], src[i]);
}

void orc_scalar_mul_slice(const orc_field *f, uint32_t *dst, uint32_t scalar, size_t len) {
    for (size_t i = 0; i < len; i++) dst[i] = orc_mul(f, dst[i], scalar);
}

/* add_assign_scaled_slice, prime.rs:449-465: dst += src * scalar */
void orc_add_assign_scaled_slice(const orc_field *f, uint32_t *dst, const uint32_t *src,
                                 uint32_t scalar, size_t len) {
    for (size_t i = 0; i < len; i++) dst[i] = orc_add(f, dst[i], orc_mul(f, src[i], scalar));
}

uint32_t orc_dot_product(const orc_field *f, const uint32_t *lhs, const uint32_t *rhs, size_t len) {
    uint32_t acc = 0;
    for (size_t i = 0; i < len; i++) acc = orc_add(f, acc, orc_mul(f, lhs[i], rhs[i]));
    return acc;
}

/* ------------------------------------------------------------------------ */
/* Ring products by the schoolbook rule, for any odd prime q < 2^32: the    */
/* path the reference takes when q has no 2d-th root of unity               */
/* (NegacyclicMulRing::negacyclic_mul_coeffs falls back to                  */
/* naive_negacyclic_mul_coeffs, poly/ring.rs:60-100).                       */
/* ------------------------------------------------------------------------ */

/* out = sum_k a_k * b_k in R_q (Ring::dot_product default, arith/ring.rs:167-175,
 * each term a negacyclic schoolbook product). The exact integer sums of the
 * word products are kept per output coefficient, positive and negative
 * (X^d = -1) separately, in 128 bits, and reduced once: sum of Montgomery
 * products = (sum of word products) * 2^-32 mod q, so the canonical words equal
 * those of the reference's term-by-term field arithmetic
 * (tests/test_oracle_ring.py checks this against orc_naive_negacyclic). */
static void ring_dot_schoolbook(const orc_field *f, uint32_t d, const uint32_t *a, size_t a_stride,
                                const uint32_t *b, size_t b_stride, size_t len, uint32_t *out,
                                unsigned __int128 *pos, unsigned __int128 *neg) {
    for (uint32_t c = 0; c < d; c++) pos[c] = neg[c] = 0;
    for (size_t k = 0; k < len; k++) {
        const uint32_t *x = a + k * a_stride, *y = b + k * b_stride;
        for (uint32_t i = 0; i < d; i++) {
            const uint64_t xi = x[i];
            for (uint32_t j = 0; j < d - i; j++) pos[i + j] += xi * y[j];
            for (uint32_t j = d - i; j < d; j++) neg[i + j - d] += xi * y[j];
        }
    }
    for (uint32_t c = 0; c < d; c++) {
        const uint32_t pm = (uint32_t)(pos[c] % f->q), nm = (uint32_t)(neg[c] % f->q);
        out[c] = mont_reduce(f, orc_sub(f, pm, nm));  /* x < q: x * 2^-32 mod q */
    }
}

/* RingMat::mul_slice per witness (lattice/types.rs:334-343):
 * t[b][i] = sum_k A[i][k] * s[b][k]. */
int orc_ring_matvec(const orc_field *f, uint32_t d, const uint32_t *A, size_t rows, size_t cols,
                    const uint32_t *s, size_t batch, uint32_t *t, int threads) {
    if (threads <= 0) threads = 1;
    int st = ORC_OK;
#pragma omp parallel num_threads(threads)
    {
        unsigned __int128 *pos = (unsigned __int128 *)malloc(sizeof(unsigned __int128) * d);
        unsigned __int128 *neg = (unsigned __int128 *)malloc(sizeof(unsigned __int128) * d);
        if (!pos || !neg) {
#pragma omp atomic write
            st = ORC_ERR_OOM;
        } else {
#pragma omp for schedule(dynamic)
            for (long long u = 0; u < (long long)(batch * rows); u++) {
                const size_t b = (size_t)u / rows, i = (size_t)u % rows;
                ring_dot_schoolbook(f, d, A + i * cols * d, d, s + b * cols * d, d, cols,
                                    t + u * d, pos, neg);
            }
        }
        free(pos);
        free(neg);
    }
    return st;
}

/* compute_garbage_g (labrador/src/main_protocol/garbage.rs:76-93) with
 * schoolbook products: g_ij = <s_i, s_j>, i <= j, garbage_index order. */
int orc_ring_gram(const orc_field *f, uint32_t d, const uint32_t *S, size_t r, size_t n,
                  uint32_t *G, int threads) {
    if (threads <= 0) threads = 1;
    const size_t cnt = r * (r + 1) / 2;
    int st = ORC_OK;
#pragma omp parallel num_threads(threads)
    {
        unsigned __int128 *pos = (unsigned __int128 *)malloc(sizeof(unsigned __int128) * d);
        unsigned __int128 *neg = (unsigned __int128 *)malloc(sizeof(unsigned __int128) * d);
        if (!pos || !neg) {
#pragma omp atomic write
            st = ORC_ERR_OOM;
        } else {
#pragma omp for schedule(dynamic)
            for (long long u = 0; u < (long long)cnt; u++) {
                size_t i = 0, rem = (size_t)u;
                while (rem >= r - i) { rem -= r - i; i++; }
                const size_t j = i + rem;
                ring_dot_schoolbook(f, d, S + i * n * d, d, S + j * n * d, d, n, G + u * d, pos,
                                    neg);
            }
        }
        free(pos);
        free(neg);
    }
    return st;
}

/* compute_garbage_h (garbage.rs:101-133) with schoolbook products:
 * h_ij = (<phi_i, s_j> + <phi_j, s_i>) * 2^-1, 2^-1 = R::from_u64(q / 2 + 1). */
int orc_ring_garbage_h(const orc_field *f, uint32_t d, const uint32_t *S, const uint32_t *Phi,
                       size_t r, size_t n, uint32_t *H, int threads) {
    if (threads <= 0) threads = 1;
    const size_t cnt = r * (r + 1) / 2;
    const uint32_t two_inv = orc_to_mont(f, f->q / 2 + 1);
    int st = ORC_OK;
#pragma omp parallel num_threads(threads)
    {
        unsigned __int128 *pos = (unsigned __int128 *)malloc(sizeof(unsigned __int128) * d);
        unsigned __int128 *neg = (unsigned __int128 *)malloc(sizeof(unsigned __int128) * d);
        uint32_t *t2 = (uint32_t *)malloc(sizeof(uint32_t) * d);
        if (!pos || !neg || !t2) {
#pragma omp atomic write
            st = ORC_ERR_OOM;
        } else {
#pragma omp for schedule(dynamic)
            for (long long u = 0; u < (long long)cnt; u++) {
                size_t i = 0, rem = (size_t)u;
                while (rem >= r - i) { rem -= r - i; i++; }
                const size_t j = i + rem;
                uint32_t *h = H + u * d;
                ring_dot_schoolbook(f, d, Phi + i * n * d, d, S + j * n * d, d, n, h, pos, neg);
                ring_dot_schoolbook(f, d, Phi + j * n * d, d, S + i * n * d, d, n, t2, pos, neg);
                for (uint32_t c = 0; c < d; c++) h[c] = orc_mul(f, orc_add(f, h[c], t2[c]), two_inv);
            }
        }
        free(pos);
        free(neg);
        free(t2);
    }
    return st;
}

/* compute_amortized_witness (labrador/src/main_protocol/amortization.rs:61-84)
 * without the challenge sampling: z[k] = sum_i c_i * s_i[k], schoolbook products. */
int orc_ring_amortize(const orc_field *f, uint32_t d, const uint32_t *S, const uint32_t *c,
                      size_t r, size_t n, uint32_t *Z, int threads) {
    if (threads <= 0) threads = 1;
    int st = ORC_OK;
#pragma omp parallel num_threads(threads)
    {
        unsigned __int128 *pos = (unsigned __int128 *)malloc(sizeof(unsigned __int128) * d);
        unsigned __int128 *neg = (unsigned __int128 *)malloc(sizeof(unsigned __int128) * d);
        if (!pos || !neg) {
#pragma omp atomic write
            st = ORC_ERR_OOM;
        } else {
#pragma omp for schedule(dynamic)
            for (long long k = 0; k < (long long)n; k++)
                ring_dot_schoolbook(f, d, c, d, S + (size_t)k * d, n * d, r, Z + (size_t)k * d,
                                    pos, neg);
        }
        free(pos);
        free(neg);
    }
    return st;
}

/* ------------------------------------------------------------------------ */
/* Matrix-vector in R_q and the linear commitment (commit/src/linear.rs)     */
/* ------------------------------------------------------------------------ */

/* TwistedNttPoly::dot_product, poly/twisted_ntt.rs:378-408: evaluation-wise
 * sum of Montgomery products. The CHUNK / len<=8 branches there change no
 * value, so one loop restates all of them. */
static void eval_dot(const orc_field *f, uint32_t n, const uint32_t *lhs, size_t lhs_stride,
                     const uint32_t *rhs, size_t rhs_stride, size_t len, uint32_t *acc) {
    for (uint32_t e = 0; e < n; e++) acc[e] = 0;
    for (size_t k = 0; k < len; k++) {
        const uint32_t *a = lhs + k * lhs_stride, *b = rhs + k * rhs_stride;
        for (uint32_t e = 0; e < n; e++) acc[e] = orc_add(f, acc[e], orc_mul(f, a[e], b[e]));
    }
}

static int matvec_impl(const orc_plan *p, const uint32_t *A, size_t rows, size_t cols,
                       int a_is_eval, const uint32_t *s, size_t batch, uint32_t *t, int threads) {
    const uint32_t n = p->n;
    uint32_t *ahat = (uint32_t *)malloc(sizeof(uint32_t) * rows * cols * n);
    if (!ahat) return ORC_ERR_OOM;
    memcpy(ahat, A, sizeof(uint32_t) * rows * cols * n);
    if (!a_is_eval) orc_twisted_forward(p, ahat, rows * cols); /* prepare_poly_matrix */
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
        orc_twisted_forward(p, shat, cols); /* prepare_poly_vector */
        for (size_t row = 0; row < rows; row++) {
            uint32_t *out = t + ((size_t)b * rows + row) * n;
            eval_dot(&p->f, n, ahat + row * cols * n, n, shat, n, cols, out); /* mul_matrix_vector_trusted */
            orc_twisted_inverse(p, out, 1); /* finish_prepared_vector */
        }
        free(shat);
    }
    (void)threads;
    free(ahat);
    return err ? ORC_ERR_OOM : ORC_OK;
}

int orc_matvec(const orc_plan *p, const uint32_t *A, size_t rows, size_t cols, int a_is_eval,
               const uint32_t *s, size_t batch, uint32_t *t) {
    return matvec_impl(p, A, rows, cols, a_is_eval, s, batch, t, 1);
}

int orc_matvec_mt(const orc_plan *p, const uint32_t *A, size_t rows, size_t cols, int a_is_eval,
                  const uint32_t *s, size_t batch, uint32_t *t, int threads) {
    return matvec_impl(p, A, rows, cols, a_is_eval, s, batch, t, threads);
}

/* recompute_linear_commitment_parts_trusted + finish, linear.rs:476-506,512-529:
 * t[row] = INTT( <A_msg[row], m_hat> + <A_open[row], r_hat> ). */
int orc_linear_commit(const orc_plan *p, const uint32_t *a_msg, size_t rows, size_t msg_cols,
                      const uint32_t *a_open, size_t open_cols, const uint32_t *m,
                      const uint32_t *r, uint32_t *t) {
    const uint32_t n = p->n;
    if (rows == 0 || msg_cols == 0 || open_cols == 0) return ORC_ERR_INVALID_PARAMETERS;
    size_t na = rows * msg_cols * n, no = rows * open_cols * n;
    uint32_t *am = (uint32_t *)malloc(sizeof(uint32_t) * na);
    uint32_t *ao = (uint32_t *)malloc(sizeof(uint32_t) * no);
    uint32_t *mh = (uint32_t *)malloc(sizeof(uint32_t) * msg_cols * n);
    uint32_t *rh = (uint32_t *)malloc(sizeof(uint32_t) * open_cols * n);
    uint32_t *tmp = (uint32_t *)malloc(sizeof(uint32_t) * n);
    memcpy(am, a_msg, sizeof(uint32_t) * na);
    memcpy(ao, a_open, sizeof(uint32_t) * no);
    memcpy(mh, m, sizeof(uint32_t) * msg_cols * n);
    memcpy(rh, r, sizeof(uint32_t) * open_cols * n);
    orc_twisted_forward(p, am, rows * msg_cols);
    orc_twisted_forward(p, ao, rows * open_cols);
    orc_twisted_forward(p, mh, msg_cols);
    orc_twisted_forward(p, rh, open_cols);
    for (size_t row = 0; row < rows; row++) {
        uint32_t *out = t + row * n;
        eval_dot(&p->f, n, am + row * msg_cols * n, n, mh, n, msg_cols, out);
        eval_dot(&p->f, n, ao + row * open_cols * n, n, rh, n, open_cols, tmp);
        for (uint32_t e = 0; e < n; e++) out[e] = orc_add(&p->f, out[e], tmp[e]);
        orc_twisted_inverse(p, out, 1);
    }
    free(am); free(ao); free(mh); free(rh); free(tmp);
    return ORC_OK;
}

/* ------------------------------------------------------------------------ */
/* Gram / garbage g (labrador/src/main_protocol/garbage.rs:76-93)            */
/* ------------------------------------------------------------------------ */

size_t orc_garbage_index(size_t r, size_t i, size_t j) {
    /* garbage_index, main_protocol/mod.rs:664-670 */
    return i * r - (i * (i - 1)) / 2 * (i > 0) + (j - i);
}

int orc_gram(const orc_plan *p, const uint32_t *S, size_t r, size_t n, uint32_t *G, int threads) {
    const uint32_t d = p->n;
    size_t total = r * n * d;
    uint32_t *sh = (uint32_t *)malloc(sizeof(uint32_t) * total);
    if (!sh) return ORC_ERR_OOM;
    memcpy(sh, S, sizeof(uint32_t) * total);
    orc_twisted_forward(p, sh, r * n);
    const long long npairs = (long long)(r * (r + 1) / 2);
#ifdef _OPENMP
    if (threads < 1) threads = omp_get_max_threads();
#pragma omp parallel for num_threads(threads) schedule(dynamic)
#endif
    for (long long idx = 0; idx < npairs; idx++) {
        /* invert the upper-triangular index */
        size_t i = 0, rem = (size_t)idx;
        while (rem >= r - i) { rem -= r - i; i++; }
        size_t j = i + rem;
        uint32_t *out = G + (size_t)idx * d;
        eval_dot(&p->f, d, sh + i * n * d, d, sh + j * n * d, d, n, out);
        orc_twisted_inverse(p, out, 1);
    }
    (void)threads;
    free(sh);
    return ORC_OK;
}

int orc_gram_naive(const orc_plan *p, const uint32_t *S, size_t r, size_t n, uint32_t *G) {
    /* Ring::dot_product default (arith/ring.rs:167-175): sum of full
     * coefficient-domain products, each via negacyclic_mul_coeffs. */
    const uint32_t d = p->n;
    uint32_t *prod = (uint32_t *)malloc(sizeof(uint32_t) * d);
    size_t idx = 0;
    for (size_t i = 0; i < r; i++)
        for (size_t j = i; j < r; j++, idx++) {
            uint32_t *out = G + idx * d;
            for (uint32_t e = 0; e < d; e++) out[e] = 0;
            for (size_t k = 0; k < n; k++) {
                orc_poly_mul_ntt(p, S + (i * n + k) * d, S + (j * n + k) * d, prod);
                for (uint32_t e = 0; e < d; e++) out[e] = orc_add(&p->f, out[e], prod[e]);
            }
        }
    free(prod);
    return ORC_OK;
}

/* compute_garbage_h, garbage.rs:101-133:
 * h_ij = (<phi_i, s_j> + <phi_j, s_i>) * 2^-1, i <= j in garbage_index order.
 * 2^-1 is the field element (q + 1) / 2 (R::from_u64(q / 2 + 1)), applied to
 * every coefficient; the dot products are ring inner products, evaluated here
 * in the twisted domain (exact field arithmetic, the same words). */
int orc_garbage_h(const orc_plan *p, const uint32_t *S, const uint32_t *Phi, size_t r, size_t n,
                  uint32_t *H) {
    const uint32_t d = p->n;
    const size_t total = r * n * d;
    uint32_t *sh = (uint32_t *)malloc(sizeof(uint32_t) * total);
    uint32_t *ph = (uint32_t *)malloc(sizeof(uint32_t) * total);
    uint32_t *tmp = (uint32_t *)malloc(sizeof(uint32_t) * d);
    if (!sh || !ph || !tmp) { free(sh); free(ph); free(tmp); return ORC_ERR_OOM; }
    memcpy(sh, S, sizeof(uint32_t) * total);
    memcpy(ph, Phi, sizeof(uint32_t) * total);
    orc_twisted_forward(p, sh, r * n);
    orc_twisted_forward(p, ph, r * n);
    const uint32_t two_inv = orc_to_mont(&p->f, (uint64_t)p->f.q / 2 + 1);
    size_t idx = 0;
    for (size_t i = 0; i < r; i++)
        for (size_t j = i; j < r; j++, idx++) {
            uint32_t *out = H + idx * d;
            eval_dot(&p->f, d, ph + i * n * d, d, sh + j * n * d, d, n, out);
            eval_dot(&p->f, d, ph + j * n * d, d, sh + i * n * d, d, n, tmp);
            for (uint32_t e = 0; e < d; e++) out[e] = orc_add(&p->f, out[e], tmp[e]);
            orc_twisted_inverse(p, out, 1);
            for (uint32_t e = 0; e < d; e++) out[e] = orc_mul(&p->f, out[e], two_inv);
        }
    free(sh); free(ph); free(tmp);
    return ORC_OK;
}

/* compute_amortized_witness, amortization.rs:61-84 (the challenge sampling
 * from the transcript stays with the caller): z[k] = sum_i c_i * s_i[k], ring
 * products evaluated in the twisted domain. */
int orc_amortize(const orc_plan *p, const uint32_t *S, const uint32_t *c, size_t r, size_t n,
                 uint32_t *Z) {
    const uint32_t d = p->n;
    uint32_t *sh = (uint32_t *)malloc(sizeof(uint32_t) * r * n * d);
    uint32_t *ch = (uint32_t *)malloc(sizeof(uint32_t) * r * d);
    if (!sh || !ch) { free(sh); free(ch); return ORC_ERR_OOM; }
    memcpy(sh, S, sizeof(uint32_t) * r * n * d);
    memcpy(ch, c, sizeof(uint32_t) * r * d);
    orc_twisted_forward(p, sh, r * n);
    orc_twisted_forward(p, ch, r);
    for (size_t k = 0; k < n; k++) {
        uint32_t *out = Z + k * d;
        /* sum over i of c_hat[i] (stride d) times s_hat[i][k] (stride n * d) */
        eval_dot(&p->f, d, ch, d, sh + k * d, n * d, r, out);
        orc_twisted_inverse(p, out, 1);
    }
    free(sh); free(ch);
    return ORC_OK;
}

/* ------------------------------------------------------------------------ */
/* Decompositions                                                            */
/* ------------------------------------------------------------------------ */

/* centered_mod, main_protocol/mod.rs:279-289 (truncating % like Rust) */
int64_t orc_centered_mod(int64_t v, int64_t base) {
    int64_t half = base / 2;
    int64_t r = v % base;
    if (r > half) return r - base;
    if (r < -half) return r + base;
    return r;
}

/* decompose_coeff_balanced, main_protocol/mod.rs:258-275. The reference
 * computes in i128; for q < 2^32 every intermediate fits in i64. */
void orc_decompose_coeff_balanced(uint64_t c, uint64_t base, size_t num_limbs, uint64_t q,
                                  int64_t *limbs_out) {
    int64_t half_q = (int64_t)(q / 2);
    int64_t carry = (int64_t)c;
    if (carry > half_q) carry -= (int64_t)q;
    for (size_t k = 0; k < num_limbs; k++) {
        int64_t limb = orc_centered_mod(carry, (int64_t)base);
        limbs_out[k] = limb;
        carry = (carry - limb) / (int64_t)base;
    }
}

/* decompose_polys + decompose_poly_balanced, main_protocol/mod.rs:296-323,731-747.
 * out layout: [poly][limb][coeff], limbs stored as Montgomery words of
 * limb mod q (negative limb v -> q - |v|). */
int orc_decompose_polys(const orc_field *f, uint32_t d, const uint32_t *polys, size_t npolys,
                        uint64_t base, size_t num_limbs, uint32_t *out) {
    if (base < 2 || num_limbs == 0) return ORC_ERR_INVALID_PARAMETERS;
    int64_t *limbs = (int64_t *)malloc(sizeof(int64_t) * num_limbs);
    for (size_t pi = 0; pi < npolys; pi++)
        for (uint32_t i = 0; i < d; i++) {
            uint64_t c = orc_from_mont(f, polys[pi * d + i]);
            orc_decompose_coeff_balanced(c, base, num_limbs, f->q, limbs);
            for (size_t k = 0; k < num_limbs; k++) {
                int64_t l = limbs[k];
                uint64_t u = l >= 0 ? (uint64_t)l : (uint64_t)f->q - (uint64_t)(-l);
                out[(pi * num_limbs + k) * d + i] = orc_to_mont(f, u);
            }
        }
    free(limbs);
    return ORC_OK;
}

/* reconstruct_from_limbs, main_protocol/mod.rs:331-359 */
int orc_reconstruct_from_limbs(const orc_field *f, uint32_t d, const uint32_t *limbs,
                               size_t num_limbs, uint64_t base, uint32_t *out) {
    const __int128 q = f->q;
    const __int128 b = (__int128)base;
    for (uint32_t i = 0; i < d; i++) {
        __int128 acc = 0, pw = 1;
        for (size_t k = 0; k < num_limbs; k++) {
            __int128 lu = orc_from_mont(f, limbs[k * d + i]);
            __int128 ls = lu > b / 2 ? lu - q : lu;
            acc = (acc + ls * pw) % q;
            if (acc < 0) acc += q;
            pw = (pw * b) % q;
        }
        out[i] = orc_to_mont(f, (uint64_t)acc);
    }
    return ORC_OK;
}

/* num_digits(q - 1, base), algebra/src/poly/decomposition.rs:9-17,19-22 */
size_t orc_gadget_digits(uint64_t q, uint64_t base) {
    uint64_t m = q - 1;
    size_t digits = 0;
    while (m > 0) { digits++; m /= base; }
    return digits ? digits : 1;
}

/* gadget_decompose, algebra/src/poly/decomposition.rs:47-61 */
int orc_gadget_decompose(const orc_field *f, const uint32_t *x, size_t len, uint64_t base,
                         uint32_t *out) {
    if (base < 2) return ORC_ERR_INVALID_PARAMETERS;
    size_t k = orc_gadget_digits(f->q, base);
    for (size_t i = 0; i < len; i++) {
        uint64_t v = orc_from_mont(f, x[i]);
        for (size_t dg = 0; dg < k; dg++) {
            out[dg * len + i] = orc_to_mont(f, v % base);
            v /= base;
        }
    }
    return ORC_OK;
}

/* ------------------------------------------------------------------------ */
/* ChaCha20 (RFC 8439) and the JL projection (labrador/src/jl.rs)            */
/* ------------------------------------------------------------------------ */

static inline uint32_t rotl32(uint32_t x, int r) { return (x << r) | (x >> (32 - r)); }

void orc_chacha20_quarter(uint32_t *a, uint32_t *b, uint32_t *c, uint32_t *d) {
    *a += *b; *d ^= *a; *d = rotl32(*d, 16);
    *c += *d; *b ^= *c; *b = rotl32(*b, 12);
    *a += *b; *d ^= *a; *d = rotl32(*d, 8);
    *c += *d; *b ^= *c; *b = rotl32(*b, 7);
}

static inline uint32_t load_le32(const uint8_t *p) {
    return (uint32_t)p[0] | ((uint32_t)p[1] << 8) | ((uint32_t)p[2] << 16) | ((uint32_t)p[3] << 24);
}

void orc_chacha20_block(const uint8_t key[32], uint32_t counter, const uint8_t nonce[12],
                        uint8_t out[64]) {
    uint32_t s[16], x[16];
    s[0] = 0x61707865u; s[1] = 0x3320646eu; s[2] = 0x79622d32u; s[3] = 0x6b206574u;
    for (int i = 0; i < 8; i++) s[4 + i] = load_le32(key + 4 * i);
    s[12] = counter;
    for (int i = 0; i < 3; i++) s[13 + i] = load_le32(nonce + 4 * i);
    memcpy(x, s, sizeof(s));
    for (int i = 0; i < 10; i++) {
        orc_chacha20_quarter(&x[0], &x[4], &x[8], &x[12]);
        orc_chacha20_quarter(&x[1], &x[5], &x[9], &x[13]);
        orc_chacha20_quarter(&x[2], &x[6], &x[10], &x[14]);
        orc_chacha20_quarter(&x[3], &x[7], &x[11], &x[15]);
        orc_chacha20_quarter(&x[0], &x[5], &x[10], &x[15]);
        orc_chacha20_quarter(&x[1], &x[6], &x[11], &x[12]);
        orc_chacha20_quarter(&x[2], &x[7], &x[8], &x[13]);
        orc_chacha20_quarter(&x[3], &x[4], &x[9], &x[14]);
    }
    for (int i = 0; i < 16; i++) {
        uint32_t v = x[i] + s[i];
        out[4 * i + 0] = (uint8_t)v;
        out[4 * i + 1] = (uint8_t)(v >> 8);
        out[4 * i + 2] = (uint8_t)(v >> 16);
        out[4 * i + 3] = (uint8_t)(v >> 24);
    }
}

/* Byte `pos` of the keystream for (key, nonce): block pos/64, offset pos%64. */
typedef struct {
    const uint8_t *key;
    uint8_t nonce[12];
    uint64_t block_idx;
    uint8_t block[64];
} ks_cursor;

static inline uint8_t ks_byte(ks_cursor *c, uint64_t pos) {
    uint64_t bi = pos >> 6;
    if (bi != c->block_idx) {
        orc_chacha20_block(c->key, (uint32_t)bi, c->nonce, c->block);
        c->block_idx = bi;
    }
    return c->block[pos & 63];
}

/* project_and_extract_seq, jl.rs:388-508. Part i uses key = seed, nonce =
 * (u32 i little-endian) || 0^8, keystream counter from 0; column `col`
 * consumes packed_len = ceil(rows/4) bytes starting at col*packed_len; row r
 * reads bits 2*(r%4) of byte r/4: 00 -> +1, 01 -> -1, 1x -> 0. */
int orc_jl_project(const orc_field *f, const uint8_t seed[32], size_t rows, size_t cols,
                   const uint32_t *parts, size_t num_parts, size_t d, uint32_t *p_out,
                   int8_t *flat_out, int threads) {
    if (d == 0 || cols % d != 0 || rows == 0) return ORC_ERR_INVALID_PARAMETERS;
    const size_t n = cols / d;
    const size_t packed_len = (rows + 3) / 4;
    const size_t plane = num_parts * d * n; /* flat stride per row */
    uint32_t *partial = (uint32_t *)calloc(num_parts * rows, sizeof(uint32_t));
    if (!partial) return ORC_ERR_OOM;
    const long long np = (long long)num_parts;
#ifdef _OPENMP
    if (threads < 1) threads = omp_get_max_threads();
#pragma omp parallel for num_threads(threads) schedule(dynamic)
#endif
    for (long long part_idx = 0; part_idx < np; part_idx++) {
        ks_cursor cur;
        cur.key = seed;
        memset(cur.nonce, 0, 12);
        cur.nonce[0] = (uint8_t)part_idx;
        cur.nonce[1] = (uint8_t)(part_idx >> 8);
        cur.nonce[2] = (uint8_t)(part_idx >> 16);
        cur.nonce[3] = (uint8_t)(part_idx >> 24);
        cur.block_idx = ~0ull;
        uint32_t *acc = partial + (size_t)part_idx * rows;
        const uint32_t *part = parts + (size_t)part_idx * cols;
        for (size_t col = 0; col < cols; col++) {
            const uint32_t coeff = part[col];
            const size_t poly_idx = col / d, coeff_idx = col % d;
            const size_t part_flat_base = ((size_t)part_idx * d + coeff_idx) * n + poly_idx;
            const uint64_t ks_base = (uint64_t)col * packed_len;
            for (size_t byte_idx = 0; byte_idx < packed_len; byte_idx++) {
                uint8_t byte = ks_byte(&cur, ks_base + byte_idx);
                for (int nib = 0; nib < 4; nib++) {
                    size_t row = byte_idx * 4 + nib;
                    if (row >= rows) break;
                    uint8_t val = (byte >> (nib * 2)) & 3;
                    int8_t e = 0;
                    if (val == 0) { acc[row] = orc_add(f, acc[row], coeff); e = 1; }
                    else if (val == 1) { acc[row] = orc_sub(f, acc[row], coeff); e = -1; }
                    if (flat_out) flat_out[row * plane + part_flat_base] = e;
                }
            }
        }
    }
    (void)threads;
    /* p accumulates parts in order; field addition is exact, so summing the
     * per-part partials gives the same words as the sequential loop. */
    for (size_t row = 0; row < rows; row++) {
        uint32_t v = 0;
        for (size_t pi = 0; pi < num_parts; pi++) v = orc_add(f, v, partial[pi * rows + row]);
        p_out[row] = v;
    }
    free(partial);
    return ORC_OK;
}

/* jl_rows_flat_to_conjugated_polys (main_protocol/mod.rs:885-923) and the
 * jl_evals loop of prove_step (step_prover.rs:185-206):
 * evals[m] = sum_{i < num_parts} sum_j conj(pi_{m,i,j}) * s_{i,j}, where
 * conj(pi)_0 = pi_0 and conj(pi)_k = -pi_{d-k}, each entry taken as the field
 * element of a residue in {0, 1, q - 1} (R::from_u64). flat: the int8 entries
 * [m][part][k][j] from orc_jl_project; parts: num_parts x (n * d) words. */
int orc_jl_evals(const orc_plan *p, const int8_t *flat, size_t rows, const uint32_t *parts,
                 size_t num_parts, size_t n, uint32_t *evals) {
    const uint32_t d = p->n;
    const uint64_t q = p->f.q;
    uint32_t *conj = (uint32_t *)malloc(sizeof(uint32_t) * d);
    uint32_t *prod = (uint32_t *)malloc(sizeof(uint32_t) * d);
    if (!conj || !prod) { free(conj); free(prod); return ORC_ERR_OOM; }
    for (size_t m = 0; m < rows; m++) {
        uint32_t *out = evals + m * d;
        for (uint32_t e = 0; e < d; e++) out[e] = 0;
        for (size_t i = 0; i < num_parts; i++)
            for (size_t j = 0; j < n; j++) {
                for (uint32_t k = 0; k < d; k++) {
                    const uint32_t src = k == 0 ? 0 : d - k;
                    const int8_t v = flat[((m * num_parts + i) * d + src) * n + j];
                    const uint64_t u = v < 0 ? q - (uint64_t)(-v) : (uint64_t)v;
                    const uint64_t val = (k == 0 || u == 0) ? u : q - u;
                    conj[k] = orc_to_mont(&p->f, val);
                }
                orc_poly_mul_ntt(p, conj, parts + (i * n + j) * d, prod);
                for (uint32_t e = 0; e < d; e++) out[e] = orc_add(&p->f, out[e], prod[e]);
            }
    }
    free(conj); free(prod);
    return ORC_OK;
}

/* CommitKey::from_seed / sample_uniform_mat (labrador/src/crs.rs:136-198,
 * 308-326): npolys ring elements drawn in order from ChaCha20Rng(seed), each
 * coefficient by PrimeField::rand (algebra/src/arith/prime.rs:730-743): u64
 * rejection sampling (accept s <= u64::MAX - ((u64::MAX % q + 1) % q)), then
 * from_u64(s % q). ChaCha20Rng is the rand_chacha 0.10.0 generator
 * (Cargo.lock): ChaCha20 blocks with a 64-bit block counter from 0 and stream
 * 0; rand_core 0.10.1's block RNG returns each u64 as two consecutive
 * little-endian keystream words (low word first). accept_max = 0 selects the
 * reference's threshold; another value replaces it (to exercise rejections). */
int orc_sample_uniform_polys(const orc_field *f, const uint8_t seed[32], size_t npolys,
                             uint32_t d, uint64_t accept_max, uint32_t *out) {
    const uint64_t q = f->q;
    const uint64_t reject = (UINT64_MAX % q + 1) % q;
    const uint64_t upper = accept_max ? accept_max : UINT64_MAX - reject;
    uint8_t block[64], nonce[12] = {0};
    uint64_t blk = 0;
    int idx = 16; /* words left in the current block: none */
    uint32_t words[16];
    for (size_t i = 0; i < npolys * d; i++) {
        for (;;) {
            if (idx >= 16) {
                const uint32_t hi = (uint32_t)(blk >> 32);
                for (int b = 0; b < 4; b++) nonce[b] = (uint8_t)(hi >> (8 * b));
                orc_chacha20_block(seed, (uint32_t)blk, nonce, block);
                for (int w = 0; w < 16; w++) words[w] = load_le32(block + 4 * w);
                blk++;
                idx = 0;
            }
            const uint64_t sample = (uint64_t)words[idx] | ((uint64_t)words[idx + 1] << 32);
            idx += 2;
            if (sample <= upper) {
                out[i] = orc_to_mont(f, sample % q);
                break;
            }
        }
    }
    return ORC_OK;
}
