/*
 * grid_gpu.h — C ABI of the B200 (sm_100a) ring-arithmetic hot path for
 * Gridland (mrain/lattica): R_q = Z_q[X]/(X^d + 1), q an odd prime < 2^32.
 *
 * Data convention (zero-copy with the reference's types):
 *   - A coefficient of R_q is one uint32_t PrimeField<Q, u32> Montgomery word,
 *     value * 2^32 mod q, canonical in [0, q) (algebra/src/arith/prime.rs:24-29,
 *     repr(transparent) over u32).
 *   - A polynomial is d consecutive words (CyclotomicPolyRing / TwistedNttPoly
 *     are inline [R; N], algebra/src/poly/ring.rs:111-118,
 *     algebra/src/poly/twisted_ntt.rs:22-27).
 *   - A ring matrix is row-major rows x cols polynomials (RingMat,
 *     algebra/src/lattice/types.rs:230-265); a batch of vectors is
 *     batch x len polynomials.
 *   - "Evaluations" means the reference's twisted NTT domain: slot k holds
 *     a(psi^(2k+1)) with psi = g^((q-1)/2d), g the smallest generator.
 *
 * Entry points come in two flavours:
 *   - *_dev: device pointers, asynchronous on the caller's cudaStream_t
 *     (passed as void*; NULL = legacy default stream). 16-byte aligned
 *     buffers are required.
 *   - host-buffer calls (no suffix): host pointers, synchronous; they copy in,
 *     compute, copy out. Pinned buffers (grid_gpu_host_register) overlap copies
 *     with compute.
 *
 * Every call returns a grid_status; none aborts. Plans are bound to the CUDA
 * device current at creation. Host-buffer calls on one plan are serialised
 * internally; *_dev calls are safe from several threads with distinct streams.
 */
#ifndef GRID_GPU_H
#define GRID_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum grid_status {
  GRID_OK = 0,
  /* NttError (algebra/src/arith/ntt.rs:40-50) */
  GRID_ERR_LENGTH_MISMATCH = 1,
  GRID_ERR_LENGTH_NOT_POW2 = 2,
  GRID_ERR_UNSUPPORTED_SIZE = 3,
  GRID_ERR_UNSUPPORTED_TWIST = 4,
  /* CommitmentError (commit/src/error.rs:7-18) */
  GRID_ERR_INVALID_PARAMETERS = 5,
  GRID_ERR_DIMENSION_MISMATCH = 6,
  /* PrimeField const checks (algebra/src/arith/prime.rs:31-46) */
  GRID_ERR_INVALID_MODULUS = 7,
  /* ABI-level */
  GRID_ERR_NULL_POINTER = 8,
  GRID_ERR_OUT_OF_MEMORY = 9,
  GRID_ERR_CUDA = 10,
  GRID_ERR_TIMEOUT = 11,           /* a bounded device-side wait gave up */
  GRID_ERR_UNSUPPORTED_DEGREE = 12, /* valid plan, but no kernel compiled for this d */
  GRID_ERR_MISALIGNED = 13,
  GRID_ERR_NO_DEVICE = 14,
  GRID_ERR_SCRATCH_LIMIT = 15,     /* needs more than the no-alloc entry point's fixed buffer */
  GRID_ERR_SAMPLE_EXHAUSTED = 16   /* uniform sampling met more rejections than its margin */
} grid_status;

typedef struct grid_gpu_plan grid_gpu_plan;
typedef struct grid_gpu_matrix grid_gpu_matrix;

typedef struct grid_gpu_plan_info {
  uint32_t q;
  uint32_t d;
  uint32_t generator; /* Montgomery word of the smallest generator of Z_q^* */
  uint32_t psi;       /* Montgomery word of root_of_unity(2d) */
  uint32_t omega;     /* Montgomery word of root_of_unity(d) = psi^2 */
  uint32_t n_inv;     /* Montgomery word of d^-1 */
  uint32_t r_mod_q;   /* 2^32 mod q (the Montgomery one) */
  uint32_t r2_mod_q;  /* 2^64 mod q */
  uint64_t max_ntt_size;
} grid_gpu_plan_info;

/* ---- library ---------------------------------------------------------- */

/* Human-readable name of a status code (static string). */
const char* grid_gpu_status_string(int status);
/* ABI version: (major << 16) | minor. */
uint32_t grid_gpu_abi_version(void);
/* Largest ring degree with compiled kernels (256). */
uint32_t grid_gpu_max_degree(void);

/* ---- plans: replace NttPlan::build / TwistedNttPlan::build ------------- */

/* Mirrors TwistedNttPlan::build (algebra/src/poly/ntt.rs:139-154) over
 * NttPlan::build (algebra/src/arith/ntt.rs:124-154): validates q, then
 * LengthNotPowerOfTwo, UnsupportedSize, UnsupportedTwist in that order. */
int grid_gpu_plan_create(uint64_t q, uint64_t d, grid_gpu_plan** out);
int grid_gpu_plan_destroy(grid_gpu_plan* plan);
/* Ring plan: the plan of CyclotomicPolyRing<PrimeField<q>, d> arithmetic,
 * mirroring NegacyclicMulRing::negacyclic_mul_coeffs (algebra/src/poly/ring.rs:79-102),
 * which multiplies through the twisted NTT when q has a primitive 2d-th root of
 * unity and by the schoolbook rule (naive_negacyclic_mul_coeffs, ring.rs:60-77)
 * otherwise. For an NTT-friendly (q, d) this is grid_gpu_plan_create. For any
 * other odd prime q < 2^32 and d in {8, ..., 256} it returns a plan whose ring
 * products are exact integer sums of the word products, computed through three
 * auxiliary NTT primes just below 2^32 and reconstructed mod q: the same words as
 * the schoolbook rule. On such a plan the ring-level calls work (poly_mul,
 * matrix_create with a_is_evals = 0, commit, linear/BDLOP commits, Gram,
 * garbage h, amortization, the prover round, JL, decompositions, sampling,
 * slice hooks); calls that need an evaluation domain mod q (NTT, ntt_mul_inverse,
 * matrix evaluations, a_is_evals = 1, batch commits) return the error
 * TwistedNttPlan::build reports for (q, d). Exactness bound: an output
 * coefficient sums at most terms * d word products (terms = n for a commitment
 * or Gram row, r for the amortized witness, 1 for poly_mul); calls with
 * terms * d * (q - 1)^2 >= 2^93 return GRID_ERR_INVALID_PARAMETERS. */
int grid_gpu_ring_plan_create(uint64_t q, uint64_t d, grid_gpu_plan** out);
/* kind = 0: NTT plan; 1: ring plan through auxiliary primes (their three
 * moduli written to aux_moduli when it is not NULL). */
int grid_gpu_plan_ring_kind(const grid_gpu_plan* plan, int* kind, uint32_t* aux_moduli);
/* Host-only: validate (q, d) exactly like grid_gpu_plan_create and return the
 * plan's parameters and merged twiddles without touching a device. Any output
 * pointer may be NULL (zeta/izeta: d words each). */
int grid_gpu_plan_describe(uint64_t q, uint64_t d, grid_gpu_plan_info* info, uint32_t* zeta,
                           uint32_t* izeta);
int grid_gpu_plan_get_info(const grid_gpu_plan* plan, grid_gpu_plan_info* out);
/* Host copy of the merged-NTT twiddle tables (d words each, index 0 unused):
 * zeta[k] = psi^brv(k), izeta[k] = zeta[k]^-1 (Montgomery words). */
int grid_gpu_plan_get_twiddles(const grid_gpu_plan* plan, uint32_t* zeta, uint32_t* izeta);
/* Reads and clears the plan's device error word (GRID_ERR_TIMEOUT if a
 * bounded device wait gave up since the last check). Synchronises `stream`. */
int grid_gpu_plan_check(grid_gpu_plan* plan, void* stream);
/* Test support for the failure path (no counterpart in the reference, whose
 * CPU code has no device waits): one warp waits on an mbarrier that nothing
 * arrives at, giving up after max_spins polls (1 .. 2^22) exactly as a stalled
 * kernel's bounded wait does, which records a timeout in the plan's error
 * word. The next grid_gpu_plan_check returns GRID_ERR_TIMEOUT and clears it;
 * the plan stays usable. */
int grid_gpu_selftest_wait_timeout_dev(const grid_gpu_plan* plan, uint32_t max_spins,
                                       void* stream);

/* ---- NTT: replace NTTRing::ntt_{forward,inverse}_with_plan for twisted plans
 *      (algebra/src/poly/ntt.rs:75-104, arith/prime.rs:617-637) ------------- */

int grid_gpu_ntt_forward_dev(const grid_gpu_plan* plan, uint32_t* polys, size_t npolys,
                             void* stream);
int grid_gpu_ntt_inverse_dev(const grid_gpu_plan* plan, uint32_t* polys, size_t npolys,
                             void* stream);
/* out = INTT(NTT(a) (.) b_evals): forward twisted NTT, Montgomery pointwise
 * product with evaluations b, inverse twisted NTT. out may alias a. */
int grid_gpu_ntt_mul_inverse_dev(const grid_gpu_plan* plan, const uint32_t* a,
                                 const uint32_t* b_evals, uint32_t* out, size_t npolys,
                                 void* stream);
/* Negacyclic product out = a * b mod (X^d + 1), poly_mul_ntt
 * (algebra/src/poly/ntt.rs:305-319), or the schoolbook product's words on a
 * ring plan without an NTT for q. b_scratch holds
 * grid_gpu_poly_mul_scratch_words(plan, npolys) words (npolys * d on an NTT plan). */
size_t grid_gpu_poly_mul_scratch_words(const grid_gpu_plan* plan, size_t npolys);
int grid_gpu_poly_mul_dev(const grid_gpu_plan* plan, const uint32_t* a, const uint32_t* b,
                          uint32_t* out, uint32_t* b_scratch, size_t npolys, void* stream);
/* Ring::pointwise_mul_assign_slice (algebra/src/arith/prime.rs:433-447): dst *= rhs. */
int grid_gpu_pointwise_mul_dev(const grid_gpu_plan* plan, uint32_t* dst, const uint32_t* rhs,
                               size_t nwords, void* stream);
/* The other slice hooks of Ring for PrimeField (algebra/src/arith/prime.rs:433-491):
 * add_assign_slice dst += src, sub_assign_slice dst -= src, scalar_mul_slice
 * dst *= scalar, add_assign_scaled_slice dst += src * scalar, and dot_product
 * (*out = sum lhs_i * rhs_i, one word in device memory). Canonical words;
 * scalar >= q returns GRID_ERR_INVALID_PARAMETERS. */
int grid_gpu_add_assign_dev(const grid_gpu_plan* plan, uint32_t* dst, const uint32_t* src,
                            size_t nwords, void* stream);
int grid_gpu_sub_assign_dev(const grid_gpu_plan* plan, uint32_t* dst, const uint32_t* src,
                            size_t nwords, void* stream);
int grid_gpu_scalar_mul_dev(const grid_gpu_plan* plan, uint32_t* dst, uint32_t scalar,
                            size_t nwords, void* stream);
int grid_gpu_add_assign_scaled_dev(const grid_gpu_plan* plan, uint32_t* dst, const uint32_t* src,
                                   uint32_t scalar, size_t nwords, void* stream);
int grid_gpu_dot_product_dev(const grid_gpu_plan* plan, const uint32_t* lhs, const uint32_t* rhs,
                             size_t nwords, uint32_t* out, void* stream);
/* The reference's default limb: PrimeField<Q> = PrimeField<Q, u64> stores
 * value * 2^64 mod q in a u64 (algebra/src/arith/prime.rs:24-29); this library
 * computes on u32 words value * 2^32 mod q. A u64 caller converts at the
 * boundary (HBM-bound, 12 bytes per word): from_u64 maps each canonical u64 word
 * to its u32 word and sets *noncanonical (device int, optional) to 1 if a word
 * was >= q; to_u64 maps u32 words back. Outputs equal the u64 words the
 * reference's arithmetic produces. */
int grid_gpu_words_from_u64_dev(const grid_gpu_plan* plan, const uint64_t* in, size_t nwords,
                                uint32_t* out, int* noncanonical, void* stream);
int grid_gpu_words_to_u64_dev(const grid_gpu_plan* plan, const uint32_t* in, size_t nwords,
                              uint64_t* out, void* stream);

int grid_gpu_ntt_forward(grid_gpu_plan* plan, uint32_t* polys, size_t npolys);
int grid_gpu_ntt_inverse(grid_gpu_plan* plan, uint32_t* polys, size_t npolys);
int grid_gpu_ntt_mul_inverse(grid_gpu_plan* plan, const uint32_t* a, const uint32_t* b_evals,
                             uint32_t* out, size_t npolys);
int grid_gpu_poly_mul(grid_gpu_plan* plan, const uint32_t* a, const uint32_t* b, uint32_t* out,
                      size_t npolys);

/* ---- prepared matrices: the device-resident key cache of
 *      PreparedLinearOps::build_linear_key_cache / build_matrix_cache
 *      (commit/src/linear.rs:576-631, 690-715) ---------------------------- */

/* Upload a rows x cols ring matrix (row-major polys) and keep its twisted
 * evaluations resident on the device. a_is_evals = 1 takes A already in the
 * evaluation domain (TwistedNttPoly::from_evals, poly/twisted_ntt.rs:47-49). */
int grid_gpu_matrix_create(grid_gpu_plan* plan, const uint32_t* A, size_t rows, size_t cols,
                           int a_is_evals, grid_gpu_matrix** out);
int grid_gpu_matrix_create_dev(grid_gpu_plan* plan, const uint32_t* A, size_t rows, size_t cols,
                               int a_is_evals, grid_gpu_matrix** out, void* stream);
int grid_gpu_matrix_destroy(grid_gpu_matrix* m);
/* A view of the first `cols` columns of a prepared matrix (shares its device
 * evaluations; destroy the view before the parent). */
int grid_gpu_matrix_view(const grid_gpu_matrix* parent, size_t cols, grid_gpu_matrix** out);
int grid_gpu_matrix_shape(const grid_gpu_matrix* m, size_t* rows, size_t* cols);
int grid_gpu_matrix_device_evals(const grid_gpu_matrix* m, const uint32_t** evals);

/* ---- commitments: t = A * s, replacing mul_matrix_vector_runtime /
 *      CommitKey::inner_commit_slice (commit/src/linear.rs:459-473,
 *      labrador/src/crs.rs:211-216) ---------------------------------------- */

/* s: batch x cols coefficient polys; t: batch x rows coefficient polys. */
int grid_gpu_commit_workspace(const grid_gpu_matrix* A, size_t batch, size_t* bytes);
int grid_gpu_commit_dev(const grid_gpu_matrix* A, const uint32_t* s, size_t batch, uint32_t* t,
                        void* workspace, size_t workspace_bytes, void* stream);
int grid_gpu_commit(grid_gpu_matrix* A, const uint32_t* s, size_t batch, uint32_t* t);
/* t = A_msg * m + A_open * r per batch entry: recompute_linear_commitment_parts_trusted
 * (commit/src/linear.rs:476-506). Ajtai with a zero opening is grid_gpu_commit. */
int grid_gpu_linear_commit(grid_gpu_matrix* A_msg, grid_gpu_matrix* A_open, const uint32_t* m,
                           const uint32_t* r, size_t batch, uint32_t* t);
int grid_gpu_linear_commit_workspace(const grid_gpu_matrix* A_msg, const grid_gpu_matrix* A_open,
                                     size_t batch, size_t* bytes);
int grid_gpu_linear_commit_dev(const grid_gpu_matrix* A_msg, const grid_gpu_matrix* A_open,
                               const uint32_t* m, const uint32_t* r, size_t batch, uint32_t* t,
                               void* workspace, size_t workspace_bytes, void* stream);

/* ---- BDLOP parts: recompute_bdlop_parts_runtime (commit/src/linear.rs:552-573,
 *      800-938): u = A_mask * r and v = A_msg * m + A_open * r per batch entry
 *      (A_mask and A_open share the randomness: equal column counts). ------- */
int grid_gpu_bdlop_workspace(const grid_gpu_matrix* A_mask, const grid_gpu_matrix* A_msg,
                             const grid_gpu_matrix* A_open, size_t batch, size_t* bytes);
int grid_gpu_bdlop_commit_dev(const grid_gpu_matrix* A_mask, const grid_gpu_matrix* A_msg,
                              const grid_gpu_matrix* A_open, const uint32_t* m, const uint32_t* r,
                              size_t batch, uint32_t* u, uint32_t* v, void* workspace,
                              size_t workspace_bytes, void* stream);
int grid_gpu_bdlop_commit(grid_gpu_matrix* A_mask, grid_gpu_matrix* A_msg, grid_gpu_matrix* A_open,
                          const uint32_t* m, const uint32_t* r, size_t batch, uint32_t* u,
                          uint32_t* v);

/* ---- Gram matrix: compute_garbage_g (labrador/src/main_protocol/garbage.rs:76-93)
 *      G[idx(i,j)] = <s_i, s_j> for i <= j, row-major upper triangle
 *      (garbage_index, main_protocol/mod.rs:664-670). S: r x n polys. ------- */

int grid_gpu_gram_workspace(const grid_gpu_plan* plan, size_t r, size_t n, size_t* bytes);
int grid_gpu_gram_dev(const grid_gpu_plan* plan, const uint32_t* S, size_t r, size_t n,
                      uint32_t* G, void* workspace, size_t workspace_bytes, void* stream);
int grid_gpu_gram(grid_gpu_plan* plan, const uint32_t* S, size_t r, size_t n, uint32_t* G);

/* ---- uniform ring elements: CommitKey::from_seed / sample_uniform_mat
 *      (labrador/src/crs.rs:136-198, 308-326) with PrimeField::rand
 *      (algebra/src/arith/prime.rs:730-743): npolys ring elements drawn in
 *      order from ChaCha20Rng(seed) (rand_chacha 0.10.0), Montgomery words.
 *      The commitment key's A, B, C, D are consecutive spans of one call.
 *      accept_max = 0 uses the reference's rejection threshold; another value
 *      replaces it (rejections then become frequent; for testing that path). */
int grid_gpu_sample_uniform_polys_workspace(const grid_gpu_plan* plan, size_t npolys,
                                            uint64_t accept_max, size_t* bytes);
int grid_gpu_sample_uniform_polys_dev(const grid_gpu_plan* plan, const uint8_t* seed, size_t npolys,
                                      uint64_t accept_max, uint32_t* out, void* workspace,
                                      size_t workspace_bytes, void* stream);
int grid_gpu_sample_uniform_polys(grid_gpu_plan* plan, const uint8_t* seed, size_t npolys,
                                  uint64_t accept_max, uint32_t* out);

/* ---- JL evaluations, aggregation side: jl_rows_flat_to_conjugated_polys +
 *      the jl_evals loop of prove_step (labrador/src/main_protocol/mod.rs:885-923,
 *      step_prover.rs:185-206): evals[m] = sum_{i,j} conj(pi_{m,i,j}) * s_{i,j}
 *      for the rows x (num_parts * cols) JL matrix of `seed`, straight from the
 *      keystream (the int8 entries are never stored). evals: rows x d words.
 *      Kernel shape: rows = 256, d = 64 (else GRID_ERR_UNSUPPORTED_SIZE). -- */
int grid_gpu_jl_evals_workspace(size_t* bytes);
int grid_gpu_jl_evals_dev(const grid_gpu_plan* plan, const uint8_t* seed, size_t rows,
                          const uint32_t* parts, size_t num_parts, size_t cols, size_t d,
                          uint32_t* evals, void* workspace, size_t workspace_bytes, void* stream);
int grid_gpu_jl_evals(grid_gpu_plan* plan, const uint8_t* seed, size_t rows, const uint32_t* parts,
                      size_t num_parts, size_t cols, size_t d, uint32_t* evals);

/* ---- garbage h: compute_garbage_h (labrador/src/main_protocol/garbage.rs:101-133)
 *      H[idx(i,j)] = (<phi_i, s_j> + <phi_j, s_i>) * 2^-1 for i <= j, row-major upper
 *      triangle (garbage_index, main_protocol/mod.rs:664-670). S, Phi: r x n polys. */
int grid_gpu_garbage_h_workspace(const grid_gpu_plan* plan, size_t r, size_t n, size_t* bytes);
int grid_gpu_garbage_h_dev(const grid_gpu_plan* plan, const uint32_t* S, const uint32_t* Phi,
                           size_t r, size_t n, uint32_t* H, void* workspace,
                           size_t workspace_bytes, void* stream);
int grid_gpu_garbage_h(grid_gpu_plan* plan, const uint32_t* S, const uint32_t* Phi, size_t r,
                       size_t n, uint32_t* H);

/* ---- amortized witness: compute_amortized_witness
 *      (labrador/src/main_protocol/amortization.rs:61-84) without the challenge
 *      sampling, which stays with the transcript on the host:
 *      z[k] = sum_i c_i * s_i[k]. S: r x n polys, c: r polys, z: n polys. */
int grid_gpu_amortize_workspace(const grid_gpu_plan* plan, size_t r, size_t n, size_t* bytes);
int grid_gpu_amortize_dev(const grid_gpu_plan* plan, const uint32_t* S, const uint32_t* c,
                          size_t r, size_t n, uint32_t* z, void* workspace,
                          size_t workspace_bytes, void* stream);
int grid_gpu_amortize(grid_gpu_plan* plan, const uint32_t* S, const uint32_t* c, size_t r,
                      size_t n, uint32_t* z);

/* ---- JL projection: JLMatrix::project_and_extract_jl_rows (labrador/src/jl.rs:267-303)
 *      seed: 32 bytes; parts: num_parts x cols words; rows <= 256; p_out: rows words;
 *      flat_out (optional, NULL to skip): rows*num_parts*cols int8 in the
 *      reference's [row][part][coeff][poly] order, cols = n*d. ---------------- */

int grid_gpu_jl_workspace(size_t rows, size_t* bytes);
int grid_gpu_jl_project_dev(const grid_gpu_plan* plan, const uint8_t* seed, size_t rows,
                            const uint32_t* parts, size_t num_parts, size_t cols, size_t d,
                            uint32_t* p_out, int8_t* flat_out, void* workspace,
                            size_t workspace_bytes, void* stream);
int grid_gpu_jl_project(grid_gpu_plan* plan, const uint8_t* seed, size_t rows,
                        const uint32_t* parts, size_t num_parts, size_t cols, size_t d,
                        uint32_t* p_out, int8_t* flat_out);

/* ---- decompositions ------------------------------------------------------ */

/* decompose_polys (labrador/src/main_protocol/mod.rs:731-747): out is
 * npolys x num_limbs x d, limbs centered in [-base/2, base/2] stored mod q. */
int grid_gpu_decompose_balanced_dev(const grid_gpu_plan* plan, const uint32_t* polys,
                                    size_t npolys, uint64_t base, size_t num_limbs,
                                    uint32_t* out, void* stream);
int grid_gpu_decompose_balanced(grid_gpu_plan* plan, const uint32_t* polys, size_t npolys,
                                uint64_t base, size_t num_limbs, uint32_t* out);
/* Number of unsigned base-`base` digits of q - 1 (decomposition.rs:9-22). */
int grid_gpu_gadget_digits(uint64_t q, uint64_t base, size_t* digits);
/* gadget_decompose (algebra/src/poly/decomposition.rs:47-61): digit_major = 1
 * gives out[digit][len]; 0 gives GadgetRing::decompose_element order
 * out[poly][digit][coeff] (commit/src/gadget/mod.rs:151-162, len % d == 0). */
int grid_gpu_gadget_decompose_dev(const grid_gpu_plan* plan, const uint32_t* x, size_t len,
                                  uint64_t base, int digit_major, uint32_t* out, void* stream);
int grid_gpu_gadget_decompose(grid_gpu_plan* plan, const uint32_t* x, size_t len, uint64_t base,
                              int digit_major, uint32_t* out);

/* ---- uneven batched commitments: many AjtaiCommitmentScheme::commit calls
 *      (commit/src/ajtai/mod.rs:429-441) of different lengths in one launch
 *      sequence (NTT of all witnesses, the persistent grouped product on the
 *      tensor cores, one launch per tile class, then fold and INTT) --
 * Instance i commits s_i (n polys starting at poly s_offset of the packed
 * witness buffer) with the first n columns of matrix `matrix` (rows <= 32)
 * and writes rows polys starting at poly t_offset of the packed output. */
typedef struct grid_gpu_batch grid_gpu_batch;
typedef struct grid_gpu_batch_item {
  uint64_t s_offset;
  uint64_t t_offset;
  uint32_t n;
  uint32_t matrix;
} grid_gpu_batch_item;
/* Engines of the grouped product: POINT_MAJOR runs the tensor cores over
 * point-major evaluations (the witnesses' transform stores [point][poly], each
 * instance at its own 128-aligned columns; every matrix needs its point-major
 * copy: d = 64, rows <= 32, cols a multiple of 4; k_split a multiple of 32;
 * else GRID_ERR_UNSUPPORTED_DEGREE / GRID_ERR_INVALID_PARAMETERS); TENSOR runs
 * them over gathered poly-major evaluations (d % 4 == 0, tensor-core plan,
 * else GRID_ERR_UNSUPPORTED_DEGREE); CUDA_CORE never uses them; AUTO =
 * POINT_MAJOR where it applies, else TENSOR where the plan allows, else
 * CUDA_CORE. All give the same words. */
enum {
  GRID_GPU_ENGINE_AUTO = 0,
  GRID_GPU_ENGINE_TENSOR = 1,
  GRID_GPU_ENGINE_CUDA_CORE = 2,
  GRID_GPU_ENGINE_POINT_MAJOR = 3
};
typedef struct grid_gpu_batch_config {
  uint32_t k_split;        /* K range of one work item (multiple of 16, <= 8192) */
  uint32_t work_items;     /* output of get_config */
  uint32_t tiles;          /* output of get_config */
  uint32_t tile_instances; /* instances per tile (multiple of 4, <= 128); 0: the engine's */
  uint32_t engine;         /* GRID_GPU_ENGINE_* */
  uint32_t tensor_cores;   /* output of get_config: 1 if the grouped product runs on them */
} grid_gpu_batch_config;
int grid_gpu_batch_create(grid_gpu_plan* plan, grid_gpu_matrix* const* mats, size_t nmats,
                          const grid_gpu_batch_item* items, size_t nitems, grid_gpu_batch** out);
int grid_gpu_batch_destroy(grid_gpu_batch* batch);
int grid_gpu_batch_set_config(grid_gpu_batch* batch, const grid_gpu_batch_config* cfg);
int grid_gpu_batch_get_config(const grid_gpu_batch* batch, grid_gpu_batch_config* cfg);
/* Polys the packed witness / output buffers must hold. */
int grid_gpu_batch_shape(const grid_gpu_batch* batch, uint64_t* s_polys, uint64_t* t_polys);
int grid_gpu_batch_workspace(const grid_gpu_batch* batch, size_t* bytes);
int grid_gpu_batch_commit_dev(grid_gpu_batch* batch, const uint32_t* s, uint32_t* t,
                              void* workspace, size_t workspace_bytes, void* stream);
/* Same work, captured once per (s, t, workspace, stream) into a CUDA graph and
 * replayed; `stream` must be a non-default stream. */
int grid_gpu_batch_commit_graph(grid_gpu_batch* batch, const uint32_t* s, uint32_t* t,
                                void* workspace, size_t workspace_bytes, void* stream);
/* One-shot form for request loops: no handle and no device allocation; the
 * work tables are built on the host and copied into the caller's workspace.
 * k_split 0 lets the library pick the K range from the batch's size (about
 * four work items per SM, at most 8192); both calls must get the same value. */
int grid_gpu_batch_oneshot_workspace(grid_gpu_plan* plan, grid_gpu_matrix* const* mats,
                                     size_t nmats, const grid_gpu_batch_item* items,
                                     size_t nitems, uint32_t k_split, size_t* bytes);
int grid_gpu_batch_commit_oneshot_dev(grid_gpu_plan* plan, grid_gpu_matrix* const* mats,
                                      size_t nmats, const grid_gpu_batch_item* items,
                                      size_t nitems, uint32_t k_split, const uint32_t* s,
                                      uint32_t* t, void* workspace, size_t workspace_bytes,
                                      void* stream);

/* ---- batched Gram matrices: compute_garbage_g (labrador/src/main_protocol/
 *      garbage.rs:76-93) for many witnesses of different rank r <= 64 and
 *      length n in one launch sequence (the witnesses' transforms, one
 *      persistent grouped tensor-core product per tile class, one fold, one
 *      inverse transform). Item i's witness is r x n polys at poly s_offset of S;
 *      its r(r+1)/2 Gram polys (garbage_index order) follow item i-1's in G.
 *      k_split: K words per work item (0: chosen from the batch's size). On a
 *      plan without tensor-core products the items run one grid_gpu_gram_dev
 *      after another in the same workspace. ---------------------------------- */
typedef struct grid_gpu_gram_item {
  uint64_t s_offset;
  uint32_t r;
  uint32_t n;
} grid_gpu_gram_item;
int grid_gpu_batch_gram_workspace(const grid_gpu_plan* plan, const grid_gpu_gram_item* items,
                                  size_t nitems, uint32_t k_split, size_t* bytes);
int grid_gpu_batch_gram_dev(const grid_gpu_plan* plan, const uint32_t* S,
                            const grid_gpu_gram_item* items, size_t nitems, uint32_t k_split,
                            uint32_t* G, void* workspace, size_t workspace_bytes, void* stream);

/* ---- Gram matrix without allocation (no counterpart in the reference) ----
 * Same result as grid_gpu_gram_dev, for callers that cannot allocate device
 * memory (a latency-bound prover loop, where cudaMalloc would synchronise the
 * device, or a plugin whose host owns the memory pool): the scratch comes from
 * a buffer compiled into the library, grid_gpu_noalloc_scratch_bytes() bytes
 * (48 MiB) on every GPU that loads it, held until exit. Problems needing more
 * (grid_gpu_gram_workspace) return GRID_ERR_SCRATCH_LIMIT. The first call on a
 * device looks up the buffer's device address (cudaGetSymbolAddress); make that
 * first call before any stream capture. All calls share the buffer: calls
 * that overlap on the GPU race, so order them (for example on one stream).
 * The current device must be the plan's (else GRID_ERR_INVALID_PARAMETERS);
 * the looked-up address does not survive cudaDeviceReset. */
size_t grid_gpu_noalloc_scratch_bytes(void);
int grid_gpu_gram_noalloc_dev(const grid_gpu_plan* plan, const uint32_t* S, size_t r, size_t n,
                              uint32_t* G, void* stream);

/* ---- fused LaBRADOR prover round: the hot calls of prove_step
 *      (labrador/src/main_protocol/step_prover.rs:118-170) on one witness ----
 * A: kappa x n (CommitKey::a), S: r x n coefficient polys. Outputs:
 *   t_limbs  r*kappa*t1 polys  inner_commit_decomposed (crs.rs:225-256)
 *   g        r(r+1)/2 polys    compute_garbage_g
 *   g_limbs  r(r+1)/2*t2 polys decompose_polys(g, b2, t2)       (NULL: skip)
 *   p_out    jl_rows words     JL projection with jl_seed        (NULL: skip)
 *   jl_flat  jl_rows*r*n*d i8  extracted JL entries              (NULL: skip)
 * The witness is moved to the evaluation domain once and shared by the
 * commitment and the Gram matrix. */
int grid_gpu_prover_round_workspace(const grid_gpu_matrix* A, size_t r, size_t jl_rows,
                                    size_t* bytes);
int grid_gpu_prover_round_dev(const grid_gpu_matrix* A, const uint32_t* S, size_t r,
                              uint64_t b1, size_t t1, uint64_t b2, size_t t2,
                              const uint8_t* jl_seed, size_t jl_rows, uint32_t* t_limbs,
                              uint32_t* g, uint32_t* g_limbs, uint32_t* p_out, int8_t* jl_flat,
                              void* workspace, size_t workspace_bytes, void* stream);

/* ---- host memory ------------------------------------------------------ */

/* Page-lock a caller buffer so host-buffer calls can DMA it asynchronously. */
int grid_gpu_host_register(void* ptr, size_t bytes);
int grid_gpu_host_unregister(void* ptr);

#ifdef __cplusplus
}
#endif
#endif /* GRID_GPU_H */
