// Internal host-side declarations shared by the CUDA translation units.
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include <mutex>
#include <vector>

#include "../../include/grid_gpu.h"
#include "grid_field.cuh"

namespace grid {

// Merged (twist-folded) negacyclic NTT twiddles for one (q, d).
// zeta[k] = psi^brv(k) for k in [1, d), psi the primitive 2d-th root used by
// the reference (smallest generator g, psi = g^((q-1)/2d)); izeta[k] is its
// inverse. Each entry is a Montgomery word plus its Shoup companion
// w * q^-1 mod 2^32.
struct TwiddleTable {
  std::vector<uint32_t> zeta, zeta_q, izeta, izeta_q;  // index 0 unused
  uint32_t ninv = 0, ninv_q = 0;                       // d^-1
  uint32_t izeta1_ninv = 0, izeta1_ninv_q = 0;         // izeta[1] * d^-1
};

// Largest d for which kernels are compiled.
constexpr uint32_t kMaxDegree = 256;

// Kernel-parameter copy of the twiddles for thread-per-poly kernels (d <= 64).
template <int D>
struct Tw1 {
  FieldParams f;
  uint32_t fw[D][2];
  uint32_t iw[D][2];
  uint32_t ninv[2];
  uint32_t iw1n[2];
};

enum NttMode : int {
  MODE_FWD = 0,     // coefficients -> twisted evaluations (natural order)
  MODE_INV = 1,     // twisted evaluations -> coefficients
  MODE_MULINV = 2,  // out = INTT(NTT(a) (.) b_evals)
  MODE_POLYMUL = 3, // out = INTT(NTT(a) (.) NTT(b))  (negacyclic product)
  MODE_FWD_PM = 4,  // MODE_FWD stored point-major: out[e * ps + poly], ps = npolys rounded
                    // up to a multiple of 4, pad polys zero (d = 64 tensor cores)
};

struct DeviceScratch {
  void* ptr = nullptr;
  size_t bytes = 0;
};

// Constants of the exact reconstruction of ring_crt.cu: residues mod the three
// auxiliary primes -> the Montgomery word mod q.
struct CrtConsts {
  uint32_t p[3], pinv[3];   // auxiliary primes, their inverses mod 2^32
  uint32_t r2_0;            // 2^64 mod p0
  uint32_t c1a, c1b;        // 2^64 p0^-1, 2^32 p0^-1 (mod p1)
  uint32_t c2a, c2b, c2c;   // 2^64 (p0 p1)^-1, 2^32 (p0 p1)^-1, 2^32 p1^-1 (mod p2)
  uint32_t half_p2;         // p2 / 2: the sign threshold of the top mixed-radix digit
  FieldParams fq;           // the ring's modulus q
  uint32_t m1, m2, p_rinv;  // p0, p0 p1 (mod q); P 2^-32 (mod q)
};

}  // namespace grid

struct grid_gpu_plan {
  uint32_t q = 0, d = 0, log_d = 0;
  int device = 0;
  grid::FieldParams f{};
  uint32_t generator = 0, psi = 0, omega = 0, n_inv = 0;  // Montgomery words
  uint64_t psi_value = 0, n_inv_value = 0;                 // the same, canonical integers
  grid::TwiddleTable tw;
  // Device copy of the twiddle table as uint2 {w, wq}: fw[d], iw[d], {ninv}, {izeta1*ninv}.
  uint2* d_tw = nullptr;
  // Tensor-core tables. d = 64: byte planes of the Montgomery-form forward /
  // inverse matrices (2 x 64 KB). d = 256: the 64-point matrix (64 KB) and the
  // twist constants of the products. Null selects the CUDA-core kernels.
  void* d_tcw = nullptr;
  bool tc_emm = false;  // evaluation-domain products on the tensor cores where the shape allows
  bool pm_emm = false;  // ... over point-major evaluations loaded by TMA (emm_pm.cu)
  int* d_err = nullptr;
  cudaStream_t stream = nullptr;   // host-buffer entry points: first pipeline stream
  cudaStream_t stream2 = nullptr;  // second pipeline stream
  // Forked work of *_dev calls (joined back into the caller's stream through
  // events): the highest-priority stream for the critical path, the lowest for
  // the independent work that fills the SMs around it.
  cudaStream_t fork_hi = nullptr, fork_lo = nullptr;
  std::mutex mu;                   // serialises host-buffer calls and scratch growth
  grid::DeviceScratch scratch[16];
  int num_sms = 0;
  // Ring plans for a q without a 2d-th root of unity (ring_crt.cu): ordinary
  // plans for the three auxiliary primes carry the products; null otherwise.
  grid_gpu_plan* crt[3] = {nullptr, nullptr, nullptr};
  grid::CrtConsts crt_c{};
  int ntt_status = 0;  // what TwistedNttPlan::build reports for (q, d) on a ring plan
};

struct grid_gpu_matrix {
  grid_gpu_plan* plan = nullptr;
  size_t rows = 0, cols = 0;
  size_t ld = 0;                // row stride in polys (cols of the owning matrix)
  uint32_t* d_evals = nullptr;  // rows x ld polys in the twisted evaluation domain
  // The same evaluations point-major, [d][rows][ld], for the tensor-core
  // contraction over TMA-loaded operands (null where that path does not apply).
  uint32_t* d_evals_pm = nullptr;
  bool owned = true;            // false for views sharing another matrix's evaluations
  // On a ring plan without an NTT for q: the matrix's residues mod each
  // auxiliary prime, prepared on that prime's plan (d_evals stays null).
  grid_gpu_matrix* crt[3] = {nullptr, nullptr, nullptr};
};

namespace grid {

// ntt.cu
int launch_ntt(const grid_gpu_plan* p, int mode, const uint32_t* a, const uint32_t* b,
               uint32_t* out, size_t npolys, cudaStream_t s);
int ntt_max_degree();
// One-launch commitment t = A s for small shapes (d = 64, rows <= 32, cols <= 128,
// batch <= 1024): transform, contraction and inverse in one kernel.
bool commit_small_fits(const grid_gpu_plan* p, size_t rows, size_t cols, size_t batch);
int launch_commit_small(const grid_gpu_plan* p, const uint32_t* A_evals, size_t rows,
                        size_t cols, size_t ld, const uint32_t* s, size_t batch, uint32_t* t,
                        cudaStream_t st);
// ntt_tc.cu (d = 64, tcgen05)
bool ntt_tc_available(const grid_gpu_plan* p);
int launch_ntt_tc(const grid_gpu_plan* p, int mode, const uint32_t* a, const uint32_t* b,
                  uint32_t* out, size_t npolys, cudaStream_t s);
void build_tc_tables(uint32_t q, uint32_t d, uint64_t psi, uint64_t ninv,
                     std::vector<unsigned char>& out);
// MODE_FWD_PM over a tile list: tile t transforms the 128 polys from source
// row ptiles[t].x of a (npolys polys) into columns ptiles[t].y .. + 127 of
// out [64][ps_out], polys from ptiles[t].z of the tile on as zeros. Columns
// are multiples of 4 and tiles do not overlap.
int launch_ntt_tc_pm_tiles(const grid_gpu_plan* p, const uint32_t* a, size_t npolys,
                           uint32_t* out, unsigned long long ps_out, const uint4* ptiles,
                           unsigned long long nptiles, cudaStream_t s);
// ntt256_tc.cu (d = 256 products, tcgen05)
bool ntt256_tc_available(const grid_gpu_plan* p);
int launch_ntt256_tc(const grid_gpu_plan* p, const uint32_t* a, const uint32_t* b, uint32_t* out,
                     size_t npolys, cudaStream_t s);
void build_tc256_tables(uint32_t q, uint64_t psi, std::vector<unsigned char>& out);

// commit.cu: out_e[m][n] = sum_k X[m][k][e] * Y[n][k][e] for every evaluation point.
enum EmmOut : int { EMM_DENSE = 0, EMM_UPPER = 1 };
size_t emm_workspace_words(const grid_gpu_plan* p, int M, int N, int K, int mode);
int launch_emm(const grid_gpu_plan* p, const uint32_t* X, const uint32_t* Y, int M, int N, int K,
               int ldy, int mode, uint32_t* out_evals, uint32_t* work, cudaStream_t s);
int launch_pointwise(const grid_gpu_plan* p, uint32_t* dst, const uint32_t* rhs, size_t words,
                     cudaStream_t s);
// emm_tc.cu: the same products on the tensor cores (X rows <= 128, Y rows <= 64).
struct EmmTcGeometry {
  int np;           // Y rows padded to 16, 32, 48 or 64
  int groups;       // CTAs along the evaluation points
  int splits, k_per_split;
};
bool emm_tc_geometry(const grid_gpu_plan* p, int M, int N, int K, int mode, EmmTcGeometry* g);
int launch_emm_tc(const grid_gpu_plan* p, const uint32_t* X, const uint32_t* Y, int M, int N,
                  int K, int ldy, int mode, uint32_t* dst, const EmmTcGeometry& g, size_t stride,
                  cudaStream_t s);
// out[i] = sum over splits s of work[s * stride + i] (mod q)
int launch_sum_splits(const grid_gpu_plan* p, const uint32_t* work, uint32_t* out, size_t stride,
                      int splits, cudaStream_t s);
// emm_pm.cu: the same products over point-major operands, X [d][M][K] and
// Y [d][N][ldy] (tensor cores, TMA; X rows <= 128, Y rows <= 64, K and ldy
// multiples of 4, 16-byte aligned bases). Split partials go to `work`.
struct EmmPmGeometry {
  int np;  // Y rows padded to 16, 32, 48 or 64
  int splits, k_per_split;
};
bool emm_pm_geometry(const grid_gpu_plan* p, int M, int N, int K, int ldy, int mode,
                     EmmPmGeometry* g);
size_t emm_pm_workspace_words(const grid_gpu_plan* p, int M, int N, int K, int mode);
int launch_emm_pm(const grid_gpu_plan* p, const uint32_t* X, const uint32_t* Y, int M, int N,
                  int K, int ldy, int mode, uint32_t* out_evals, uint32_t* work, cudaStream_t s);
// in [npolys][d] -> out [d][npolys] (point-major copy of evaluations)
int launch_to_point_major(const uint32_t* in, uint32_t* out, size_t npolys, int d,
                          cudaStream_t s);
// garbage.cu: (C_ij + C_ji) * 2^-1 on the upper triangle; z_hat = sum_i c_hat_i (.) s_hat_i.
int launch_symmetrize_half(const grid_gpu_plan* p, const uint32_t* C, int r, uint32_t* H,
                           cudaStream_t s);
int launch_amortize(const grid_gpu_plan* p, const uint32_t* c_hat, const uint32_t* s_hat, int r,
                    size_t n, uint32_t* z_hat, cudaStream_t s);
int launch_add(const grid_gpu_plan* p, uint32_t* dst, const uint32_t* rhs, size_t words,
               cudaStream_t s);

// decompose.cu
int launch_decompose_balanced(const grid_gpu_plan* p, const uint32_t* polys, size_t npolys,
                              uint64_t base, size_t num_limbs, uint32_t* out, cudaStream_t s);
int launch_gadget_decompose(const grid_gpu_plan* p, const uint32_t* x, size_t len, uint64_t base,
                            size_t digits, int digit_major, uint32_t* out, cudaStream_t s);
size_t gadget_digit_count(uint64_t q, uint64_t base);

// jl.cu
int launch_jl_project(const FieldParams& f, const uint8_t seed[32], size_t rows,
                      const uint32_t* parts, size_t num_parts, size_t cols, size_t d,
                      uint32_t* p_out, int8_t* flat_out, void* scratch, size_t scratch_bytes,
                      int num_sms, int* d_err, cudaStream_t s);
size_t jl_scratch_bytes(size_t rows, size_t num_parts, int num_sms);
// crs.cu: `count` uniform Montgomery words from ChaCha20Rng(seed) (accept_max 0:
// the reference's rejection threshold).
size_t sample_uniform_workspace_bytes(uint32_t q, unsigned long long count,
                                      unsigned long long accept_max);
int launch_sample_uniform(const grid_gpu_plan* p, const uint8_t seed[32], unsigned long long count,
                          unsigned long long accept_max, uint32_t* out, void* ws, size_t ws_bytes,
                          cudaStream_t s);
// JL evaluations sum conj(pi_{m,i,j}) s_{i,j} (rows = 256, d = 64 only).
size_t jl_evals_scratch_bytes();
int launch_jl_evals(const FieldParams& f, const uint8_t seed[32], size_t rows,
                    const uint32_t* parts, size_t num_parts, size_t cols, size_t d,
                    uint32_t* evals, void* scratch, size_t scratch_bytes, int num_sms, int* err,
                    cudaStream_t s);

// ring_crt.cu: exact products for q without a 2d-th root (three auxiliary primes)
inline bool is_crt(const grid_gpu_plan* p) { return p->crt[0] != nullptr; }
const uint32_t* crt_moduli();
void crt_consts(uint32_t q, CrtConsts* c);
// terms * d * (q - 1)^2 < 2^93: every output coefficient sums at most terms * d
// word products, within the reconstruction's range
bool crt_bound_ok(const grid_gpu_plan* p, size_t terms);
// o_j = x mod p_j (null outputs skipped); words % 4 == 0, 16-byte aligned buffers
int crt_lift(const grid_gpu_plan* p, const uint32_t* x, size_t words, uint32_t* o0, uint32_t* o1,
             uint32_t* o2, cudaStream_t s);
// out = Montgomery word mod q of the integer whose words mod p_j are w_j
int crt_combine(const grid_gpu_plan* p, const uint32_t* w0, const uint32_t* w1,
                const uint32_t* w2, size_t words, uint32_t* out, cudaStream_t s);

// plan.cu
int host_pipeline(grid_gpu_plan* p, const uint32_t* const* ins, int nin, uint32_t* out,
                  size_t nunits, size_t unit_words,
                  int (*op)(grid_gpu_plan*, const uint32_t* const*, uint32_t*, size_t,
                            cudaStream_t, void*),
                  void* ctx);
int finish_host_call(grid_gpu_plan* p, cudaStream_t s);

// helpers
int cuda_status(cudaError_t e);
int ensure_scratch(grid_gpu_plan* p, int slot, size_t bytes);

constexpr int kMaxDevices = 64;

inline size_t round_up(size_t x, size_t a) { return (x + a - 1) / a * a; }
inline size_t words_bytes(size_t words) { return round_up(words * 4, 256); }

// Bump allocator over a caller workspace (256-byte aligned sub-buffers).
struct Carver {
  char* base;
  size_t cap, used = 0;
  bool ok = true;
  Carver(void* b, size_t c) : base(static_cast<char*>(b)), cap(c) {}
  template <typename T>
  T* take(size_t count) {
    if (count > (cap + 1) / sizeof(T)) {  // also keeps count * sizeof(T) from wrapping
      ok = false;
      return nullptr;
    }
    const size_t bytes = round_up(count * sizeof(T), 256);
    if (used + bytes > cap || !base) {
      ok = false;
      used += bytes;
      return nullptr;
    }
    T* p = reinterpret_cast<T*>(base + used);
    used += bytes;
    return p;
  }
};

// Sets the dynamic shared-memory limit of `kernel` once per device and caches
// its resident blocks per SM (idempotent; benign if two threads race).
// max_shared: prefer the largest shared-memory carveout, for kernels meant to
// run two CTAs of about half the SM's shared memory each.
template <typename K>
int prepare_kernel(K kernel, size_t smem, int threads, int dev, int* cache, int* bps_out,
                   bool max_shared = false) {
  if (dev < 0 || dev >= kMaxDevices) return GRID_ERR_INVALID_PARAMETERS;
  if (cache[dev] == 0) {
    cudaError_t e =
        cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess && max_shared)
      e = cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                               (int)cudaSharedmemCarveoutMaxShared);
    if (e != cudaSuccess) return cuda_status(e);
    int bps = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, kernel, threads, smem);
    if (e != cudaSuccess) return cuda_status(e);
    cache[dev] = bps < 1 ? 1 : bps;
  }
  *bps_out = cache[dev];
  return GRID_OK;
}

}  // namespace grid
