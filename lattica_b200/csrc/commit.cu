// Evaluation-domain modular matrix products: the Ajtai commitment t = A * s
// and the LaBRADOR Gram matrix g_ij = <s_i, s_j>.
//
// Reference paths replaced:
//   PreparedLinearOps::recompute_linear_commitment_runtime / mul_matrix_vector
//     (commit/src/linear.rs:459-506, 690-770): prepare (NTT) the vector, a
//     TwistedNttPoly::dot_product per row (algebra/src/poly/twisted_ntt.rs:378-408),
//     finish (INTT).
//   CommitKey::inner_commit_slice (labrador/src/crs.rs:211-216) and
//   compute_garbage_g (labrador/src/main_protocol/garbage.rs:76-93), which in
//   the reference pay three NTTs (or an O(d^2) schoolbook product) per ring
//   product; here the witness is transformed once and each output is one INTT.
//
// In the twisted evaluation domain a ring product is pointwise, so the work
// is d independent dense modular matmuls, one per evaluation point e:
//     out_e[m][n] = sum_k X[m][k][e] * Y[n][k][e]   (mod q, Montgomery)
// Kernel "emm": a CTA owns 8 consecutive evaluation points (one 32-byte
// sector per (row, k)), a 32 x 32 (or 64 x 16) output tile and a K range;
// operands stream through shared memory in 16-deep K chunks; each thread keeps a 4 x 8
// register tile of exact 96-bit accumulators (64-bit product added to a 64-bit
// sum, carries counted in a third word) and reduces once at the end.
// Partial sums of a K split are canonical residues, so splits add exactly.
#include <cuda_runtime.h>

#include "grid_async.cuh"
#include "grid_field.cuh"
#include "grid_internal.h"

namespace grid {
namespace {

constexpr int EG = 8, KC = 16;
// Words per staged row: 16 K steps x 8 evaluation points, padded by 2 so that
// rows 4 apart start 8 banks apart.
constexpr int RS = KC * EG + 2;
constexpr int kEmmThreads = 256;

enum OutMode : int { OUT_DENSE = 0, OUT_UPPER = 1 };

// Output tile of a CTA: TMG groups of 4 rows of X by (32 / TMG) groups of 8
// rows of Y, for 8 evaluation points; each of the 256 threads keeps one
// evaluation point of a 4 x 8 sub-tile. TMG = 8 is the square 32 x 32 tile;
// TMG = 16 (64 x 16) fits the short Y of a commitment (kappa = 16 rows of A).
template <int TMG>
struct EmmTile {
  static constexpr int TNG = 32 / TMG;
  static constexpr int BM = 4 * TMG, BN = 8 * TNG;
  static constexpr int STAGE_WORDS = (BM + BN) * RS;
  static constexpr int STAGES = 3;
  static constexpr size_t SMEM = (size_t)STAGES * STAGE_WORDS * 4;
};

// X: [M][K][d], Y: [N][ldy][d] (first K of ldy columns used). Dense output:
// [M][N][d]; upper output (X == Y, M == N): packed upper triangle i <= j in
// row-major order (garbage_index).
// With splits > 1 the CTA of split s writes to out + s * split_stride.
// Operands stream through a cp.async ring of STAGES chunks (X rows, then Y
// rows, each in global order: [k][e]); one CTA per SM, so the 4 x 8 tile of
// 96-bit accumulators stays in registers without spilling. A warp covers 8
// evaluation points x 4 consecutive row groups of X, so its X reads hit 32
// distinct banks and its Y reads are broadcasts.
template <int TMG>
__global__ void __launch_bounds__(kEmmThreads, 1) emm_kernel(
    const uint32_t* __restrict__ X, const uint32_t* __restrict__ Y, uint32_t* __restrict__ out,
    int M, int N, int K, int ldy, int d, int mode, int k_per_split, size_t split_stride,
    FieldParams f) {
  using Tl = EmmTile<TMG>;
  constexpr int BM = Tl::BM, BN = Tl::BN, STAGES = Tl::STAGES;
  constexpr int SW = Tl::STAGE_WORDS;
  extern __shared__ __align__(16) uint32_t emm_smem[];

  const int tiles_n = (N + BN - 1) / BN;
  int ti = (int)blockIdx.y / tiles_n, tj = (int)blockIdx.y % tiles_n;
  if (mode == OUT_UPPER) {
    // Square tiles; blockIdx.y enumerates the tiles ti <= tj row by row.
    int u = (int)blockIdx.y;
    ti = 0;
    while (u >= tiles_n - ti) u -= tiles_n - ti++;
    tj = ti + u;
  }
  const int tm0 = ti * BM;
  const int tn0 = tj * BN;
  const int e0 = blockIdx.x * EG;
  const int split = blockIdx.z;
  const int kbeg = split * k_per_split;
  const int kend = min(K, kbeg + k_per_split);
  const int nchunks = kend > kbeg ? (kend - kbeg + KC - 1) / KC : 0;

  const int t = threadIdx.x;
  const int eg = t & 7;
  const int tm = (t >> 3) % TMG;
  const int tn = (t >> 3) / TMG;

  // Copy chunk c (K steps kbeg + 16c ..) into stage c % STAGES as 8-byte
  // pieces, one half row per warp; rows past M / N and steps past kend are
  // zero-filled.
  auto issue = [&](int c) {
    uint32_t* st = emm_smem + (c % STAGES) * SW;
    const int k0 = kbeg + c * KC;
#pragma unroll
    for (int i = 0; i < (BM + BN) / 4; ++i) {
      const int u = t + kEmmThreads * i;  // (row, kk, quarter)
      const int quarter = u & 3;
      const int kk = (u >> 2) & (KC - 1);
      const int row = u >> 6;
      const int k = k0 + kk;
      const uint32_t* src = X;
      bool valid;
      if (row < BM) {  // uniform per i: BM is a multiple of 4
        const int m = tm0 + row;
        valid = k < kend && m < M;
        if (valid) src = X + ((size_t)m * K + k) * d + e0 + quarter * 2;
      } else {
        const int n = tn0 + row - BM;
        valid = k < kend && n < N;
        if (valid) src = Y + ((size_t)n * ldy + k) * d + e0 + quarter * 2;
      }
      cp_async8(st + row * RS + kk * EG + quarter * 2, src, valid ? 8u : 0u);
    }
  };

  Acc96 acc[4][8];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 8; ++j) acc96_zero(acc[i][j]);

  // This thread's words: X rows tm*4 + i and Y rows BM + tn*8 + j, step kk,
  // evaluation point eg.
  const int xo = (tm * 4) * RS + eg;
  const int yo = (BM + tn * 8) * RS + eg;

#pragma unroll
  for (int c = 0; c < STAGES - 1; ++c) {
    if (c < nchunks) issue(c);
    cp_async_commit();
  }
  for (int c = 0; c < nchunks; ++c) {
    cp_async_wait<STAGES - 2>();
    __syncthreads();  // chunk c landed for every thread; stage (c - 1) % STAGES is free
    if (c + STAGES - 1 < nchunks) issue(c + STAGES - 1);
    cp_async_commit();
    const uint32_t* xs = emm_smem + (c % STAGES) * SW + xo;
    const uint32_t* ys = emm_smem + (c % STAGES) * SW + yo;
#pragma unroll
    for (int kk = 0; kk < KC; ++kk) {
      uint32_t xr[4], yr[8];
#pragma unroll
      for (int i = 0; i < 4; ++i) xr[i] = xs[kk * EG + i * RS];
#pragma unroll
      for (int j = 0; j < 8; ++j) yr[j] = ys[kk * EG + j * RS];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc96_mad(acc[i][j], xr[i], yr[j]);
    }
  }
  cp_async_wait<0>();

  const int e = e0 + eg;
  uint32_t* o = out + (size_t)split * split_stride;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int m = tm0 + tm * 4 + i;
    if (m >= M) continue;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int n = tn0 + tn * 8 + j;
      if (n >= N) continue;
      const uint32_t v = acc96_reduce(acc[i][j], f);
      if (mode == OUT_DENSE) {
        o[((size_t)m * N + n) * d + e] = v;
      } else if (m <= n) {
        const size_t idx = (size_t)m * M - ((size_t)m * (m - 1)) / 2 + (size_t)(n - m);
        o[idx * d + e] = v;
      }
    }
  }
}

constexpr int kMvMaxRows = 4;
constexpr int kMvThreads = 256;

// Products with at most four X rows (a matrix times one to four vectors, e.g.
// an outer commitment or a single commit): one thread per (Y row n,
// evaluation point e) keeps the M accumulators. Consecutive threads read
// consecutive evaluation points, so Y streams through once, coalesced, and the
// few X words are shared through L1 / L2; the tiled kernel would spend all but
// M of its 32 or 64 tile rows on padding here.
__global__ void __launch_bounds__(kMvThreads) emv_kernel(
    const uint32_t* __restrict__ X, const uint32_t* __restrict__ Y, uint32_t* __restrict__ out,
    int M, int N, int K, int ldy, int d, int k_per_split, size_t split_stride, FieldParams f) {
  const size_t w = (size_t)blockIdx.x * kMvThreads + threadIdx.x;
  if (w >= (size_t)N * d) return;
  const int n = (int)(w / d), e = (int)(w % d);
  const int kbeg = (int)blockIdx.y * k_per_split;
  const int kend = min(K, kbeg + k_per_split);
  Acc96 acc[kMvMaxRows];
#pragma unroll
  for (int m = 0; m < kMvMaxRows; ++m) acc96_zero(acc[m]);
  const uint32_t* yp = Y + (size_t)n * ldy * d + e;
  const uint32_t* xp = X + e;
#pragma unroll 4
  for (int k = kbeg; k < kend; ++k) {
    const uint32_t y = __ldg(yp + (size_t)k * d);
#pragma unroll
    for (int m = 0; m < kMvMaxRows; ++m)
      if (m < M) acc96_mad(acc[m], __ldg(xp + ((size_t)m * K + k) * d), y);
  }
  uint32_t* o = out + (size_t)blockIdx.y * split_stride;
#pragma unroll
  for (int m = 0; m < kMvMaxRows; ++m)
    if (m < M) o[((size_t)m * N + n) * d + e] = acc96_reduce(acc[m], f);
}

// out[i] = sum_s part[s][i] mod q (exact; partials are canonical).
__global__ void sum_splits_kernel(const uint32_t* __restrict__ part, uint32_t* __restrict__ out,
                                  size_t n, int splits, uint32_t q) {
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    uint32_t v = part[i];
    for (int s = 1; s < splits; ++s) v = add_mod(v, part[(size_t)s * n + i], q);
    out[i] = v;
  }
}

// Launch geometry of one product: tile shape, tiles and the K split.
struct EmmGeometry {
  bool mv;  // emv_kernel (dense, M <= kMvMaxRows) instead of the tiled kernel
  int tmg, tiles_m, tiles_n;
  int tiles;  // tiled kernel: output tiles; emv_kernel: 256-thread blocks over (N, d)
  int splits, k_per_split;
};

// The K range is split so that all CTAs fit one wave of the resident slots
// (one CTA per SM), each split a whole number of 16-step chunks and at least
// two of them; split partials go to the workspace and are summed after.
EmmGeometry emm_geometry(int M, int N, int K, int d, int mode, int num_sms) {
  EmmGeometry g;
  g.mv = mode == OUT_DENSE && M <= kMvMaxRows;
  if (g.mv) {
    // memory bound: about four 256-thread CTAs per SM, at least 32 K steps each
    const long long blocks = ((long long)N * d + kMvThreads - 1) / kMvThreads;
    long long want = 4LL * num_sms / blocks;
    if (want > K / 32) want = K / 32;
    if (want < 1) want = 1;
    g.k_per_split = (int)((K + want - 1) / want);
    g.splits = (K + g.k_per_split - 1) / g.k_per_split;
    g.tmg = g.tiles_m = g.tiles_n = 0;
    g.tiles = (int)blocks;
    return g;
  }
  g.tmg = (mode == OUT_DENSE && N <= 16) ? 16 : 8;
  const int bm = 4 * g.tmg, bn = 8 * (32 / g.tmg);
  g.tiles_m = (M + bm - 1) / bm;
  g.tiles_n = (N + bn - 1) / bn;
  g.tiles = mode == OUT_UPPER ? g.tiles_m * (g.tiles_m + 1) / 2 : g.tiles_m * g.tiles_n;
  const long long ctas = (long long)(d / EG) * g.tiles;
  const long long slots = num_sms;
  const int chunks = (K + KC - 1) / KC;
  long long want = ctas >= slots ? 1 : slots / ctas;
  if (want > chunks / 2) want = chunks / 2 > 1 ? chunks / 2 : 1;
  const int cps = (int)((chunks + want - 1) / want);  // chunks per split
  g.splits = (chunks + cps - 1) / cps;
  g.k_per_split = cps * KC;
  return g;
}

template <int TMG>
int launch_emm_tile(dim3 grid, const uint32_t* X, const uint32_t* Y, uint32_t* dst, int M, int N,
                    int K, int ldy, int mode, const EmmGeometry& g, size_t stride,
                    const grid_gpu_plan* p, cudaStream_t s) {
  static int bps_cache[kMaxDevices] = {};
  int bps = 0;
  const int rc = prepare_kernel(emm_kernel<TMG>, EmmTile<TMG>::SMEM, kEmmThreads, p->device,
                                bps_cache, &bps);
  if (rc) return rc;
  emm_kernel<TMG><<<grid, kEmmThreads, EmmTile<TMG>::SMEM, s>>>(
      X, Y, dst, M, N, K, ldy, (int)p->d, mode, g.k_per_split, stride, p->f);
  return GRID_OK;
}

}  // namespace

size_t emm_workspace_words(const grid_gpu_plan* p, int M, int N, int K, int mode) {
  if (M <= 0 || N <= 0 || K <= 0 || p->d % EG) return 0;
  const EmmGeometry g = emm_geometry(M, N, K, (int)p->d, mode, p->num_sms);
  EmmTcGeometry tg;
  const int splits = !g.mv && emm_tc_geometry(p, M, N, K, mode, &tg) ? tg.splits : g.splits;
  const size_t outputs = mode == OUT_UPPER ? (size_t)M * (M + 1) / 2 : (size_t)M * N;
  const size_t words = splits > 1 ? (size_t)splits * outputs * p->d : 0;
  const size_t pm = emm_pm_workspace_words(p, M, N, K, mode);  // point-major operands
  return words > pm ? words : pm;
}

// out_evals: dense [M][N][d] or packed-upper [M(M+1)/2][d]. work: >= emm_workspace_words.
int launch_emm(const grid_gpu_plan* p, const uint32_t* X, const uint32_t* Y, int M, int N, int K,
               int ldy, int mode, uint32_t* out_evals, uint32_t* work, cudaStream_t s) {
  if (is_crt(p)) return p->ntt_status;  // evaluation-domain products need an NTT for q
  if (M <= 0 || N <= 0 || K <= 0) return GRID_OK;
  if (p->d % EG) return GRID_ERR_UNSUPPORTED_DEGREE;
  if (mode == OUT_UPPER && M != N) return GRID_ERR_DIMENSION_MISMATCH;
  const EmmGeometry g = emm_geometry(M, N, K, (int)p->d, mode, p->num_sms);
  EmmTcGeometry tg;
  const bool tc = !g.mv && emm_tc_geometry(p, M, N, K, mode, &tg);
  const int splits = tc ? tg.splits : g.splits;
  const size_t outputs = mode == OUT_UPPER ? (size_t)M * (M + 1) / 2 : (size_t)M * N;
  const size_t stride = outputs * p->d;
  uint32_t* dst = splits > 1 ? work : out_evals;
  if (splits > 1 && !work) return GRID_ERR_NULL_POINTER;
  int rc = GRID_OK;
  if (tc) {
    rc = launch_emm_tc(p, X, Y, M, N, K, ldy, mode, dst, tg, stride, s);
  } else if (g.mv) {
    emv_kernel<<<dim3((unsigned)g.tiles, splits), kMvThreads, 0, s>>>(
        X, Y, dst, M, N, K, ldy, (int)p->d, g.k_per_split, stride, p->f);
  } else {
    dim3 grid(p->d / EG, g.tiles, splits);
    rc = g.tmg == 16 ? launch_emm_tile<16>(grid, X, Y, dst, M, N, K, ldy, mode, g, stride, p, s)
                     : launch_emm_tile<8>(grid, X, Y, dst, M, N, K, ldy, mode, g, stride, p, s);
  }
  if (rc) return rc;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_status(e);
  return splits > 1 ? launch_sum_splits(p, work, out_evals, stride, splits, s) : GRID_OK;
}

int launch_sum_splits(const grid_gpu_plan* p, const uint32_t* work, uint32_t* out, size_t stride,
                      int splits, cudaStream_t s) {
  size_t blocks = (stride + 255) / 256;
  if (blocks > (size_t)p->num_sms * 8) blocks = (size_t)p->num_sms * 8;
  sum_splits_kernel<<<(unsigned)blocks, 256, 0, s>>>(work, out, stride, splits, p->f.q);
  return cuda_status(cudaGetLastError());
}

namespace {

// out[e][i] = in[i][e]: 32 x 32 tiles through shared memory.
__global__ void to_point_major_kernel(const uint32_t* __restrict__ in, uint32_t* __restrict__ out,
                                      size_t npolys, int d) {
  __shared__ uint32_t t[32][33];
  const size_t i0 = (size_t)blockIdx.x * 32;
  const int e0 = blockIdx.y * 32;
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const size_t i = i0 + r;
    const int e = e0 + threadIdx.x;
    if (i < npolys && e < d) t[r][threadIdx.x] = in[i * d + e];
  }
  __syncthreads();
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int e = e0 + r;
    const size_t i = i0 + threadIdx.x;
    if (i < npolys && e < d) out[(size_t)e * npolys + i] = t[threadIdx.x][r];
  }
}

}  // namespace

int launch_to_point_major(const uint32_t* in, uint32_t* out, size_t npolys, int d,
                          cudaStream_t s) {
  if (npolys == 0) return GRID_OK;
  const size_t bx = (npolys + 31) / 32;
  if (bx > 0x7fffffffu) return GRID_ERR_INVALID_PARAMETERS;
  to_point_major_kernel<<<dim3((unsigned)bx, (d + 31) / 32), dim3(32, 8), 0, s>>>(in, out, npolys,
                                                                                   d);
  return cuda_status(cudaGetLastError());
}

}  // namespace grid
