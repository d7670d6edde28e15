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
// sector per (row, k)), a 32 x 32 output tile and a K range; operands are
// staged through shared memory in 16-deep K chunks; each thread keeps a 4 x 8
// register tile of exact 96-bit accumulators (64-bit product added to a 64-bit
// sum, carries counted in a third word) and reduces once at the end.
// Partial sums of a K split are canonical residues, so splits add exactly.
#include <cuda_runtime.h>

#include "grid_field.cuh"
#include "grid_internal.h"

namespace grid {
namespace {

constexpr int BM = 32, BN = 32, EG = 8, KC = 16, PAD = 4;
constexpr int ROWX = BM + PAD;  // words per (k, e) row of the X tile
constexpr int ROWY = BN + PAD;
constexpr int kEmmThreads = 256;

enum OutMode : int { OUT_DENSE = 0, OUT_UPPER = 1 };

// X: [M][K][d], Y: [N][ldy][d] (first K of ldy columns used). Dense output:
// [M][N][d]; upper output (X == Y, M == N): packed upper triangle i <= j in
// row-major order (garbage_index).
// With splits > 1 the CTA of split s writes to out + s * split_stride.
__global__ void __launch_bounds__(kEmmThreads) emm_kernel(
    const uint32_t* __restrict__ X, const uint32_t* __restrict__ Y, uint32_t* __restrict__ out,
    int M, int N, int K, int ldy, int d, int mode, int k_per_split, size_t split_stride,
    FieldParams f) {
  __shared__ __align__(16) uint32_t Xs[KC * EG * ROWX];
  __shared__ __align__(16) uint32_t Ys[KC * EG * ROWY];

  const int tiles_n = (N + BN - 1) / BN;
  const int tile = blockIdx.y;
  const int tm0 = (tile / tiles_n) * BM;
  const int tn0 = (tile % tiles_n) * BN;
  if (mode == OUT_UPPER && tm0 > tn0) return;  // strictly-lower tiles hold no output
  const int e0 = blockIdx.x * EG;
  const int split = blockIdx.z;
  const int kbeg = split * k_per_split;
  const int kend = min(K, kbeg + k_per_split);

  const int t = threadIdx.x;
  const int eg = t & 7;
  const int tn = (t >> 3) & 3;
  const int tm = t >> 5;

  Acc96 acc[4][8];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 8; ++j) acc96_zero(acc[i][j]);

  for (int k0 = kbeg; k0 < kend; k0 += KC) {
    // Stage X[tm0 .. +32][k0 .. +16][e0 .. +8] and the same of Y.
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int u = t + kEmmThreads * i;  // 0 .. 1023: (mm, kk, half)
      const int half = u & 1;
      const int kk = (u >> 1) & (KC - 1);
      const int mm = u >> 5;
      const int k = k0 + kk;
      uint4 vx = make_uint4(0, 0, 0, 0), vy = make_uint4(0, 0, 0, 0);
      if (k < kend) {
        const int m = tm0 + mm, n = tn0 + mm;
        if (m < M)
          vx = *reinterpret_cast<const uint4*>(X + ((size_t)m * K + k) * d + e0 + half * 4);
        if (n < N)
          vy = *reinterpret_cast<const uint4*>(Y + ((size_t)n * ldy + k) * d + e0 + half * 4);
      }
      uint32_t* xs = Xs + (kk * EG + half * 4) * ROWX + mm;
      uint32_t* ys = Ys + (kk * EG + half * 4) * ROWY + mm;
      xs[0] = vx.x; xs[ROWX] = vx.y; xs[2 * ROWX] = vx.z; xs[3 * ROWX] = vx.w;
      ys[0] = vy.x; ys[ROWY] = vy.y; ys[2 * ROWY] = vy.z; ys[3 * ROWY] = vy.w;
    }
    __syncthreads();
#pragma unroll 4
    for (int kk = 0; kk < KC; ++kk) {
      const uint4 xv = *reinterpret_cast<const uint4*>(Xs + (kk * EG + eg) * ROWX + tm * 4);
      const uint4 y0 = *reinterpret_cast<const uint4*>(Ys + (kk * EG + eg) * ROWY + tn * 8);
      const uint4 y1 = *reinterpret_cast<const uint4*>(Ys + (kk * EG + eg) * ROWY + tn * 8 + 4);
      const uint32_t xr[4] = {xv.x, xv.y, xv.z, xv.w};
      const uint32_t yr[8] = {y0.x, y0.y, y0.z, y0.w, y1.x, y1.y, y1.z, y1.w};
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc96_mad(acc[i][j], xr[i], yr[j]);
    }
    __syncthreads();
  }

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

int choose_splits(int ctas, int K, int num_sms) {
  // Enough CTAs for ~2 waves, but keep each split at >= 64 K steps.
  int splits = 1;
  while (ctas * splits < 2 * num_sms && K / (splits * 2) >= 64) splits *= 2;
  return splits;
}

}  // namespace

size_t emm_workspace_words(const grid_gpu_plan* p, int M, int N, int K, int mode) {
  const int tiles = ((M + BM - 1) / BM) * ((N + BN - 1) / BN);
  const int ctas = (int)(p->d / EG) * tiles;
  const int splits = choose_splits(ctas, K, p->num_sms);
  const size_t outputs = mode == OUT_UPPER ? (size_t)M * (M + 1) / 2 : (size_t)M * N;
  return splits > 1 ? (size_t)splits * outputs * p->d : 0;
}

// out_evals: dense [M][N][d] or packed-upper [M(M+1)/2][d]. work: >= emm_workspace_words.
int launch_emm(const grid_gpu_plan* p, const uint32_t* X, const uint32_t* Y, int M, int N, int K,
               int ldy, int mode, uint32_t* out_evals, uint32_t* work, cudaStream_t s) {
  if (M <= 0 || N <= 0 || K <= 0) return GRID_OK;
  if (p->d % EG) return GRID_ERR_UNSUPPORTED_DEGREE;
  const int tiles_m = (M + BM - 1) / BM, tiles_n = (N + BN - 1) / BN;
  const int ctas = (int)(p->d / EG) * tiles_m * tiles_n;
  const int splits = choose_splits(ctas, K, p->num_sms);
  int kps = (K + splits - 1) / splits;
  kps = (kps + KC - 1) / KC * KC;
  const size_t outputs = mode == OUT_UPPER ? (size_t)M * (M + 1) / 2 : (size_t)M * N;
  const size_t stride = outputs * p->d;
  dim3 grid(p->d / EG, tiles_m * tiles_n, splits);
  uint32_t* dst = splits > 1 ? work : out_evals;
  if (splits > 1 && !work) return GRID_ERR_NULL_POINTER;
  emm_kernel<<<grid, kEmmThreads, 0, s>>>(X, Y, dst, M, N, K, ldy, (int)p->d, mode, kps, stride,
                                          p->f);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_status(e);
  if (splits > 1) {
    size_t blocks = (stride + 255) / 256;
    if (blocks > (size_t)p->num_sms * 8) blocks = (size_t)p->num_sms * 8;
    sum_splits_kernel<<<(unsigned)blocks, 256, 0, s>>>(work, out_evals, stride, splits, p->f.q);
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_status(e);
  }
  return GRID_OK;
}

}  // namespace grid
