// Evaluation-domain products on the tensor cores (tcgen05, kind::i8):
//     out_e[m][n] = sum_k X[m][k][e] * Y[n][k][e] * 2^-32 (mod q)
// for every evaluation point e, the contraction behind the Ajtai commitment,
// the Gram matrix and garbage h (commit.cu has the CUDA-core kernels and the
// reference paths they replace).
//
// Per evaluation point this is an integer matrix product on Montgomery words,
// done exactly with u8 MMAs by the byte-plane method of the transforms
// (ntt_tc_common.cuh), with Y in the role of the constant matrix:
//  * A (128 rows x 4K bytes, K-major): row m holds the words X[m][k][e] in
//    natural byte order, byte 4k + i = byte i of x_k (rows >= M are zero);
//  * B (4 NP rows x 4K bytes): row l NP + n, byte 4k + i = byte l of
//    Y^(i)[n][k] = 2^(8i) y mod q (rows n >= N are zero), so that
//    D[m][l NP + n] = sum_{k,i} byte_i(x_k) byte_l(Y^(i)_k) and
//    sum_l 2^(8l) D_l = sum_k x_k y_k (mod q); one Montgomery reduction of that
//    sum gives the canonical word. D < 4 K 255^2 stays below 2^31 for K <= 8192
//    per CTA (the K range is split beyond that and the partials are summed).
// A CTA takes EPC consecutive evaluation points and a K range; its 512 threads
// gather the operands of each 32-word K chunk from global memory (the words of
// one (row, k) for the CTA's evaluation points are contiguous: one vector
// load), into one of two register buffers sized for the shape (X rows <= MX,
// Y rows <= NP), so that chunk c + 1's loads are in flight while chunk c is
// scaled, byte-transposed and written as two 128-byte-swizzled tiles into one
// of two shared-memory stages; thread 0 issues 4 MMAs (M 128, N 4 NP, K 32) per
// evaluation point and commits them to the stage's mbarrier, which the
// producers wait on before they reuse the stage. Tensor memory holds the EPC
// accumulators (4 NP columns each); the epilogue combines the planes, reduces
// and stores. Every wait is bounded.
#include <cuda_runtime.h>

#include "grid_async.cuh"
#include "grid_field.cuh"
#include "grid_internal.h"
#include "grid_tc.cuh"
#include "ntt_tc_common.cuh"

namespace grid {
namespace {

using namespace tcx;

constexpr int kEtThreads = 512;
constexpr int KCH = 32;                // K words per chunk: one 128-byte swizzled row
constexpr uint32_t ABOX = 128u * 128;  // A tile of one evaluation point: 128 rows x 128 bytes
constexpr int kEtMaxK = 8192;          // K words per CTA: 4 * 8192 * 255^2 < 2^31
enum : int { ET_DENSE = 0, ET_UPPER = 1 };

template <int NP>
struct EtShape {
  static constexpr int NMMA = 4 * NP;               // B rows (4 byte planes)
  static constexpr uint32_t BBOX = NMMA * 128u;
  static constexpr int EPC = NP == 16 ? 4 : 2;      // evaluation points per CTA
  static constexpr uint32_t STAGE = EPC * (ABOX + BBOX);
  static constexpr uint32_t SMEM = 2 * STAGE + 64 + 1024;  // two stages, barriers, alignment
  static constexpr uint32_t TCOLS = EPC * NMMA <= 256 ? 256u : 512u;
};

// EPC consecutive words, loaded with one vector access (e0 is a multiple of EPC).
template <int EPC> struct EtWords;
template <> struct EtWords<2> { using type = uint2; };
template <> struct EtWords<4> { using type = uint4; };

template <int NP, int MX>
__global__ void __launch_bounds__(kEtThreads, 1)
    emm_tc_kernel(const uint32_t* __restrict__ X, const uint32_t* __restrict__ Y,
                  uint32_t* __restrict__ out, int M, int N, int K, int ldy, int d, int mode,
                  int k_per_split, size_t split_stride, uint4 scale, const TcConsts k,
                  bool vec, int* __restrict__ err) {
  using S = EtShape<NP>;
  constexpr int EPC = S::EPC, NMMA = S::NMMA;
  extern __shared__ __align__(1024) unsigned char sm_raw[];
  const uint32_t raw = smem_addr(sm_raw);
  unsigned char* sm = sm_raw + (((raw + 1023u) & ~1023u) - raw);
  const uint32_t s0 = smem_addr(sm);
  uint64_t* bars = reinterpret_cast<uint64_t*>(sm + 2 * S::STAGE);
  uint32_t* taddr_slot = reinterpret_cast<uint32_t*>(bars + 2);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int e0 = blockIdx.x * EPC;
  const int split = blockIdx.y;
  const int kbeg = split * k_per_split;
  const int kend = min(K, kbeg + k_per_split);
  const int nch = kend > kbeg ? (kend - kbeg + KCH - 1) / KCH : 0;
  const bool upper = mode == ET_UPPER;  // X == Y: the gathered words feed both tiles

  // rows past M (A) and past N (each plane of B) stay zero in both stages
  for (uint32_t i = tid; i < 2 * S::STAGE / 16; i += kEtThreads)
    reinterpret_cast<uint4*>(sm)[i] = make_uint4(0, 0, 0, 0);
  if (warp == 0) {
    tc::tmem_alloc(taddr_slot, S::TCOLS);
    tc::tmem_relinquish();
  }
  if (tid == 0) {
    mbar_init(&bars[0], 1);
    mbar_init(&bars[1], 1);
    fence_mbar_init();
  }
  tc::fence_async_smem();
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tbase = *taddr_slot;
  const uint32_t idesc = tc::idesc_u8(128, NMMA);

  // B row l NP + n, K word kk: bytes l of 2^(8i) y mod q for i = 0 .. 3
  auto put_b = [&](unsigned char* bbox, int n, int kk, uint32_t y) {
    const uint32_t y1 = mont_mul(y, scale.x, k.q, k.qinv);  // 2^8 y
    const uint32_t y2 = mont_mul(y, scale.y, k.q, k.qinv);  // 2^16 y
    const uint32_t y3 = mont_mul(y, scale.z, k.q, k.qinv);  // 2^24 y
    const uint32_t lo = __byte_perm(y, y1, 0x5140), hi = __byte_perm(y2, y3, 0x5140);
    const uint32_t lo2 = __byte_perm(y, y1, 0x7362), hi2 = __byte_perm(y2, y3, 0x7362);
    const uint32_t w[4] = {__byte_perm(lo, hi, 0x5410), __byte_perm(lo, hi, 0x7632),
                           __byte_perm(lo2, hi2, 0x5410), __byte_perm(lo2, hi2, 0x7632)};
#pragma unroll
    for (int l = 0; l < 4; ++l)
      *reinterpret_cast<uint32_t*>(bbox + sw128(l * NP + n, 0, kk >> 2, S::BBOX) + 4 * (kk & 3)) =
          w[l];
  };

  // (row, k) units per thread: X has at most MX rows, Y at most NP
  constexpr int kUnitsX = MX * KCH / kEtThreads, kUnitsY = NP * KCH / kEtThreads;
  using Words = typename EtWords<EPC>::type;
  struct Regs {
    uint32_t x[kUnitsX][EPC], y[kUnitsY][EPC];
  };
  auto gather_rows = [&](const uint32_t* src, int rows, int ld, int k0, auto& dst) {
    constexpr int kUnits = sizeof(dst) / sizeof(dst[0]);
#pragma unroll
    for (int it = 0; it < kUnits; ++it) {
      const int u = tid + it * kEtThreads;
      const int r = u >> 5, kg = k0 + (u & (KCH - 1));
      Words w{};
      uint32_t* wv = reinterpret_cast<uint32_t*>(&w);
      if (u < rows * KCH && kg < kend) {
        const uint32_t* a = src + ((size_t)r * ld + kg) * d + e0;
        if (vec) {
          w = *reinterpret_cast<const Words*>(a);
        } else {
#pragma unroll
          for (int el = 0; el < EPC; ++el) wv[el] = a[el];
        }
      }
#pragma unroll
      for (int el = 0; el < EPC; ++el) dst[it][el] = wv[el];
    }
  };
  // issue every load of chunk c (one vector load of the CTA's EPC adjacent
  // evaluation points per (row, k)); nothing waits on them until put_chunk
  auto gather_chunk = [&](int c, Regs& r) {
    const int k0 = kbeg + c * KCH;
    gather_rows(X, M, K, k0, r.x);
    if (!upper) gather_rows(Y, N, ldy, k0, r.y);
  };
  // write chunk c's tiles into its stage, then thread 0 issues its MMAs
  auto put_chunk = [&](int c, const Regs& r) -> bool {
    const int st = c & 1;
    unsigned char* stage = sm + st * S::STAGE;
    // the MMAs of chunk c - 2 must be done reading this stage
    if (c >= 2 && !__syncthreads_and(mbar_wait(&bars[st], ((c - 2) >> 1) & 1, err))) return false;
#pragma unroll
    for (int it = 0; it < kUnitsX; ++it) {
      const int u = tid + it * kEtThreads;
      if (u >= M * KCH) break;
      const int m = u >> 5, kk = u & (KCH - 1);
#pragma unroll
      for (int el = 0; el < EPC; ++el) {
        *reinterpret_cast<uint32_t*>(stage + el * ABOX + sw128(m, 0, kk >> 2, ABOX) + 4 * (kk & 3)) =
            r.x[it][el];
        if (upper) put_b(stage + EPC * ABOX + el * S::BBOX, m, kk, r.x[it][el]);
      }
    }
    if (!upper) {
#pragma unroll
      for (int it = 0; it < kUnitsY; ++it) {
        const int u = tid + it * kEtThreads;
        if (u >= N * KCH) break;
        const int n = u >> 5, kk = u & (KCH - 1);
#pragma unroll
        for (int el = 0; el < EPC; ++el)
          put_b(stage + EPC * ABOX + el * S::BBOX, n, kk, r.y[it][el]);
      }
    }
    tc::fence_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    if (tid == 0) {
      tc::fence_after_sync();
      const uint32_t sa = s0 + st * S::STAGE;
#pragma unroll
      for (int el = 0; el < EPC; ++el)
#pragma unroll
        for (int s = 0; s < 4; ++s)
          tc::mma_u8(tbase + el * NMMA, desc_sw128(sa + el * ABOX + 32 * s),
                     desc_sw128(sa + EPC * ABOX + el * S::BBOX + 32 * s), idesc, (c | s) != 0);
      tc::mma_commit(&bars[st]);
    }
    return true;
  };

  // two register buffers in turn: chunk c + 1's loads are in flight while
  // chunk c is transposed into shared memory
  bool ok = true;
  Regs ra, rb;
  if (nch > 0) gather_chunk(0, ra);
  for (int c = 0; c < nch; c += 2) {
    if (c + 1 < nch) gather_chunk(c + 1, rb);
    if (!(ok = put_chunk(c, ra)) || c + 1 >= nch) break;
    if (c + 2 < nch) gather_chunk(c + 2, ra);
    if (!(ok = put_chunk(c + 1, rb))) break;
  }
  // the last commit covers every MMA issued before it
  if (ok && nch > 0) ok = mbar_wait(&bars[(nch - 1) & 1], ((nch - 1) >> 1) & 1, err);
  ok = __syncthreads_and(ok);
  tc::fence_after_sync();
  if (ok) {
    const int m = 32 * (warp & 3) + lane;
    uint32_t* o = out + (size_t)split * split_stride;
    for (int el = warp >> 2; el < EPC; el += kEtThreads / 128) {
      const uint32_t taddr = tc::tmem_addr(tbase, 32 * (warp & 3), el * NMMA);
      const int e = e0 + el;
#pragma unroll 1
      for (int n0 = 0; n0 < NP; n0 += 8) {
        uint32_t eb[4][8];
#pragma unroll
        for (int l = 0; l < 4; ++l) tc::tmem_ld8(taddr + l * NP + n0, eb[l]);
        tc::tmem_ld_wait32(eb);
        if (m >= M) continue;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          const int n = n0 + j;
          if (n >= N || (upper && n < m)) continue;
          uint64_t v = mad_wide(eb[1][j], 256u, (uint64_t)eb[0][j]);
          v = mad_wide(eb[2][j], 65536u, v);
          v = mad_wide(eb[3][j], 16777216u, v);
          const uint32_t r = redc64(v, k.q, k.qinv);
          const size_t idx = upper ? (size_t)m * M - ((size_t)m * (m - 1)) / 2 + (size_t)(n - m)
                                   : (size_t)m * N + n;
          o[idx * d + e] = r;
        }
      }
    }
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    tc::fence_after_sync();
    tc::tmem_dealloc(tbase, S::TCOLS);
  }
}

template <int NP, int MX>
int launch_np(const grid_gpu_plan* p, const uint32_t* X, const uint32_t* Y, int M, int N, int K,
              int ldy, int mode, uint32_t* dst, const EmmTcGeometry& g, size_t stride,
              cudaStream_t s) {
  using S = EtShape<NP>;
  static int bps_cache[kMaxDevices] = {};
  int bps = 0;
  const int rc =
      prepare_kernel(emm_tc_kernel<NP, MX>, S::SMEM, kEtThreads, p->device, bps_cache, &bps);
  if (rc) return rc;
  // 2^(8i) R mod q: mont_mul(y, .) = 2^(8i) y mod q
  uint32_t c[3];
  for (int i = 1; i <= 3; ++i)
    c[i - 1] = (uint32_t)(((unsigned __int128)1 << (32 + 8 * i)) % p->f.q);
  TcConsts k;
  k.q = p->f.q;
  k.qinv = p->f.qinv;
  // vector gathers need both operands aligned to the EPC words they load
  const uintptr_t bytes = 4u * S::EPC;
  const bool vec = reinterpret_cast<uintptr_t>(X) % bytes == 0 &&
                   (mode == ET_UPPER || reinterpret_cast<uintptr_t>(Y) % bytes == 0);
  emm_tc_kernel<NP, MX><<<dim3(g.groups, g.splits), kEtThreads, S::SMEM, s>>>(
      X, Y, dst, M, N, K, ldy, (int)p->d, mode, g.k_per_split, stride,
      make_uint4(c[0], c[1], c[2], 0), k, vec, p->d_err);
  return cuda_status(cudaGetLastError());
}

}  // namespace

bool emm_tc_geometry(const grid_gpu_plan* p, int M, int N, int K, int mode, EmmTcGeometry* g) {
  if (!p->tc_emm || M <= 0 || N <= 0 || K <= 0 || M > 128 || N > 64) return false;
  if (mode == ET_UPPER && M != N) return false;
  g->np = N <= 16 ? 16 : N <= 32 ? 32 : N <= 48 ? 48 : 64;
  const int epc = g->np == 16 ? 4 : 2;
  if ((int)p->d % epc) return false;
  g->groups = (int)p->d / epc;
  const int chunks = (K + KCH - 1) / KCH;
  // one CTA per SM (tensor memory and shared memory): split K to fill the SMs,
  // at least 2 chunks per split, at most kEtMaxK words per CTA
  int want = p->num_sms / g->groups;
  if (want > chunks / 2) want = chunks / 2;
  if (want < 1) want = 1;
  int cps = (chunks + want - 1) / want;
  if (cps * KCH > kEtMaxK) cps = kEtMaxK / KCH;
  g->k_per_split = cps * KCH;
  g->splits = (chunks + cps - 1) / cps;
  return true;
}

int launch_emm_tc(const grid_gpu_plan* p, const uint32_t* X, const uint32_t* Y, int M, int N,
                  int K, int ldy, int mode, uint32_t* dst, const EmmTcGeometry& g, size_t stride,
                  cudaStream_t s) {
  // X rows: register buffers sized for 64 or 128
  if (M <= 64) {
    switch (g.np) {
      case 16: return launch_np<16, 64>(p, X, Y, M, N, K, ldy, mode, dst, g, stride, s);
      case 32: return launch_np<32, 64>(p, X, Y, M, N, K, ldy, mode, dst, g, stride, s);
      case 48: return launch_np<48, 64>(p, X, Y, M, N, K, ldy, mode, dst, g, stride, s);
      default: return launch_np<64, 64>(p, X, Y, M, N, K, ldy, mode, dst, g, stride, s);
    }
  }
  switch (g.np) {
    case 16: return launch_np<16, 128>(p, X, Y, M, N, K, ldy, mode, dst, g, stride, s);
    case 32: return launch_np<32, 128>(p, X, Y, M, N, K, ldy, mode, dst, g, stride, s);
    case 48: return launch_np<48, 128>(p, X, Y, M, N, K, ldy, mode, dst, g, stride, s);
    default: return launch_np<64, 128>(p, X, Y, M, N, K, ldy, mode, dst, g, stride, s);
  }
}

}  // namespace grid
