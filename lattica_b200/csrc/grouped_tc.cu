// Grouped contractions on the tensor cores: many independent products
//     out_e[x][y] = sum_k X[x][k][e] * Y[y][k][e] * 2^-32 (mod q)
// of different shapes in one persistent launch, the tensor-core counterpart of
// batch.cu's CUDA-core kernel. Used for uneven batched commitments (X rows =
// instances of one matrix, each with its own length; Y = the matrix rows) and
// batched Gram matrices of uneven rank (X = Y = one instance's r witness rows,
// upper triangle only).
//
// Each work item (tile, K range, group of EPC evaluation points) runs the
// byte-plane product of emm_tc.cu: per 32-word K chunk the 512 threads gather
// the tile's X rows (per-row base and length; zero past a row's length) and Y
// rows for the item's points into registers (one vector load per (row, k)),
// write them as 128-byte-swizzled A and B tiles (B scaled by 2^(8i) mod q and
// byte-transposed), and thread 0 issues the MMAs (M 128, N 4 NP, K 32) into
// tensor memory, double-buffered through two shared-memory stages guarded by
// mbarriers; chunk c + 1's loads are in flight while chunk c is written. The
// epilogue combines the four byte planes, reduces once (canonical word) and
// adds it into the 64-bit accumulator of its output word, so work items may
// split K. CTAs pull work items from an atomic counter (longest first) and keep
// their tensor memory and barriers for the whole launch; the mbarrier phases
// run on across work items (a CTA-wide chunk counter). Every wait is bounded.
#include <cuda_runtime.h>

#include "batch_tables.cuh"
#include "grid_async.cuh"
#include "grid_field.cuh"
#include "grid_internal.h"
#include "grid_tc.cuh"
#include "ntt_tc_common.cuh"

namespace grid {
namespace {

using namespace tcx;

constexpr int kGtThreads = 512;
constexpr int KCH = 32;                // K words per chunk: one 128-byte swizzled row
constexpr uint32_t ABOX = 128u * 128;  // A tile of one evaluation point: 128 rows x 128 bytes

template <int NP>
struct GtShape {
  static constexpr int NMMA = 4 * NP;                 // B rows (4 byte planes)
  static constexpr uint32_t BBOX = NMMA * 128u;
  static constexpr int EPC = tc_points(NP);           // evaluation points per work item
  static constexpr uint32_t STAGE = EPC * (ABOX + BBOX);
};
constexpr uint32_t kGtStage =
    GtShape<16>::STAGE > GtShape<64>::STAGE ? GtShape<16>::STAGE : GtShape<64>::STAGE;
constexpr uint32_t kGtSmem = 2 * kGtStage + 64 + 1024;  // two stages, barriers, alignment
constexpr uint32_t kGtCols = 512;                         // tensor memory: every NP class
static_assert(2 * GtShape<32>::STAGE <= 2 * kGtStage, "stage size");
static_assert(GtShape<64>::EPC * GtShape<64>::NMMA <= (int)kGtCols, "tensor memory");

template <int EPC> struct GtWords;
template <> struct GtWords<2> { using type = uint2; };
template <> struct GtWords<4> { using type = uint4; };

struct GtCtx {
  unsigned char* sm;        // 1 KB-aligned dynamic shared memory
  uint32_t s0;              // its shared-space address
  uint64_t* bars;           // two stage barriers
  uint32_t tbase;           // tensor-memory base
  uint32_t chunk;           // chunks of this CTA's finished items (stage / parity)
  uint32_t issued;          // chunks whose MMAs this CTA has issued and committed
  uint4 scale;              // 2^(8i) R mod q, i = 1..3
  TcConsts k;
  int d;
  int* err;
};

// One work item with NP padded Y rows and at most MX X rows. Returns false if a
// bounded wait gave up (the CTA then stops taking work).
template <int NP, int MX>
__device__ bool gt_item(const WorkDev& wk, const TileDev& tile, const MatDev& mat,
                        const ItemDev* __restrict__ rows, const uint32_t* __restrict__ s_hat,
                        unsigned long long* __restrict__ acc, GtCtx& cx) {
  using S = GtShape<NP>;
  constexpr int EPC = S::EPC, NMMA = S::NMMA;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const bool upper = tile.matrix == kUpperTile;
  const int M = (int)tile.count;
  const int N = upper ? M : (int)mat.rows;
  const int d = cx.d;
  const int e0 = (int)wk.eg * EPC;
  const uint32_t kbeg = wk.k0, kend = wk.k1;
  const int nch = (int)((kend - kbeg + KCH - 1) / KCH);
  const uint32_t idesc = tc::idesc_u8(128, NMMA);
  unsigned char* sm = cx.sm;
  const TcConsts k = cx.k;
  const uint4 scale = cx.scale;

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

  constexpr int kUnitsX = MX * KCH / kGtThreads, kUnitsY = NP * KCH / kGtThreads;
  using Words = typename GtWords<EPC>::type;
  struct Regs {
    uint32_t x[kUnitsX][EPC], y[kUnitsY > 0 ? kUnitsY : 1][EPC];
  };
  auto gather_chunk = [&](int c, Regs& r) {
    const uint32_t k0 = kbeg + (uint32_t)(c * KCH);
#pragma unroll
    for (int it = 0; it < kUnitsX; ++it) {
      const int u = tid + it * kGtThreads;
      const int m = u >> 5;
      const uint32_t kg = k0 + (uint32_t)(u & (KCH - 1));
      Words w{};
      if (m < M && kg < kend && kg < rows[m].n)
        w = *reinterpret_cast<const Words*>(s_hat + (rows[m].s_off + kg) * (size_t)d + e0);
      const uint32_t* wv = reinterpret_cast<const uint32_t*>(&w);
#pragma unroll
      for (int el = 0; el < EPC; ++el) r.x[it][el] = wv[el];
    }
    if (!upper) {
#pragma unroll
      for (int it = 0; it < kUnitsY; ++it) {
        const int u = tid + it * kGtThreads;
        const int n = u >> 5;
        const uint32_t kg = k0 + (uint32_t)(u & (KCH - 1));
        Words w{};
        if (n < N && kg < kend)
          w = *reinterpret_cast<const Words*>(mat.evals + ((size_t)n * mat.ld + kg) * d + e0);
        const uint32_t* wv = reinterpret_cast<const uint32_t*>(&w);
#pragma unroll
        for (int el = 0; el < EPC; ++el) r.y[it][el] = wv[el];
      }
    }
  };
  auto put_chunk = [&](int c, const Regs& r) -> bool {
    const uint32_t g = cx.chunk + (uint32_t)c;  // CTA-wide chunk index
    const int st = (int)(g & 1u);
    unsigned char* stage = sm + st * kGtStage;
    // the MMAs of chunk g - 2 must be done reading this stage
    if (g >= 2 && !__syncthreads_and(mbar_wait(&cx.bars[st], ((g - 2) >> 1) & 1u, cx.err)))
      return false;
#pragma unroll
    for (int it = 0; it < kUnitsX; ++it) {
      const int u = tid + it * kGtThreads;
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
        const int u = tid + it * kGtThreads;
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
      const uint32_t sa = cx.s0 + st * kGtStage;
#pragma unroll
      for (int el = 0; el < EPC; ++el)
#pragma unroll
        for (int s = 0; s < 4; ++s)
          tc::mma_u8(cx.tbase + el * NMMA, desc_sw128(sa + el * ABOX + 32 * s),
                     desc_sw128(sa + EPC * ABOX + el * S::BBOX + 32 * s), idesc, (c | s) != 0);
      tc::mma_commit(&cx.bars[st]);
    }
    cx.issued = g + 1;
    return true;
  };

  bool ok = true;
  if (nch > 0) {
    Regs ra, rb;
    gather_chunk(0, ra);
    for (int c = 0; c < nch; c += 2) {
      if (c + 1 < nch) gather_chunk(c + 1, rb);
      if (!(ok = put_chunk(c, ra)) || c + 1 >= nch) break;
      if (c + 2 < nch) gather_chunk(c + 2, ra);
      if (!(ok = put_chunk(c + 1, rb))) break;
    }
    // the last commit covers every MMA of the item
    const uint32_t last = cx.chunk + (uint32_t)(nch - 1);
    if (ok) ok = mbar_wait(&cx.bars[last & 1u], (last >> 1) & 1u, cx.err);
    cx.chunk += (uint32_t)nch;
  }
  ok = __syncthreads_and(ok);
  tc::fence_after_sync();
  if (ok && nch > 0) {
    const int m = 32 * (warp & 3) + lane;
    for (int el = warp >> 2; el < EPC; el += kGtThreads / 128) {
      const uint32_t taddr = tc::tmem_addr(cx.tbase, 32 * (warp & 3), el * NMMA);
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
          const unsigned long long poly =
              upper ? rows[0].t_off + (unsigned long long)(m * M - (m * (m - 1)) / 2 + (n - m))
                    : rows[m].t_off + (unsigned long long)n;
          atomicAdd(&acc[poly * (unsigned long long)d + e], (unsigned long long)r);
        }
      }
    }
  }
  // tensor memory and the stages are reused by the next work item
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  return ok;
}

template <int NP, int MX>
__global__ void __launch_bounds__(kGtThreads, 1)
    batch_tc_kernel(const WorkDev* __restrict__ work, unsigned nwork,
                    const TileDev* __restrict__ tiles, const ItemDev* __restrict__ items,
                    const MatDev* __restrict__ mats, const uint32_t* __restrict__ s_hat,
                    unsigned long long* __restrict__ acc, unsigned* __restrict__ counter, int d,
                    uint4 scale, TcConsts k, int* __restrict__ err) {
  extern __shared__ __align__(1024) unsigned char gt_raw[];
  __shared__ ItemDev rows[kTcMaxTileRows];
  __shared__ unsigned widx;
  const uint32_t raw = smem_addr(gt_raw);
  unsigned char* sm = gt_raw + (((raw + 1023u) & ~1023u) - raw);
  uint64_t* bars = reinterpret_cast<uint64_t*>(sm + 2 * kGtStage);
  uint32_t* taddr_slot = reinterpret_cast<uint32_t*>(bars + 2);
  const int tid = threadIdx.x, warp = tid >> 5;
  if (warp == 0) {
    tc::tmem_alloc(taddr_slot, kGtCols);
    tc::tmem_relinquish();
  }
  if (tid == 0) {
    mbar_init(&bars[0], 1);
    mbar_init(&bars[1], 1);
    fence_mbar_init();
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  GtCtx cx{sm, smem_addr(sm), bars, *taddr_slot, 0u, 0u, scale, k, d, err};

  bool ok = true;
  for (;;) {
    if (tid == 0) widx = atomicAdd(counter, 1u);
    __syncthreads();
    const unsigned w = widx;
    if (w >= nwork) break;
    const WorkDev wk = work[w];
    const TileDev tile = tiles[wk.tile];
    const bool upper = tile.matrix == kUpperTile;
    const MatDev mat = upper ? MatDev{nullptr, nullptr, tile.count, 0} : mats[tile.matrix];
    for (int i = tid; i < kTcMaxTileRows; i += kGtThreads) {
      ItemDev it = {0, 0, 0, 0};
      if ((uint32_t)i < tile.count) it = items[tile.first + i];
      rows[i] = it;
    }
    __syncthreads();
    ok = gt_item<NP, MX>(wk, tile, mat, rows, s_hat, acc, cx);
    if (!ok) break;  // a bounded wait gave up: stop taking work (recorded in err)
  }
  // After a timeout, wait (bounded) for the MMAs this CTA committed before the
  // tensor memory is freed; otherwise each item already waited for its last one.
  if (!ok && cx.issued > 0) {
    const uint32_t l = cx.issued - 1;
    mbar_wait(&bars[l & 1u], (l >> 1) & 1u, err);
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    tc::fence_after_sync();
    tc::tmem_dealloc(cx.tbase, kGtCols);
  }
}

template <int NP, int MX>
int launch_class(const grid_gpu_plan* p, const WorkDev* work, unsigned nwork,
                 const TileDev* tiles, const ItemDev* items, const MatDev* mats,
                 const uint32_t* s_hat, unsigned long long* acc, unsigned* counter,
                 uint4 scale, TcConsts k, cudaStream_t s) {
  static int bps_cache[kMaxDevices] = {};
  int bps = 0;
  const int rc =
      prepare_kernel(batch_tc_kernel<NP, MX>, kGtSmem, kGtThreads, p->device, bps_cache, &bps);
  if (rc) return rc;
  unsigned grid = (unsigned)p->num_sms;  // one CTA per SM: all tensor memory and the stages
  if (grid > nwork) grid = nwork;
  batch_tc_kernel<NP, MX><<<grid, kGtThreads, kGtSmem, s>>>(work, nwork, tiles, items, mats,
                                                            s_hat, acc, counter, (int)p->d,
                                                            scale, k, p->d_err);
  return cuda_status(cudaGetLastError());
}

}  // namespace

int tc_class(const TileDev& tile, const MatDev* host_mats) {
  const bool upper = tile.matrix == kUpperTile;
  const uint32_t ny = upper ? tile.count : host_mats[tile.matrix].rows;
  if (upper) return ny <= 16 ? TC_U16 : ny <= 32 ? TC_U32 : TC_U64;
  return ny <= 16 ? TC_D16 : TC_D32;
}

int launch_batch_tc(const grid_gpu_plan* p, int cls, const WorkDev* work, unsigned nwork,
                    const TileDev* tiles, const ItemDev* items, const MatDev* mats,
                    const uint32_t* s_hat, unsigned long long* acc, unsigned* counter,
                    cudaStream_t s) {
  if (nwork == 0) return GRID_OK;
  if (p->d % 4) return GRID_ERR_UNSUPPORTED_DEGREE;
  uint32_t c[3];
  for (int i = 1; i <= 3; ++i)
    c[i - 1] = (uint32_t)(((unsigned __int128)1 << (32 + 8 * i)) % p->f.q);
  const uint4 scale = make_uint4(c[0], c[1], c[2], 0);
  TcConsts k;
  k.q = p->f.q;
  k.qinv = p->f.qinv;
  switch (cls) {
    case TC_D16: return launch_class<16, 128>(p, work, nwork, tiles, items, mats, s_hat, acc, counter, scale, k, s);
    case TC_D32: return launch_class<32, 128>(p, work, nwork, tiles, items, mats, s_hat, acc, counter, scale, k, s);
    case TC_U16: return launch_class<16, 64>(p, work, nwork, tiles, items, mats, s_hat, acc, counter, scale, k, s);
    case TC_U32: return launch_class<32, 64>(p, work, nwork, tiles, items, mats, s_hat, acc, counter, scale, k, s);
    case TC_U64: return launch_class<64, 64>(p, work, nwork, tiles, items, mats, s_hat, acc, counter, scale, k, s);
    default: return GRID_ERR_INVALID_PARAMETERS;
  }
}

}  // namespace grid
