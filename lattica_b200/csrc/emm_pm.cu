// Evaluation-domain products on the tensor cores over point-major operands:
//     out_e[m][n] = sum_k X_e[m][k] * Y_e[n][k] * 2^-32 (mod q)
// where X_e = X + e M K and Y_e = Y + e N ldy hold the words of evaluation
// point e row-major ([point][row][k]): the layout the forward transform's
// point-major mode writes (ntt_tc.cu) and prepared matrices keep beside their
// poly-major evaluations. The products are those of emm_tc.cu (the Ajtai
// commitment's, the Gram matrix's and garbage h's contraction), computed by
// the same byte-plane method:
//  * A (128 rows x 128 K bytes per chunk): row m holds X_e[m][k0 .. k0 + 31]
//    in natural byte order, exactly the 128-byte-swizzled box TMA writes;
//  * B (4 NP rows): row l NP + n, byte 4k + i = byte l of 2^(8i) Y_e[n][k] mod q,
//    built in shared memory by CUDA-core warps from a TMA-loaded Y box (dense
//    products) or from the A box itself (the Gram, X = Y), so that
//    sum_l 2^(8l) D_l = sum_k x_k y_k (mod q) with v = sum_l 2^(8l) D_l <
//    4 K 255 q: one Montgomery reduction of v gives the canonical word; each
//    D_l < 4 K 255^2 < 2^31 for K <= 8192 per CTA.
// Result (m, n) depends only on A row m and B rows l NP + n, so rows past the
// operands' are never cleared: whatever they hold reaches only results that
// are not stored. With X rows <= 64 an A slot holds 64 rows (8 KB) and the
// MMA's rows 64-127 read whatever follows it.
//
// One CTA per (evaluation point, K range), 10 warps:
//  * warp 8 (one lane) streams the X (and Y) boxes of each 32-word chunk with
//    TMA into a ring of NSA slots, refilling a slot once its MMAs are done;
//  * warps 0-7 build the B planes of chunk c into a ring of NSB slots (each
//    thread first loads all of its words of the chunk, then scales and
//    byte-transposes them), once the boxes landed and the slot's previous
//    MMAs are done;
//  * warp 9 (one lane) issues four MMAs (M 128, N 4 NP, K 32) per chunk into
//    tensor memory and commits them to both slots' mbarriers;
//  * after the last chunk warps 0-7 combine the planes, reduce, stage the
//    point's results in shared memory and store them contiguously, [split][e]
//    [output], for the transposing sum over K ranges that follows.
// Every wait is bounded.
#include <cuda.h>
#include <cuda_runtime.h>

#include "grid_async.cuh"
#include "grid_field.cuh"
#include "grid_internal.h"
#include "grid_tc.cuh"
#include "ntt_tc_common.cuh"

namespace grid {
namespace {

using namespace tcx;

constexpr int kPmBuildWarps = 8;
constexpr int kPmBuilders = kPmBuildWarps * 32;
constexpr int kPmLoadWarp = kPmBuildWarps;
constexpr int kPmMmaWarp = kPmBuildWarps + 1;
constexpr int kPmThreads = (kPmBuildWarps + 2) * 32;
constexpr int KCH = 32;        // K words per chunk: one 128-byte swizzled row
constexpr int kPmMaxK = 8192;  // K words per CTA: 4 * 8192 * 255^2 < 2^31

// NP: Y rows padded to 16 .. 64; MX: X rows per A slot (64 or 128).
template <int NP, int MX, bool UPPER>
struct PmShape {
  static constexpr int NMMA = 4 * NP;                         // B rows: four byte planes
  static constexpr uint32_t XSLOT = MX * 128u;                // X box
  static constexpr uint32_t YSLOT = UPPER ? 0u : NP * 128u;   // Y box (dense products)
  static constexpr uint32_t ASLOT = XSLOT + YSLOT;            // multiples of 1024 bytes
  static constexpr uint32_t BSLOT = NMMA * 128u;
  static constexpr int NSB = BSLOT >= 16384 ? 2 : 3;
  // as many A slots (2 to 8) as keep a CTA within half the SM's shared memory
  static constexpr uint32_t kBudget = 106496;
  static constexpr int NSA_FIT = (int)((kBudget - NSB * BSLOT) / ASLOT);
  static constexpr int NSA = NSA_FIT < 2 ? 2 : NSA_FIT > 8 ? 8 : NSA_FIT;
  static constexpr uint32_t OFF_B = NSA * ASLOT;  // the B ring follows the A ring
  static constexpr uint32_t OFF_BAR = OFF_B + NSB * BSLOT;
  static constexpr int NBARS = 2 * NSA + 2 * NSB + 1;
  static constexpr uint32_t SMEM = OFF_BAR + NBARS * 8 + 16 + 1024;  // + alignment slack
  static constexpr uint32_t TCOLS = NMMA <= 64 ? 64u : NMMA <= 128 ? 128u : 256u;
  // the MMA reads 128 rows from every A slot: the last one's rows past MX lie
  // in the B ring
  static_assert(MX == 128 || NSB * BSLOT >= 64u * 128, "A slot overrun");
  // the point's results are staged in the B ring
  static_assert(NSB * BSLOT >= (UPPER ? 64u * 65 / 2 : (uint32_t)MX * NP) * 4, "staging");
};

// Bounded wait by lane 0 alone (mbarrier operations of a whole warp on one
// barrier serialise over its lanes); __syncwarp then orders what lane 0
// acquired before every lane's later accesses.
__device__ __forceinline__ bool lane0_wait(uint64_t* bar, uint32_t parity, int lane, int* err) {
  bool ok = true;
  if (lane == 0) ok = mbar_wait(bar, parity, err);
  __syncwarp();
  return __shfl_sync(0xffffffffu, ok, 0);
}

// The builder warps' own barrier (named barrier 1; the CTA's is 0).
__device__ __forceinline__ void builders_sync() {
  asm volatile("bar.sync 1, %0;" ::"n"(kPmBuilders) : "memory");
}

template <int NP, int MX, bool UPPER>
__global__ void __launch_bounds__(kPmThreads, 1)
    emm_pm_kernel(const __grid_constant__ CUtensorMap tmap_x,
                  const __grid_constant__ CUtensorMap tmap_y, uint32_t* __restrict__ part, int M,
                  int N, int K, int k_per_split, uint32_t box_bytes, uint4 scale, uint4 scale_q,
                  const TcConsts k, int* __restrict__ err) {
  using S = PmShape<NP, MX, UPPER>;
  constexpr int NSA = S::NSA, NSB = S::NSB, NMMA = S::NMMA;
  extern __shared__ __align__(1024) unsigned char sm_raw[];
  const uint32_t raw = smem_addr(sm_raw);
  unsigned char* sm = sm_raw + (((raw + 1023u) & ~1023u) - raw);
  const uint32_t s0 = smem_addr(sm);
  uint64_t* full = reinterpret_cast<uint64_t*>(sm + S::OFF_BAR);  // A slot landed
  uint64_t* a_free = full + NSA;                                  // A slot's MMAs done
  uint64_t* built = a_free + NSA;                                 // B slot written
  uint64_t* b_free = built + NSB;                                 // B slot's MMAs done
  uint64_t* done = b_free + NSB;                                  // every MMA done
  uint32_t* taddr_slot = reinterpret_cast<uint32_t*>(done + 1);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int e = blockIdx.x;
  const int kbeg = blockIdx.y * k_per_split;
  const int kend = min(K, kbeg + k_per_split);
  const int nch = kend > kbeg ? (kend - kbeg + KCH - 1) / KCH : 0;

  if (warp == kPmMmaWarp) {
    tc::tmem_alloc(taddr_slot, S::TCOLS);
    tc::tmem_relinquish();
  }
  if (threadIdx.x == 0) {
    for (int i = 0; i < NSA; ++i) {
      mbar_init(&full[i], 1);
      mbar_init(&a_free[i], 1);
    }
    for (int i = 0; i < NSB; ++i) {
      mbar_init(&built[i], kPmBuildWarps);
      mbar_init(&b_free[i], 1);
    }
    mbar_init(done, 1);
    fence_mbar_init();
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tbase = *taddr_slot;

  if (warp == kPmLoadWarp) {
    // ------------------------------------------------------------ TMA loads
    if (lane == 0) {
      int issued = 0;
      for (int c = 0; c < nch; ++c) {
        const int sl = c % NSA;
        if (c >= NSA && !mbar_wait(&a_free[sl], ((c / NSA) - 1) & 1, err)) break;
        const uint32_t sa = s0 + sl * S::ASLOT;
        const uint32_t bar = smem_addr(&full[sl]);
        mbar_arrive_expect_tx(&full[sl], box_bytes);
        tma_load_3d(sa, &tmap_x, kbeg + c * KCH, 0, e, bar);
        if (!UPPER) tma_load_3d(sa + S::XSLOT, &tmap_y, kbeg + c * KCH, 0, e, bar);
        ++issued;
      }
      // no copy may still be writing shared memory when the CTA exits
      for (int sl = 0; sl < NSA; ++sl) {
        const int loads = issued > sl ? (issued - sl + NSA - 1) / NSA : 0;
        if (loads) mbar_wait_sleep(&full[sl], (loads - 1) & 1, err);
      }
    }
    __syncwarp();
  } else if (warp == kPmMmaWarp) {
    // ------------------------------------------------------------ MMA issue
    if (lane == 0) {
      const uint32_t idesc = tc::idesc_u8(128, NMMA);
      for (int c = 0; c < nch; ++c) {
        const int sl = c % NSA, bs = c % NSB;
        if (!mbar_wait(&full[sl], (c / NSA) & 1, err) ||
            !mbar_wait(&built[bs], (c / NSB) & 1, err))
          break;
        tc::fence_after_sync();
        const uint32_t sa = s0 + sl * S::ASLOT, sb = s0 + S::OFF_B + bs * S::BSLOT;
#pragma unroll
        for (int s = 0; s < 4; ++s)
          tc::mma_u8(tbase, desc_sw128(sa + 32 * s), desc_sw128(sb + 32 * s), idesc,
                     (c | s) != 0);
        tc::mma_commit(&a_free[sl]);
        tc::mma_commit(&b_free[bs]);
      }
      // completes once every MMA issued above has (at once if none was)
      tc::mma_commit(done);
      mbar_wait_sleep(done, 0, err);
    }
    __syncwarp();
  } else {
    // ------------------------------------------------------------ B planes
    const int rows = UPPER ? M : N;
    // a warp takes one row's 32 words per step: one 128-byte row, no bank
    // conflict; every thread holds at most NP / 8 words of a chunk
    constexpr int kWords = NP * KCH / kPmBuilders;
    const int n_base = threadIdx.x >> 5, kk = lane;
    bool ok = true;
    for (int c = 0; ok && c < nch; ++c) {
      const int sl = c % NSA, bs = c % NSB;
      ok = lane0_wait(&full[sl], (c / NSA) & 1, lane, err);
      if (ok && c >= NSB) ok = lane0_wait(&b_free[bs], ((c / NSB) - 1) & 1, lane, err);
      if (!ok) break;
      const unsigned char* src = sm + sl * S::ASLOT + (UPPER ? 0u : S::XSLOT);
      unsigned char* bt = sm + S::OFF_B + bs * S::BSLOT;
      uint32_t y[kWords];
#pragma unroll
      for (int i = 0; i < kWords; ++i) {
        const int n = n_base + 8 * i;
        y[i] = n < rows ? *reinterpret_cast<const uint32_t*>(src + sw128(n, 0, kk >> 2, 0) +
                                                             4 * (kk & 3))
                        : 0u;
      }
#pragma unroll
      for (int i = 0; i < kWords; ++i) {
        const int n = n_base + 8 * i;
        if (n >= rows) continue;
        // B row l NP + n, K word kk: byte l of 2^(8i) y mod q for i = 0 .. 3
        const uint32_t v = y[i];
        const uint32_t y1 = mont_c(v, scale.x, scale_q.x, k.q);  // 2^8 y
        const uint32_t y2 = mont_c(v, scale.y, scale_q.y, k.q);  // 2^16 y
        const uint32_t y3 = mont_c(v, scale.z, scale_q.z, k.q);  // 2^24 y
        const uint32_t lo = __byte_perm(v, y1, 0x5140), hi = __byte_perm(y2, y3, 0x5140);
        const uint32_t lo2 = __byte_perm(v, y1, 0x7362), hi2 = __byte_perm(y2, y3, 0x7362);
        unsigned char* dst = bt + sw128(n, 0, kk >> 2, 0) + 4 * (kk & 3);
        *reinterpret_cast<uint32_t*>(dst) = __byte_perm(lo, hi, 0x5410);
        *reinterpret_cast<uint32_t*>(dst + NP * 128) = __byte_perm(lo, hi, 0x7632);
        *reinterpret_cast<uint32_t*>(dst + 2 * NP * 128) = __byte_perm(lo2, hi2, 0x5410);
        *reinterpret_cast<uint32_t*>(dst + 3 * NP * 128) = __byte_perm(lo2, hi2, 0x7632);
      }
      tc::fence_async_smem();  // the planes are read by the tensor cores
      __syncwarp();
      if (lane == 0) mbar_arrive(&built[bs]);
    }
    // ------------------------------------------------------------ epilogue
    ok = ok && lane0_wait(done, 0, lane, err);
    tc::fence_after_sync();
    // every builder reaches the barrier below (a failed wait skips only work)
    const int outputs = UPPER ? M * (M + 1) / 2 : M * N;
    uint32_t* stage = reinterpret_cast<uint32_t*>(sm + S::OFF_B);  // B ring: MMAs are done
    if (ok) {
      // warp w reads tensor-memory lanes 32 (w % 4) .. + 31 (rows m) and
      // column groups of 8 starting at 8 (w / 4)
      const int m = 32 * (warp & 3) + lane;
      const uint32_t taddr = tc::tmem_addr(tbase, 32 * (warp & 3), 0);
#pragma unroll 1
      for (int n0 = 8 * (warp >> 2); n0 < NP; n0 += 8 * (kPmBuildWarps / 4)) {
        uint32_t eb[4][8];
#pragma unroll
        for (int l = 0; l < 4; ++l) tc::tmem_ld8(taddr + l * NP + n0, eb[l]);
        tc::tmem_ld_wait32(eb);
        if (m >= M) continue;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          const int n = n0 + j;
          if (n >= N || (UPPER && n < m)) continue;
          uint64_t v = mad_wide(eb[1][j], 256u, (uint64_t)eb[0][j]);
          v = mad_wide(eb[2][j], 65536u, v);
          v = mad_wide(eb[3][j], 16777216u, v);
          const int idx = UPPER ? m * M - (m * (m - 1)) / 2 + (n - m) : m * N + n;
          stage[idx] = nch ? redc64(v, k.q, k.qinv) : 0u;  // an empty K range sums to 0
        }
      }
    }
    builders_sync();
    if (ok) {
      uint32_t* o = part + ((size_t)blockIdx.y * gridDim.x + e) * outputs;
      for (int i = threadIdx.x; i < outputs; i += kPmBuilders) o[i] = stage[i];
    }
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == kPmMmaWarp) {
    tc::fence_after_sync();
    tc::tmem_dealloc(tbase, S::TCOLS);
  }
}

// out[idx][e] = sum over K ranges s of part[s][e][idx] (mod q): 32 x 32 tiles
// through shared memory, reads along idx, writes along e.
__global__ void sum_transpose_kernel(const uint32_t* __restrict__ part, uint32_t* __restrict__ out,
                                     int outputs, int d, int splits, uint32_t q) {
  __shared__ uint32_t t[32][33];
  const int i0 = blockIdx.x * 32, e0 = blockIdx.y * 32;
  const size_t stride = (size_t)d * outputs;
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int e = e0 + r, i = i0 + threadIdx.x;
    if (e < d && i < outputs) {
      const uint32_t* src = part + (size_t)e * outputs + i;
      uint32_t v = 0;
      for (int s0 = 0; s0 < splits; s0 += 4) {  // four independent loads in flight
        uint32_t w[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) w[j] = s0 + j < splits ? src[(size_t)(s0 + j) * stride] : 0u;
#pragma unroll
        for (int j = 0; j < 4; ++j) v = add_mod(v, w[j], q);
      }
      t[r][threadIdx.x] = v;
    }
  }
  __syncthreads();
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int i = i0 + r, e = e0 + threadIdx.x;
    if (e < d && i < outputs) out[(size_t)i * d + e] = t[threadIdx.x][r];
  }
}

// A [d][rows][K] point-major operand (row stride ld words) as a 3D tensor map
// with boxes of 32 words x box_rows rows x one point, 128-byte swizzle.
bool make_pm_map(CUtensorMap* map, const uint32_t* base, int K, int rows, int ld, int d,
                 int box_rows) {
  EncodeTiled enc = encoder();
  if (!enc) return false;
  const cuuint64_t dims[3] = {(cuuint64_t)K, (cuuint64_t)rows, (cuuint64_t)d};
  const cuuint64_t strides[2] = {(cuuint64_t)ld * 4, (cuuint64_t)rows * ld * 4};
  const cuuint32_t box[3] = {(cuuint32_t)KCH, (cuuint32_t)box_rows, 1};
  const cuuint32_t estr[3] = {1, 1, 1};
  return enc(map, CU_TENSOR_MAP_DATA_TYPE_UINT32, 3, const_cast<uint32_t*>(base), dims, strides,
             box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
             CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <int NP, int MX, bool UPPER>
int launch_pm(const grid_gpu_plan* p, const uint32_t* X, const uint32_t* Y, int M, int N, int K,
              int ldy, uint32_t* part, const EmmPmGeometry& g, cudaStream_t s) {
  using S = PmShape<NP, MX, UPPER>;
  static int bps_cache[kMaxDevices] = {};
  int bps = 0;
  const int rc = prepare_kernel(emm_pm_kernel<NP, MX, UPPER>, S::SMEM, kPmThreads, p->device,
                                bps_cache, &bps, true);
  if (rc) return rc;
  // boxes of whole 8-row groups: rows past M (N) read as zero fill
  const int bx = (M + 7) & ~7, by = (N + 7) & ~7;
  CUtensorMap mx, my;
  if (!make_pm_map(&mx, X, K, M, K, (int)p->d, bx)) return GRID_ERR_CUDA;
  if (UPPER)
    my = mx;
  else if (!make_pm_map(&my, Y, K, N, ldy, (int)p->d, by))
    return GRID_ERR_CUDA;
  const uint32_t box_bytes = 128u * (uint32_t)bx + (UPPER ? 0u : 128u * (uint32_t)by);
  // 2^(8i) R mod q (a Montgomery product with it is 2^(8i) y mod q) and the
  // Shoup companions c qinv mod 2^32
  uint32_t c[3], cq[3];
  for (int i = 1; i <= 3; ++i) {
    c[i - 1] = (uint32_t)(((unsigned __int128)1 << (32 + 8 * i)) % p->f.q);
    cq[i - 1] = c[i - 1] * p->f.qinv;
  }
  TcConsts k;
  k.q = p->f.q;
  k.qinv = p->f.qinv;
  emm_pm_kernel<NP, MX, UPPER><<<dim3(p->d, g.splits), kPmThreads, S::SMEM, s>>>(
      mx, my, part, M, N, K, g.k_per_split, box_bytes, make_uint4(c[0], c[1], c[2], 0),
      make_uint4(cq[0], cq[1], cq[2], 0), k, p->d_err);
  return cuda_status(cudaGetLastError());
}

template <int NP>
int launch_np(const grid_gpu_plan* p, const uint32_t* X, const uint32_t* Y, int M, int N, int K,
              int ldy, int mode, uint32_t* part, const EmmPmGeometry& g, cudaStream_t s) {
  if (mode == EMM_UPPER) return launch_pm<NP, 64, true>(p, X, X, M, N, K, K, part, g, s);
  return M <= 64 ? launch_pm<NP, 64, false>(p, X, Y, M, N, K, ldy, part, g, s)
                 : launch_pm<NP, 128, false>(p, X, Y, M, N, K, ldy, part, g, s);
}

}  // namespace

bool emm_pm_geometry(const grid_gpu_plan* p, int M, int N, int K, int ldy, int mode,
                     EmmPmGeometry* g) {
  if (!p->pm_emm || is_crt(p) || M <= 0 || N <= 0 || K <= 0 || M > 128 || N > 64) return false;
  if (mode == EMM_UPPER && M != N) return false;
  // row strides of whole 16-byte units (tensor-map strides)
  if (K % 4 || (mode != EMM_UPPER && ldy % 4)) return false;
  g->np = N <= 16 ? 16 : N <= 32 ? 32 : N <= 48 ? 48 : 64;
  // one CTA per evaluation point and K range: split K so that about two CTAs
  // per SM are resident, at least 2 chunks per split, at most kPmMaxK words
  const int chunks = (K + KCH - 1) / KCH;
  int want = 2 * p->num_sms / (int)p->d;
  if (want > chunks / 2) want = chunks / 2;
  if (want < 1) want = 1;
  int cps = (chunks + want - 1) / want;
  if (cps * KCH > kPmMaxK) cps = kPmMaxK / KCH;
  g->k_per_split = cps * KCH;
  g->splits = (chunks + cps - 1) / cps;
  return true;
}

size_t emm_pm_workspace_words(const grid_gpu_plan* p, int M, int N, int K, int mode) {
  EmmPmGeometry g;  // the split count does not depend on Y's row stride
  if (!emm_pm_geometry(p, M, N, K, 4, mode, &g)) return 0;
  const size_t outputs = mode == EMM_UPPER ? (size_t)M * (M + 1) / 2 : (size_t)M * N;
  return (size_t)g.splits * outputs * p->d;
}

int launch_emm_pm(const grid_gpu_plan* p, const uint32_t* X, const uint32_t* Y, int M, int N,
                  int K, int ldy, int mode, uint32_t* out_evals, uint32_t* work, cudaStream_t s) {
  EmmPmGeometry g;
  if (!emm_pm_geometry(p, M, N, K, ldy, mode, &g)) return GRID_ERR_INVALID_PARAMETERS;
  if (!work) return GRID_ERR_NULL_POINTER;
  auto unaligned = [](const void* a) { return reinterpret_cast<uintptr_t>(a) % 16 != 0; };
  if (unaligned(X) || (mode != EMM_UPPER && unaligned(Y))) return GRID_ERR_MISALIGNED;
  int rc;
  switch (g.np) {
    case 16: rc = launch_np<16>(p, X, Y, M, N, K, ldy, mode, work, g, s); break;
    case 32: rc = launch_np<32>(p, X, Y, M, N, K, ldy, mode, work, g, s); break;
    case 48: rc = launch_np<48>(p, X, Y, M, N, K, ldy, mode, work, g, s); break;
    default: rc = launch_np<64>(p, X, Y, M, N, K, ldy, mode, work, g, s); break;
  }
  if (rc) return rc;
  // point-major partials [split][e][output] -> out [output][e]
  const int outputs = mode == EMM_UPPER ? M * (M + 1) / 2 : M * N;
  const int d = (int)p->d;
  sum_transpose_kernel<<<dim3((outputs + 31) / 32, (d + 31) / 32), dim3(32, 32), 0, s>>>(
      work, out_evals, outputs, d, g.splits, p->f.q);
  return cuda_status(cudaGetLastError());
}

}  // namespace grid
