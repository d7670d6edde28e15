// Grouped contractions over point-major evaluations: many independent
// commitments t_i = A[:, :n_i] s_i of uneven length n_i (uneven batched
// commitments) per evaluation point e,
//     out_e[i][r] = sum_{k < n_i} s_i,e[k] * A_e[r][k] * 2^-32 (mod q),
// the point-major counterpart of grouped_tc.cu. The witnesses' forward
// transform stored [point][poly] (ntt_tc.cu, point-major mode over a tile
// list), so instance i's words at point e are n_i consecutive words at
// s_pm + e ps + s_off_i, and matrices keep point-major evaluations
// [point][row][ld].
//
// A work item is (tile, K range, one evaluation point); a tile holds up to 128
// instances of one matrix (the MMA's M), sorted longest first. The transform
// gives every instance its own columns from a multiple of 128, zero past its
// n_i, so that an instance row's 32-word chunk is 128 aligned bytes. Per chunk:
//  * warps 4-7 (32 instance rows each) copy the chunk of every instance row
//    still inside its length (8 lanes per row, 16-byte cp.async), zero-fill
//    the slot's rows that ran out since the slot was last filled for this
//    item, and copy the matrix rows into the slot's Y box; their lanes' copy
//    completions arrive on the slot's mbarrier (cp.async.mbarrier.arrive.noinc);
//  * warps 0-3 build the four byte planes of the matrix rows, B row l NP + r,
//    K byte 4k + i = byte l of 2^(8i) A_e[r][k] mod q (emm_tc.cu's method);
//  * one lane of warp 8 issues four MMAs (M 128, N 4 NP, K 32) into one of two
//    tensor-memory accumulators (alternating per item) and commits them to the
//    slots' barriers and, after the item's last chunk, to the accumulator's;
//  * warps 9-12 combine the planes of a finished item, reduce once and add
//    each canonical word into the 64-bit accumulator of its output poly and
//    point, so K ranges of one instance may run in different items.
// CTAs take the work list's items with a grid stride (longest first), every
// role walking the same sequence. Instance rows past a tile's count and B rows
// past the matrix's reach only results that are not stored, so they are never
// cleared. Every wait is bounded.
#include <cuda_runtime.h>

#include <algorithm>

#include "batch_tables.cuh"
#include "grid_async.cuh"
#include "grid_field.cuh"
#include "grid_internal.h"
#include "grid_tc.cuh"
#include "ntt_tc_common.cuh"

namespace grid {
namespace {

using namespace tcx;

constexpr int kGpBuildWarps = 4;
constexpr int kGpLoadWarp0 = 4, kGpLoadWarps = 4;  // 32 instance rows each
constexpr int kGpMmaWarp = 8;
constexpr int kGpEpiWarp0 = 9, kGpEpiWarps = 4;
constexpr int kGpThreads = (kGpEpiWarp0 + kGpEpiWarps) * 32;
constexpr int kGpLoaders = kGpLoadWarps * 32;
constexpr int KCH = 32;  // K words per chunk: one 128-byte swizzled row

template <int NP>
struct GpShape {
  static constexpr int NMMA = 4 * NP;            // B rows: four byte planes
  static constexpr uint32_t XSLOT = 128u * 128;  // 128 instance rows x 128 bytes
  static constexpr uint32_t YSLOT = NP * 128u;   // matrix rows
  static constexpr uint32_t ASLOT = XSLOT + YSLOT;
  static constexpr uint32_t BSLOT = NMMA * 128u;
  static constexpr int NSB = BSLOT >= 16384 ? 2 : 3;
  static constexpr uint32_t kBudget = 106496;  // two CTAs per SM
  static constexpr int NSA_FIT = (int)((kBudget - NSB * BSLOT) / ASLOT);
  static constexpr int NSA = NSA_FIT < 2 ? 2 : NSA_FIT > 6 ? 6 : NSA_FIT;
  static constexpr uint32_t OFF_B = NSA * ASLOT;
  static constexpr uint32_t OFF_BAR = OFF_B + NSB * BSLOT;
  static constexpr int NBARS = 2 * NSA + 2 * NSB + 5;
  static constexpr uint32_t SMEM = OFF_BAR + NBARS * 8 + 16 + 1024;  // + alignment slack
  static constexpr uint32_t TCOLS = 2 * NMMA;  // two accumulators
  static_assert(TCOLS == 128 || TCOLS == 256, "tensor-memory allocation");
};

__device__ __forceinline__ void cp_async16s(uint32_t dst, const void* src, uint32_t src_bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src),
               "r"(src_bytes)
               : "memory");
}

// The barrier's phase completes (for this thread's arrival) once every
// cp.async this thread issued before has landed; the arrival is one of the
// barrier's expected count.
__device__ __forceinline__ void cp_async_arrive_noinc(uint64_t* bar) {
  asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(smem_addr(bar))
               : "memory");
}

__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.wait_all;" ::: "memory");
}

// Bounded wait by lane 0; __syncwarp orders what lane 0 acquired before every
// lane's later accesses.
__device__ __forceinline__ bool lane0_wait(uint64_t* bar, uint32_t parity, int lane, int* err) {
  bool ok = true;
  if (lane == 0) ok = mbar_wait(bar, parity, err);
  __syncwarp();
  return __shfl_sync(0xffffffffu, ok, 0);
}

__device__ __forceinline__ uint32_t item_chunks(const WorkDev& w) {
  return (w.k1 - w.k0 + KCH - 1) / KCH;
}

// 64 registers: two CTAs of 13 warps put up to 8 warps on one SM sub-partition,
// whose 16384 registers hold 8 warps of 64 (not of 72).
template <int NP>
__global__ void __maxnreg__(64)
    batch_pm_kernel(const WorkDev* __restrict__ work, unsigned nwork,
                    const TileDev* __restrict__ tiles, const ItemDev* __restrict__ rows,
                    const MatDev* __restrict__ mats, const uint32_t* __restrict__ s_pm,
                    unsigned long long ps, unsigned long long* __restrict__ acc, int d,
                    uint4 scale, uint4 scale_q, const TcConsts k, int* __restrict__ err) {
  using S = GpShape<NP>;
  constexpr int NSA = S::NSA, NSB = S::NSB, NMMA = S::NMMA;
  extern __shared__ __align__(1024) unsigned char sm_raw[];
  const uint32_t raw = smem_addr(sm_raw);
  unsigned char* sm = sm_raw + (((raw + 1023u) & ~1023u) - raw);
  const uint32_t s0 = smem_addr(sm);
  uint64_t* full = reinterpret_cast<uint64_t*>(sm + S::OFF_BAR);  // slot's copies landed
  uint64_t* a_free = full + NSA;                                  // slot's MMAs done
  uint64_t* built = a_free + NSA;                                 // B slot written
  uint64_t* b_free = built + NSB;                                 // B slot's MMAs done
  uint64_t* acc_full = b_free + NSB;                              // [2] item's MMAs done
  uint64_t* acc_empty = acc_full + 2;                             // [2] item's results read
  uint64_t* drain = acc_empty + 2;                                // every MMA done (exit)
  uint32_t* taddr_slot = reinterpret_cast<uint32_t*>(drain + 1);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  if (warp == kGpMmaWarp) {
    tc::tmem_alloc(taddr_slot, S::TCOLS);
    tc::tmem_relinquish();
  }
  if (threadIdx.x == 0) {
    for (int i = 0; i < NSA; ++i) {
      mbar_init(&full[i], kGpLoaders);
      mbar_init(&a_free[i], 1);
    }
    for (int i = 0; i < NSB; ++i) {
      mbar_init(&built[i], kGpBuildWarps);
      mbar_init(&b_free[i], 1);
    }
    for (int i = 0; i < 2; ++i) {
      mbar_init(&acc_full[i], 1);
      mbar_init(&acc_empty[i], kGpEpiWarps);
    }
    mbar_init(drain, 1);
    fence_mbar_init();
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tbase = *taddr_slot;
  bool ok = true;

  if (warp >= kGpLoadWarp0 && warp < kGpLoadWarp0 + kGpLoadWarps) {
    // ------------------------------------------------------------ copies
    // Loader warp lw owns instance rows 32 lw .. + 31 of the tile. Rows are
    // sorted longest first, so the rows still inside their length at chunk k
    // form a prefix; each slot remembers from which row on it already holds
    // zeros for the current item.
    const int lw = warp - kGpLoadWarp0;
    uint32_t gc = 0;  // chunks of this CTA so far
    uint32_t zeroed[NSA];
    for (unsigned wi = blockIdx.x; ok && wi < nwork; wi += gridDim.x) {
      const WorkDev w = work[wi];
      const TileDev tl = tiles[w.tile];
      const MatDev mt = mats[tl.matrix];
      const uint32_t* se = s_pm + (unsigned long long)w.eg * ps;
      const uint32_t* ye = mt.evals_pm + (unsigned long long)w.eg * mt.rows * mt.ld;
      const uint32_t row0 = 32u * lw;
      const uint32_t cw = tl.count > row0 ? min(tl.count - row0, 32u) : 0u;  // this warp's rows
      // this lane's row: point-major column (a multiple of 128) and length
      unsigned long long off = 0;
      uint32_t len = 0;
      if ((uint32_t)lane < cw) {
        const ItemDev it = rows[tl.first + row0 + lane];
        off = it.s_off;
        len = it.n;
      }
#pragma unroll
      for (int i = 0; i < NSA; ++i) zeroed[i] = 32;  // the slots' rows hold older data
      const uint32_t nch = item_chunks(w);
      for (uint32_t c = 0; c < nch; ++c, ++gc) {
        const uint32_t sl = gc % NSA;
        if (gc >= (uint32_t)NSA && !(ok = lane0_wait(&a_free[sl], ((gc / NSA) - 1) & 1, lane, err)))
          break;
        const uint32_t kc = w.k0 + c * KCH;
        const uint32_t sa = s0 + sl * S::ASLOT;
        const uint32_t J = __popc(__ballot_sync(0xffffffffu, len > kc));  // live rows of this warp
        uint32_t zeroed_sl = 0;
#pragma unroll
        for (int i = 0; i < NSA; ++i) zeroed_sl = i == (int)sl ? zeroed[i] : zeroed_sl;
        const uint32_t zend = min(max(zeroed_sl, J), cw);
        // eight lanes per row, 16 bytes each: rows [0, J) from the witness,
        // [J, zend) as zero fill (four rows per instruction)
        const uint32_t r = lane >> 3, q4 = lane & 7;
#pragma unroll
        for (int s8 = 0; s8 < 8; ++s8) {
          const uint32_t jr = 4 * s8 + r;  // row within this warp's 32
          const unsigned long long o = __shfl_sync(0xffffffffu, off, jr);
          if (jr < zend) {
            const bool live = jr < J;
            cp_async16s(sa + sw128(row0 + jr, 0, q4, 0), live ? se + o + kc + 4 * q4 : se,
                        live ? 16u : 0u);
          }
        }
#pragma unroll
        for (int i = 0; i < NSA; ++i)
          if (i == (int)sl) zeroed[i] = min(J, cw);
        // Y: rows x eight 16-byte pieces, spread over the loader warps
        for (uint32_t u = lw * 32 + lane; u < mt.rows * 8; u += kGpLoaders) {
          const uint32_t yr = u >> 3, yq = u & 7;
          const uint32_t kw = kc + 4 * yq;
          const bool valid = kw < mt.ld;
          cp_async16s(sa + S::XSLOT + sw128(yr, 0, yq, 0),
                      valid ? ye + (unsigned long long)yr * mt.ld + kw : ye, valid ? 16u : 0u);
        }
        cp_async_arrive_noinc(&full[sl]);
      }
    }
    cp_async_wait_all();  // nothing may still be writing shared memory at exit
  } else if (warp == kGpMmaWarp) {
    // ------------------------------------------------------------ MMA issue
    if (lane == 0) {
      const uint32_t idesc = tc::idesc_u8(128, NMMA);
      uint32_t gc = 0, it = 0;
      for (unsigned wi = blockIdx.x; ok && wi < nwork; wi += gridDim.x, ++it) {
        const uint32_t buf = it & 1;
        if (it >= 2 && !(ok = mbar_wait_sleep(&acc_empty[buf], ((it >> 1) - 1) & 1, err))) break;
        tc::fence_after_sync();
        const uint32_t nch = item_chunks(work[wi]);
        for (uint32_t c = 0; c < nch; ++c, ++gc) {
          const uint32_t sl = gc % NSA, bs = gc % NSB;
          if (!(ok = mbar_wait(&full[sl], (gc / NSA) & 1, err)) ||
              !(ok = mbar_wait(&built[bs], (gc / NSB) & 1, err)))
            break;
          fence_proxy_async_smem();  // the copied rows, read by the tensor cores
          tc::fence_after_sync();
          const uint32_t sa = s0 + sl * S::ASLOT, sb = s0 + S::OFF_B + bs * S::BSLOT;
#pragma unroll
          for (int s = 0; s < 4; ++s)
            tc::mma_u8(tbase + buf * NMMA, desc_sw128(sa + 32 * s), desc_sw128(sb + 32 * s),
                       idesc, (c | (uint32_t)s) != 0);
          tc::mma_commit(&a_free[sl]);
          tc::mma_commit(&b_free[bs]);
        }
        tc::mma_commit(&acc_full[buf]);
      }
      // every MMA done before shared and tensor memory are released (at once
      // if none ran)
      tc::mma_commit(drain);
      mbar_wait_sleep(drain, 0, err);
    }
    __syncwarp();
  } else if (warp < kGpBuildWarps) {
    // ------------------------------------------------------------ B planes
    constexpr int kWords = NP * KCH / (kGpBuildWarps * 32);
    const int n_base = threadIdx.x >> 5, kk = lane;
    uint32_t gc = 0;
    for (unsigned wi = blockIdx.x; ok && wi < nwork; wi += gridDim.x) {
      const WorkDev w = work[wi];
      const uint32_t mrows = mats[tiles[w.tile].matrix].rows;
      const uint32_t nch = item_chunks(w);
      for (uint32_t c = 0; c < nch; ++c, ++gc) {
        const uint32_t sl = gc % NSA, bs = gc % NSB;
        ok = lane0_wait(&full[sl], (gc / NSA) & 1, lane, err);
        if (ok && gc >= (uint32_t)NSB) ok = lane0_wait(&b_free[bs], ((gc / NSB) - 1) & 1, lane, err);
        if (!ok) break;
        const unsigned char* src = sm + sl * S::ASLOT + S::XSLOT;
        unsigned char* bt = sm + S::OFF_B + bs * S::BSLOT;
        uint32_t y[kWords];
#pragma unroll
        for (int i = 0; i < kWords; ++i) {
          const int n = n_base + kGpBuildWarps * i;
          y[i] = n < (int)mrows ? *reinterpret_cast<const uint32_t*>(
                                      src + sw128(n, 0, kk >> 2, 0) + 4 * (kk & 3))
                                : 0u;
        }
#pragma unroll
        for (int i = 0; i < kWords; ++i) {
          const int n = n_base + kGpBuildWarps * i;
          if (n >= (int)mrows) continue;
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
        fence_proxy_async_smem();  // the planes are read by the tensor cores
        __syncwarp();
        if (lane == 0) mbar_arrive(&built[bs]);
      }
    }
  } else {
    // ------------------------------------------------------------ epilogue
    const int quarter = warp & 3;  // tensor-memory lanes 32 quarter .. + 31
    const uint32_t j = 32 * quarter + lane;
    uint32_t it = 0;
    for (unsigned wi = blockIdx.x; ok && wi < nwork; wi += gridDim.x, ++it) {
      const uint32_t buf = it & 1;
      const WorkDev w = work[wi];
      const TileDev tl = tiles[w.tile];
      const uint32_t mrows = mats[tl.matrix].rows;
      const unsigned long long toff = j < tl.count ? rows[tl.first + j].t_off : 0ull;
      // the item's whole K loop: sleep in the barrier rather than poll
      bool got = true;
      if (lane == 0) got = mbar_wait_sleep(&acc_full[buf], (it >> 1) & 1, err);
      __syncwarp();
      if (!(ok = __shfl_sync(0xffffffffu, got, 0))) break;
      tc::fence_after_sync();
      const uint32_t taddr = tc::tmem_addr(tbase, 32 * quarter, buf * NMMA);
#pragma unroll 1
      for (int n0 = 0; n0 < NP; n0 += 8) {
        uint32_t eb[4][8];
#pragma unroll
        for (int l = 0; l < 4; ++l) tc::tmem_ld8(taddr + l * NP + n0, eb[l]);
        tc::tmem_ld_wait32(eb);
        if (j >= tl.count) continue;
#pragma unroll
        for (int jj = 0; jj < 8; ++jj) {
          const uint32_t n = n0 + jj;
          if (n >= mrows) continue;
          uint64_t v = mad_wide(eb[1][jj], 256u, (uint64_t)eb[0][jj]);
          v = mad_wide(eb[2][jj], 65536u, v);
          v = mad_wide(eb[3][jj], 16777216u, v);
          atomicAdd(&acc[(toff + n) * (unsigned long long)d + w.eg],
                    (unsigned long long)redc64(v, k.q, k.qinv));
        }
      }
      tc::fence_before_sync();
      __syncwarp();
      if (lane == 0) mbar_arrive(&acc_empty[buf]);
    }
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == kGpMmaWarp) {
    tc::fence_after_sync();
    tc::tmem_dealloc(tbase, S::TCOLS);
  }
}

template <int NP>
int launch_np(const grid_gpu_plan* p, const WorkDev* work, unsigned nwork, const TileDev* tiles,
              const ItemDev* items, const MatDev* mats, const uint32_t* s_pm, uint64_t ps,
              unsigned long long* acc, cudaStream_t s) {
  using S = GpShape<NP>;
  static int bps_cache[kMaxDevices] = {};
  int bps = 0;
  const int rc = prepare_kernel(batch_pm_kernel<NP>, S::SMEM, kGpThreads, p->device, bps_cache,
                                &bps, true);
  if (rc) return rc;
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
  const unsigned grid = std::min<unsigned>(nwork, (unsigned)(p->num_sms * bps));
  batch_pm_kernel<NP><<<grid, kGpThreads, S::SMEM, s>>>(
      work, nwork, tiles, items, mats, s_pm, (unsigned long long)ps, acc, (int)p->d,
      make_uint4(c[0], c[1], c[2], 0), make_uint4(cq[0], cq[1], cq[2], 0), k, p->d_err);
  return cuda_status(cudaGetLastError());
}

}  // namespace

int launch_batch_pm(const grid_gpu_plan* p, int cls, const WorkDev* work, unsigned nwork,
                    const TileDev* tiles, const ItemDev* items, const MatDev* mats,
                    const uint32_t* s_pm, uint64_t ps, unsigned long long* acc, cudaStream_t s) {
  if (nwork == 0) return GRID_OK;
  switch (cls) {
    case TC_D16: return launch_np<16>(p, work, nwork, tiles, items, mats, s_pm, ps, acc, s);
    case TC_D32: return launch_np<32>(p, work, nwork, tiles, items, mats, s_pm, ps, acc, s);
    default: return GRID_ERR_INVALID_PARAMETERS;  // point-major tiles are dense commitments
  }
}

}  // namespace grid
