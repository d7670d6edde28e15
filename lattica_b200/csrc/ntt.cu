// Batched twisted negacyclic NTT / INTT kernels for R_q = Z_q[X]/(X^d + 1).
//
// Reference path replaced: TwistedNttPlan::{forward,inverse}_in_place_trusted
// (algebra/src/poly/ntt.rs:75-104) over the bit-reverse + DIT forward and
// GS + n^-1 + bit-reverse inverse (algebra/src/arith/ntt.rs:207-340), and the
// "NTT -> Montgomery pointwise -> INTT" chain of a negacyclic product.
//
// Design (sm_100a):
//  * The twist by psi^i, the bit-reversal and the n^-1 scale are folded into
//    a merged Cooley-Tukey / Gentleman-Sande pair with twiddles psi^brv(k).
//    The forward transform leaves evaluation x(psi^(2*brv(j)+1)) at position
//    j; the reference's natural-order slot k is position brv(k), so output
//    ordering is register renaming at the store.
//  * The forward transform runs on lazy words (any 32-bit representative,
//    grid_field.cuh), saving the canonical reduction of every sum; the
//    inverse runs on canonical words.
//  * One persistent CTA of kWarps warps per SM. Warps stream tiles of 32
//    (d <= 64) or 32/T (d = 128, 256) polys through shared memory with TMA
//    bulk copies (one piece per lane) into 16-byte-padded slots, so per-thread
//    128-bit shared loads are bank-conflict free; mbarriers track arrival and
//    each lane's bulk group tracks its store. The next tile's input is
//    prefetched into the other buffer while the current tile computes.
//  * The transforms are fully unrolled (register-resident data), which makes
//    the kernel body larger than the instruction cache, so the warps of a CTA
//    run in lock step: a CTA barrier after every stage keeps all of them
//    inside one stage's code.
//  * d <= 64: one thread per polynomial, every twiddle index a compile-time
//    constant taken from the kernel parameter block. d = 128 / 256: T = 2 / 4
//    threads per polynomial, 64 coefficients each; log2(T) stages cross
//    threads through warp shuffles; twiddles staged in shared memory.
#include <cuda_runtime.h>

#include "grid_async.cuh"
#include "grid_field.cuh"
#include "grid_internal.h"

namespace grid {
namespace {

constexpr int kWarps = 12;  // warps per (persistent) CTA
constexpr int kThreads = kWarps * 32;

__host__ __device__ constexpr int ilog2(int x) { return x <= 1 ? 0 : 1 + ilog2(x >> 1); }

__host__ __device__ constexpr int brv(int x, int bits) {
  int r = 0;
  for (int i = 0; i < bits; ++i) r |= ((x >> i) & 1) << (bits - 1 - i);
  return r;
}

struct Consts {
  uint32_t q, qinv, r1;
};

__device__ __forceinline__ Consts consts_of(const FieldParams& f) {
  return Consts{f.q, f.qinv, f.r1};
}

// CT butterfly on lazy words: (u, v) -> (u + w v, u - w v).
__device__ __forceinline__ void ct_bfly(uint32_t& u, uint32_t& v, uint32_t w, uint32_t wq,
                                        const Consts& c) {
  const uint32_t t = mont_c(v, w, wq, c.q);
  v = sub_lazy(u, t, c.q);
  u = add_lazy(u, t, c.r1);
}

// GS butterfly on canonical words: (u, v) -> (u + v, (u - v) w).
__device__ __forceinline__ void gs_bfly(uint32_t& u, uint32_t& v, uint32_t w, uint32_t wq,
                                        const Consts& c) {
  const uint32_t s = add_canon(u, v, c.q);
  const uint32_t d = sub_lazy(u, v, c.q);
  u = s;
  v = mont_c(d, w, wq, c.q);
}

// ---------------------------------------------------------------------------
// Thread-per-polynomial transforms (d <= 64).
// ---------------------------------------------------------------------------
template <int D, int LEN>
__device__ __forceinline__ void fwd1_stages(uint32_t (&x)[D], const Tw1<D>& tw, const Consts& c) {
#pragma unroll
  for (int g = 0; g < D / (2 * LEN); ++g) {
    const int k = D / (2 * LEN) + g;
#pragma unroll
    for (int j = g * 2 * LEN; j < g * 2 * LEN + LEN; ++j)
      ct_bfly(x[j], x[j + LEN], tw.fw[k][0], tw.fw[k][1], c);
  }
  __syncthreads();
  if constexpr (LEN > 1) fwd1_stages<D, LEN / 2>(x, tw, c);
}

template <int D, int LEN>
__device__ __forceinline__ void inv1_stages(uint32_t (&x)[D], const Tw1<D>& tw, const Consts& c) {
  if constexpr (LEN == D / 2) {
    // Last GS stage (single group, k = 1) with d^-1 folded in.
#pragma unroll
    for (int j = 0; j < LEN; ++j) {
      const uint32_t s = add_canon(x[j], x[j + LEN], c.q);
      const uint32_t d = sub_lazy(x[j], x[j + LEN], c.q);
      x[j] = mont_c(s, tw.ninv[0], tw.ninv[1], c.q);
      x[j + LEN] = mont_c(d, tw.iw1n[0], tw.iw1n[1], c.q);
    }
  } else {
#pragma unroll
    for (int g = 0; g < D / (2 * LEN); ++g) {
      const int k = D / (2 * LEN) + g;
#pragma unroll
      for (int j = g * 2 * LEN; j < g * 2 * LEN + LEN; ++j)
        gs_bfly(x[j], x[j + LEN], tw.iw[k][0], tw.iw[k][1], c);
    }
    __syncthreads();
    inv1_stages<D, LEN * 2>(x, tw, c);
  }
}

// Per-warp TMA pipeline state shared by both kernel families.
struct WarpPipe {
  uint64_t* bars;  // [buf * 2 + {0: a, 1: b}]
  uint32_t parity = 0, pending = 0;

  __device__ void init(uint64_t* b, int lane) {
    bars = b;
    if (lane == 0) {
#pragma unroll
      for (int i = 0; i < 4; ++i) mbar_init(&bars[i], 1);
      fence_mbar_init();
    }
    __syncwarp();
  }
  // Arm barrier `bar` for `bytes`; false (and nothing armed) if bytes == 0.
  __device__ bool arm(int bar, uint32_t bytes, int lane) {
    if (bytes == 0) return false;
    if (lane == 0) mbar_arrive_expect_tx(&bars[bar], bytes);
    __syncwarp();
    pending |= 1u << bar;
    return true;
  }
  __device__ bool wait(int bar, int* err) {
    if (!(pending & (1u << bar))) return true;
    const bool ok = mbar_wait(&bars[bar], (parity >> bar) & 1u, err);
    parity ^= 1u << bar;
    pending &= ~(1u << bar);
    return ok;
  }
  __device__ void drain(int* err) {
    for (int bar = 0; bar < 4; ++bar)
      if (pending & (1u << bar)) mbar_wait(&bars[bar], (parity >> bar) & 1u, err);
    pending = 0;
  }
};

__device__ __forceinline__ uint32_t polys_left(unsigned long long p0, unsigned long long n,
                                               uint32_t cap) {
  if (p0 >= n) return 0;
  const unsigned long long left = n - p0;
  return left < cap ? (uint32_t)left : cap;
}

template <int D, int MODE>
__global__ void __launch_bounds__(kThreads, 1) ntt1_kernel(const uint32_t* __restrict__ a,
                                                           const uint32_t* __restrict__ b,
                                                           uint32_t* out, unsigned long long npolys,
                                                           const __grid_constant__ Tw1<D> tw,
                                                           int* __restrict__ err) {
  constexpr int LOGD = ilog2(D);
  constexpr int PS = D + 4;          // padded slot stride (words)
  constexpr uint32_t PIECE = D * 4;  // bytes each lane moves per tile
  constexpr int BUF = 32 * PS;       // words per tile buffer
  constexpr unsigned long long BT = 32ull * kWarps;  // polys per CTA tile
  extern __shared__ __align__(128) uint32_t smem[];
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  uint32_t* wbase = smem + warp * 2 * BUF;
  WarpPipe pipe;
  pipe.init(reinterpret_cast<uint64_t*>(smem + kWarps * 2 * BUF) + warp * 4, lane);
  const Consts c = consts_of(tw.f);

  const unsigned long long nbt = (npolys + BT - 1) / BT;
  auto issue = [&](uint32_t* buf, const uint32_t* src, unsigned long long bt, int bar) {
    const unsigned long long p0 = bt * BT + warp * 32ull;
    const uint32_t np = polys_left(p0, npolys, 32);
    if (pipe.arm(bar, np * PIECE, lane) && (uint32_t)lane < np)
      bulk_load(buf + lane * PS, src + (p0 + lane) * D, PIECE, &pipe.bars[bar]);
  };

  bool ok = true;
  int buf = 0;
  unsigned long long bt = blockIdx.x;
  if (bt < nbt) issue(wbase, a, bt, 0);
  for (; bt < nbt; bt += gridDim.x, buf ^= 1) {  // trip count is uniform over the CTA
    uint32_t* slot = wbase + buf * BUF + lane * PS;
    const unsigned long long p0 = bt * BT + warp * 32ull;
    const uint32_t np = polys_left(p0, npolys, 32);

    ok = __syncthreads_and(pipe.wait(buf * 2, err));
    if (!ok) break;
    uint32_t x[D];
    const uint4* sv = reinterpret_cast<const uint4*>(slot);
#pragma unroll
    for (int cc = 0; cc < D / 4; ++cc) {
      const uint4 v = sv[cc];
      if constexpr (MODE == MODE_INV) {
        x[brv(4 * cc + 0, LOGD)] = v.x;
        x[brv(4 * cc + 1, LOGD)] = v.y;
        x[brv(4 * cc + 2, LOGD)] = v.z;
        x[brv(4 * cc + 3, LOGD)] = v.w;
      } else {
        x[4 * cc + 0] = v.x;
        x[4 * cc + 1] = v.y;
        x[4 * cc + 2] = v.z;
        x[4 * cc + 3] = v.w;
      }
    }
    fence_proxy_async_smem();
    __syncwarp();
    if (bt + gridDim.x < nbt) {
      bulk_wait_read_all();  // this lane's previous store out of the other buffer is done
      __syncwarp();
      issue(wbase + (buf ^ 1) * BUF, a, bt + gridDim.x, (buf ^ 1) * 2);
    }
    if constexpr (MODE == MODE_MULINV) issue(wbase + buf * BUF, b, bt, buf * 2 + 1);

    if constexpr (MODE != MODE_INV) fwd1_stages<D, D / 2>(x, tw, c);
    if constexpr (MODE == MODE_MULINV) {
      ok = __syncthreads_and(pipe.wait(buf * 2 + 1, err));
      if (!ok) break;
#pragma unroll
      for (int cc = 0; cc < D / 4; ++cc) {
        const uint4 v = sv[cc];
        x[brv(4 * cc + 0, LOGD)] = mont_v(x[brv(4 * cc + 0, LOGD)], v.x, c.q, c.qinv);
        x[brv(4 * cc + 1, LOGD)] = mont_v(x[brv(4 * cc + 1, LOGD)], v.y, c.q, c.qinv);
        x[brv(4 * cc + 2, LOGD)] = mont_v(x[brv(4 * cc + 2, LOGD)], v.z, c.q, c.qinv);
        x[brv(4 * cc + 3, LOGD)] = mont_v(x[brv(4 * cc + 3, LOGD)], v.w, c.q, c.qinv);
      }
      __syncthreads();
    }
    if constexpr (MODE != MODE_FWD) inv1_stages<D, 1>(x, tw, c);

    uint4* so = reinterpret_cast<uint4*>(slot);
#pragma unroll
    for (int cc = 0; cc < D / 4; ++cc) {
      if constexpr (MODE == MODE_FWD) {
        // lazy words -> canonical (x * 2^32 * 2^-32)
        so[cc] = make_uint4(mont_v(x[brv(4 * cc + 0, LOGD)], c.r1, c.q, c.qinv),
                            mont_v(x[brv(4 * cc + 1, LOGD)], c.r1, c.q, c.qinv),
                            mont_v(x[brv(4 * cc + 2, LOGD)], c.r1, c.q, c.qinv),
                            mont_v(x[brv(4 * cc + 3, LOGD)], c.r1, c.q, c.qinv));
      } else {
        so[cc] = make_uint4(x[4 * cc + 0], x[4 * cc + 1], x[4 * cc + 2], x[4 * cc + 3]);
      }
    }
    fence_proxy_async_smem();
    if ((uint32_t)lane < np) {
      bulk_store(out + (p0 + lane) * D, slot, PIECE);
      bulk_commit();
    }
  }
  if (!ok) pipe.drain(err);  // let copies already in flight land
  bulk_wait_all();
}

// ---------------------------------------------------------------------------
// T threads per polynomial (d = 128, 256). Thread t of a polynomial holds the
// 4-word chunks c = T*m + t (m = 0 .. D/(4T)-1): local element e = 4m + s is
// position i = 4T*m + 4t + s.
// ---------------------------------------------------------------------------
template <int D, int T, int LEN>
__device__ __forceinline__ void fwdT_stages(uint32_t (&x)[D / T], const uint2* __restrict__ tws,
                                            int t, const Consts& c) {
  constexpr int E = D / T;
  constexpr int LOG2LEN = ilog2(2 * LEN);
  if constexpr (LEN >= 4 * T) {
    constexpr int STEP = LEN / T;
#pragma unroll
    for (int e = 0; e < E; ++e) {
      if ((e & STEP) == 0) {
        const int k = D / (2 * LEN) + ((4 * T * (e >> 2)) >> LOG2LEN);
        const uint2 w = tws[k];
        ct_bfly(x[e], x[e + STEP], w.x, w.y, c);
      }
    }
  } else if constexpr (LEN >= 4) {
    constexpr int M = LEN / 4;
    const bool upper = (t & M) != 0;
#pragma unroll
    for (int e = 0; e < E; ++e) {
      const int k = D / (2 * LEN) + ((4 * T * (e >> 2) + 4 * t) >> LOG2LEN);
      const uint2 w = tws[k];
      const uint32_t prod = mont_c(x[e], w.x, w.y, c.q);
      const uint32_t mine = upper ? prod : x[e];
      const uint32_t other = __shfl_xor_sync(0xffffffffu, mine, M);
      x[e] = upper ? sub_lazy(other, mine, c.q) : add_lazy(mine, other, c.r1);
    }
  } else {
#pragma unroll
    for (int e = 0; e < E; ++e) {
      if ((e & LEN) == 0) {
        const int k = D / (2 * LEN) + ((4 * T * (e >> 2) + 4 * t + (e & 3)) >> LOG2LEN);
        const uint2 w = tws[k];
        ct_bfly(x[e], x[e + LEN], w.x, w.y, c);
      }
    }
  }
  __syncthreads();
  if constexpr (LEN > 1) fwdT_stages<D, T, LEN / 2>(x, tws, t, c);
}

template <int D, int T, int LEN>
__device__ __forceinline__ void invT_stages(uint32_t (&x)[D / T], const uint2* __restrict__ tws,
                                            int t, const Consts& c) {
  constexpr int E = D / T;
  constexpr int LOG2LEN = ilog2(2 * LEN);
  const uint2* iw = tws + D;
  if constexpr (LEN == D / 2) {
    static_assert(LEN >= 4 * T, "last stage must be thread-local");
    constexpr int STEP = LEN / T;
    const uint2 n0 = tws[2 * D], n1 = tws[2 * D + 1];
#pragma unroll
    for (int e = 0; e < E; ++e) {
      if ((e & STEP) == 0) {
        const uint32_t s = add_canon(x[e], x[e + STEP], c.q);
        const uint32_t d = sub_lazy(x[e], x[e + STEP], c.q);
        x[e] = mont_c(s, n0.x, n0.y, c.q);
        x[e + STEP] = mont_c(d, n1.x, n1.y, c.q);
      }
    }
  } else {
    if constexpr (LEN >= 4 * T) {
      constexpr int STEP = LEN / T;
#pragma unroll
      for (int e = 0; e < E; ++e) {
        if ((e & STEP) == 0) {
          const int k = D / (2 * LEN) + ((4 * T * (e >> 2)) >> LOG2LEN);
          const uint2 w = iw[k];
          gs_bfly(x[e], x[e + STEP], w.x, w.y, c);
        }
      }
    } else if constexpr (LEN >= 4) {
      constexpr int M = LEN / 4;
      const bool upper = (t & M) != 0;
#pragma unroll
      for (int e = 0; e < E; ++e) {
        const int k = D / (2 * LEN) + ((4 * T * (e >> 2) + 4 * t) >> LOG2LEN);
        const uint2 w = iw[k];
        const uint32_t other = __shfl_xor_sync(0xffffffffu, x[e], M);
        // lower keeps u + v; upper gets (u - v) * w with u = other, v = x[e]
        const uint32_t s =
            upper ? sub_lazy(other, x[e], c.q) : add_canon(x[e], other, c.q);
        const uint32_t prod = mont_c(s, w.x, w.y, c.q);
        x[e] = upper ? prod : s;
      }
    } else {
#pragma unroll
      for (int e = 0; e < E; ++e) {
        if ((e & LEN) == 0) {
          const int k = D / (2 * LEN) + ((4 * T * (e >> 2) + 4 * t + (e & 3)) >> LOG2LEN);
          const uint2 w = iw[k];
          gs_bfly(x[e], x[e + LEN], w.x, w.y, c);
        }
      }
    }
    __syncthreads();
    invT_stages<D, T, LEN * 2>(x, tws, t, c);
  }
}

template <int D, int T, int MODE>
__global__ void __launch_bounds__(kThreads, 1) nttT_kernel(const uint32_t* __restrict__ a,
                                                           const uint32_t* __restrict__ b,
                                                           uint32_t* out, unsigned long long npolys,
                                                           const uint2* __restrict__ gtw,
                                                           FieldParams f, int* __restrict__ err) {
  constexpr int LOGD = ilog2(D);
  constexpr int E = D / T;            // words per thread
  constexpr int PW = 32 / T;          // polys per warp tile
  constexpr int PS = D + 4 * T;       // padded slot stride (words)
  constexpr uint32_t PIECE = E * 4;   // bytes each lane moves
  constexpr int BUF = PW * PS;
  constexpr int TWN = 2 * D + 2;      // uint2 twiddle entries
  constexpr unsigned long long BT = (unsigned long long)PW * kWarps;
  extern __shared__ __align__(128) uint32_t smem[];
  uint2* tws = reinterpret_cast<uint2*>(smem);
  uint32_t* tiles = smem + 2 * TWN + 4;  // keeps 16-byte alignment
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int pl = lane / T;  // poly within the warp tile
  const int t = lane % T;
  for (int i = threadIdx.x; i < TWN; i += blockDim.x) tws[i] = gtw[i];
  uint32_t* wbase = tiles + warp * 2 * BUF;
  WarpPipe pipe;
  pipe.init(reinterpret_cast<uint64_t*>(tiles + kWarps * 2 * BUF) + warp * 4, lane);
  __syncthreads();
  const Consts c = consts_of(f);
  const int bt_t = brv(4 * t, LOGD);  // bit-reversed contribution of t

  const unsigned long long nbt = (npolys + BT - 1) / BT;
  auto issue = [&](uint32_t* buf, const uint32_t* src, unsigned long long bt, int bar) {
    const unsigned long long p0 = bt * BT + (unsigned long long)warp * PW;
    const uint32_t np = polys_left(p0, npolys, PW);
    if (pipe.arm(bar, np * D * 4, lane) && (uint32_t)pl < np)
      bulk_load(buf + pl * PS + t * E, src + (p0 + pl) * D + t * E, PIECE, &pipe.bars[bar]);
  };

  bool ok = true;
  int buf = 0;
  unsigned long long bt = blockIdx.x;
  if (bt < nbt) issue(wbase, a, bt, 0);
  for (; bt < nbt; bt += gridDim.x, buf ^= 1) {
    uint32_t* slot = wbase + buf * BUF + pl * PS;
    const unsigned long long p0 = bt * BT + (unsigned long long)warp * PW;
    const uint32_t np = polys_left(p0, npolys, PW);

    ok = __syncthreads_and(pipe.wait(buf * 2, err));
    if (!ok) break;
    uint32_t x[E];
    if constexpr (MODE == MODE_INV) {
#pragma unroll
      for (int e = 0; e < E; ++e) {
        const int i = 4 * T * (e >> 2) + (e & 3);
        x[e] = slot[brv(i, LOGD) | bt_t];
      }
    } else {
#pragma unroll
      for (int m = 0; m < E / 4; ++m) {
        const uint4 v = reinterpret_cast<const uint4*>(slot)[T * m + t];
        x[4 * m + 0] = v.x;
        x[4 * m + 1] = v.y;
        x[4 * m + 2] = v.z;
        x[4 * m + 3] = v.w;
      }
    }
    fence_proxy_async_smem();
    __syncwarp();
    if (bt + gridDim.x < nbt) {
      bulk_wait_read_all();
      __syncwarp();
      issue(wbase + (buf ^ 1) * BUF, a, bt + gridDim.x, (buf ^ 1) * 2);
    }
    if constexpr (MODE == MODE_MULINV) issue(wbase + buf * BUF, b, bt, buf * 2 + 1);

    if constexpr (MODE != MODE_INV) fwdT_stages<D, T, D / 2>(x, tws, t, c);
    if constexpr (MODE == MODE_MULINV) {
      ok = __syncthreads_and(pipe.wait(buf * 2 + 1, err));
      if (!ok) break;
#pragma unroll
      for (int e = 0; e < E; ++e) {
        const int i = 4 * T * (e >> 2) + (e & 3);
        x[e] = mont_v(x[e], slot[brv(i, LOGD) | bt_t], c.q, c.qinv);
      }
      __syncthreads();
    }
    if constexpr (MODE != MODE_FWD) invT_stages<D, T, 1>(x, tws, t, c);

    __syncwarp();  // every lane of the warp done reading its slots
    if constexpr (MODE == MODE_FWD) {
#pragma unroll
      for (int e = 0; e < E; ++e) {
        const int i = 4 * T * (e >> 2) + (e & 3);
        slot[brv(i, LOGD) | bt_t] = mont_v(x[e], c.r1, c.q, c.qinv);
      }
    } else {
#pragma unroll
      for (int m = 0; m < E / 4; ++m)
        reinterpret_cast<uint4*>(slot)[T * m + t] =
            make_uint4(x[4 * m + 0], x[4 * m + 1], x[4 * m + 2], x[4 * m + 3]);
    }
    fence_proxy_async_smem();
    __syncwarp();  // pieces span other lanes' chunks
    if ((uint32_t)pl < np) {
      bulk_store(out + (p0 + pl) * D + t * E, slot + t * E, PIECE);
      bulk_commit();
    }
  }
  if (!ok) pipe.drain(err);
  bulk_wait_all();
}

// ---------------------------------------------------------------------------
// Small commitments in one launch: t_b = A s_b for witness vectors of at most
// kSmallMaxCols polynomials and matrices of at most kSmallMaxRows rows (the
// plain Ajtai commitment: 8 x 64, 64 witnesses). Three separate launches
// (transform, contraction, inverse) are latency-bound at that size. CTA b
// takes witness b:
//  * its polynomials go to shared memory (coalesced); eight threads transform
//    each and write the canonical evaluations back in slot order;
//  * thread (e, slot) accumulates evaluation point e of output rows slot,
//    slot + 8, ... over the columns (96-bit carry chains), reading the
//    prepared matrix's evaluations coalesced from L2;
//  * eight threads per output row run the inverse transform and store it.
// The transforms are the shuffle stages of the d = 128 / 256 engine
// (fwdT_stages / invT_stages, bit-identical to the other engines); the
// accumulation is the one of emm_kernel.
// ---------------------------------------------------------------------------
constexpr int kSmallMaxCols = 128;
constexpr int kSmallMaxRows = 32;
constexpr int kSmallSlots = 8;  // output-row slots: CTA = D evaluation points x 8 slots

// Transforms use T = 8 threads per polynomial (the shuffle stages of the
// d = 128 / 256 engine), so 64 polynomials occupy all 16 warps; element
// placement as in nttT_kernel: thread t of a polynomial holds 4-word chunks
// T m + t, evaluations go to slot brv(i) | brv(4 t).
constexpr int kSmallT = 8;

template <int D, int RPT>
__global__ void __launch_bounds__(D * kSmallSlots) commit_small_kernel(
    const uint32_t* __restrict__ A, int rows, int cols, int ld, const uint32_t* __restrict__ s,
    uint32_t* __restrict__ t_out, const uint2* __restrict__ gtw, FieldParams f) {
  constexpr int LOGD = ilog2(D);
  constexpr int T = kSmallT;
  constexpr int E = D / T;            // words per thread in a transform
  constexpr int PS = D + 4 * T;       // padded row stride (words)
  constexpr int NT = D * kSmallSlots;
  constexpr int PPP = NT / T;         // polynomials per transform pass
  constexpr int TWN = 2 * D + 2;      // twiddle entries (uint2)
  extern __shared__ __align__(16) uint32_t small_smem[];
  uint2* tws = reinterpret_cast<uint2*>(small_smem);
  uint32_t* sh = small_smem + 2 * TWN + 4;  // [cols][PS]: witness, then its evaluations
  uint32_t* oh = sh + cols * PS;            // [rows][PS]: output evaluations
  const int tid = threadIdx.x;
  const int pl = tid / T, t = tid % T;
  const int bt_t = brv(4 * t, LOGD);
  const Consts c = consts_of(f);
  const size_t b = blockIdx.x;

  for (int i = tid; i < TWN; i += NT) tws[i] = gtw[i];
  const uint4* src = reinterpret_cast<const uint4*>(s + b * (size_t)cols * D);
  for (int i = tid; i < cols * (D / 4); i += NT)
    *reinterpret_cast<uint4*>(sh + (i / (D / 4)) * PS + 4 * (i % (D / 4))) = src[i];
  __syncthreads();

  // forward transforms, PPP polynomials per pass; groups past the last
  // polynomial transform row 0 and discard it (the stages hold CTA barriers
  // and shuffles, so every thread runs them)
  for (int k0 = 0; k0 < cols; k0 += PPP) {
    const int k = k0 + pl;
    uint32_t* row = sh + (k < cols ? k : 0) * PS;
    uint32_t x[E];
#pragma unroll
    for (int m = 0; m < E / 4; ++m) {
      const uint4 v = reinterpret_cast<const uint4*>(row)[T * m + t];
      x[4 * m + 0] = v.x;
      x[4 * m + 1] = v.y;
      x[4 * m + 2] = v.z;
      x[4 * m + 3] = v.w;
    }
    fwdT_stages<D, T, D / 2>(x, tws, t, c);  // ends with a CTA barrier: every row read
    if (k < cols) {
#pragma unroll
      for (int e = 0; e < E; ++e) {  // lazy words -> canonical, slot order
        const int i = 4 * T * (e >> 2) + (e & 3);
        row[brv(i, LOGD) | bt_t] = mont_v(x[e], c.r1, c.q, c.qinv);
      }
    }
    __syncthreads();
  }

  // out_hat[r][e] = sum_k A[r][k][e] s_hat[k][e] * 2^-32: thread (e, slot)
  // owns rows slot, slot + 8, ... (RPT of them), all columns; 16 matrix loads
  // in flight per thread
  {
    const int e = tid % D, slot = tid / D;
    Acc96 acc[RPT];
#pragma unroll
    for (int i = 0; i < RPT; ++i) acc96_zero(acc[i]);
    // 16 columns at a time: every matrix load of the group is issued before
    // the first multiply-add uses one
    constexpr int KB = 16;
    for (int k0 = 0; k0 < cols; k0 += KB) {
      uint32_t av[RPT][KB], sv[KB];
#pragma unroll
      for (int j = 0; j < KB; ++j) {
        const int k = k0 + j;
        sv[j] = k < cols ? sh[k * PS + e] : 0u;
#pragma unroll
        for (int i = 0; i < RPT; ++i) {
          const int r = slot + kSmallSlots * i;
          av[i][j] = (k < cols && r < rows) ? __ldg(A + ((size_t)r * ld + k) * D + e) : 0u;
        }
      }
#pragma unroll
      for (int j = 0; j < KB; ++j)
#pragma unroll
        for (int i = 0; i < RPT; ++i) acc96_mad(acc[i], av[i][j], sv[j]);
    }
#pragma unroll
    for (int i = 0; i < RPT; ++i) {
      const int r = slot + kSmallSlots * i;
      if (r < rows) oh[r * PS + e] = acc96_reduce(acc[i], f);
    }
  }
  __syncthreads();

  // inverse transforms of the output rows (rows <= PPP: one pass)
  {
    const int r = pl < rows ? pl : 0;
    uint32_t x[E];
#pragma unroll
    for (int e = 0; e < E; ++e) {
      const int i = 4 * T * (e >> 2) + (e & 3);
      x[e] = oh[r * PS + (brv(i, LOGD) | bt_t)];
    }
    invT_stages<D, T, 1>(x, tws, t, c);
    if (pl < rows) {
      uint4* dst = reinterpret_cast<uint4*>(t_out + (b * rows + pl) * D);
#pragma unroll
      for (int m = 0; m < E / 4; ++m)
        dst[T * m + t] = make_uint4(x[4 * m + 0], x[4 * m + 1], x[4 * m + 2], x[4 * m + 3]);
    }
  }
}

// ---------------------------------------------------------------------------
// Host launchers
// ---------------------------------------------------------------------------
template <int D>
Tw1<D> make_tw1(const grid_gpu_plan* p) {
  Tw1<D> tw{};
  tw.f = p->f;
  for (int k = 0; k < D; ++k) {
    tw.fw[k][0] = p->tw.zeta[k];
    tw.fw[k][1] = p->tw.zeta_q[k];
    tw.iw[k][0] = p->tw.izeta[k];
    tw.iw[k][1] = p->tw.izeta_q[k];
  }
  tw.ninv[0] = p->tw.ninv;
  tw.ninv[1] = p->tw.ninv_q;
  tw.iw1n[0] = p->tw.izeta1_ninv;
  tw.iw1n[1] = p->tw.izeta1_ninv_q;
  return tw;
}

int grid_size(const grid_gpu_plan* p, unsigned long long block_tiles, int blocks_per_sm) {
  const unsigned long long cap = (unsigned long long)p->num_sms * blocks_per_sm;
  const unsigned long long g = block_tiles < cap ? block_tiles : cap;
  return g < 1 ? 1 : (int)g;
}

template <int D, int MODE>
int run1(const grid_gpu_plan* p, const uint32_t* a, const uint32_t* b, uint32_t* out,
         size_t npolys, cudaStream_t s) {
  constexpr int PS = D + 4;
  constexpr size_t smem = (size_t)kWarps * 2 * 32 * PS * 4 + kWarps * 4 * 8;
  static int bps_cache[kMaxDevices] = {};
  int bps = 0;
  const int st = prepare_kernel(ntt1_kernel<D, MODE>, smem, kThreads, p->device, bps_cache, &bps);
  if (st) return st;
  const unsigned long long tiles = (npolys + 32ull * kWarps - 1) / (32ull * kWarps);
  const Tw1<D> tw = make_tw1<D>(p);
  ntt1_kernel<D, MODE><<<grid_size(p, tiles, bps), kThreads, smem, s>>>(
      a, b, out, (unsigned long long)npolys, tw, p->d_err);
  return cuda_status(cudaGetLastError());
}

template <int D, int T, int MODE>
int runT(const grid_gpu_plan* p, const uint32_t* a, const uint32_t* b, uint32_t* out,
         size_t npolys, cudaStream_t s) {
  constexpr int PW = 32 / T;
  constexpr int PS = D + 4 * T;
  constexpr size_t smem = (size_t)(2 * (2 * D + 2) + 4) * 4 +
                          (size_t)kWarps * 2 * PW * PS * 4 + kWarps * 4 * 8;
  static int bps_cache[kMaxDevices] = {};
  int bps = 0;
  const int st =
      prepare_kernel(nttT_kernel<D, T, MODE>, smem, kThreads, p->device, bps_cache, &bps);
  if (st) return st;
  const unsigned long long tiles =
      (npolys + (unsigned long long)PW * kWarps - 1) / ((unsigned long long)PW * kWarps);
  nttT_kernel<D, T, MODE><<<grid_size(p, tiles, bps), kThreads, smem, s>>>(
      a, b, out, (unsigned long long)npolys, p->d_tw, p->f, p->d_err);
  return cuda_status(cudaGetLastError());
}

template <int MODE>
int dispatch(const grid_gpu_plan* p, const uint32_t* a, const uint32_t* b, uint32_t* out,
             size_t n, cudaStream_t s) {
  switch (p->d) {
    case 8: return run1<8, MODE>(p, a, b, out, n, s);
    case 16: return run1<16, MODE>(p, a, b, out, n, s);
    case 32: return run1<32, MODE>(p, a, b, out, n, s);
    case 64: return run1<64, MODE>(p, a, b, out, n, s);
    case 128: return runT<128, 2, MODE>(p, a, b, out, n, s);
    case 256: return runT<256, 4, MODE>(p, a, b, out, n, s);
    default: return GRID_ERR_UNSUPPORTED_DEGREE;
  }
}

}  // namespace

int ntt_max_degree() { return (int)kMaxDegree; }

int launch_ntt(const grid_gpu_plan* p, int mode, const uint32_t* a, const uint32_t* b,
               uint32_t* out, size_t npolys, cudaStream_t s) {
  if (is_crt(p)) return p->ntt_status;  // q has no 2d-th root: no transform exists
  if (npolys == 0) return GRID_OK;
  if (ntt_tc_available(p)) return launch_ntt_tc(p, mode, a, b, out, npolys, s);
  if (mode == MODE_MULINV && ntt256_tc_available(p))
    return launch_ntt256_tc(p, a, b, out, npolys, s);
  switch (mode) {
    case MODE_FWD: return dispatch<MODE_FWD>(p, a, nullptr, out, npolys, s);
    case MODE_INV: return dispatch<MODE_INV>(p, a, nullptr, out, npolys, s);
    case MODE_MULINV: return dispatch<MODE_MULINV>(p, a, b, out, npolys, s);
    default: return GRID_ERR_INVALID_PARAMETERS;
  }
}

bool commit_small_fits(const grid_gpu_plan* p, size_t rows, size_t cols, size_t batch) {
  // one CTA per witness re-reads the matrix from L2: keep to small batches
  return !is_crt(p) && p->d == 64 && rows >= 1 && rows <= (size_t)kSmallMaxRows && cols >= 1 &&
         cols <= (size_t)kSmallMaxCols && batch >= 1 && batch <= 1024;
}

int launch_commit_small(const grid_gpu_plan* p, const uint32_t* A_evals, size_t rows,
                        size_t cols, size_t ld, const uint32_t* s, size_t batch, uint32_t* t,
                        cudaStream_t st) {
  constexpr int D = 64;
  constexpr int PS = D + 4 * kSmallT, TWN = 2 * D + 2;
  static_assert(kSmallMaxRows <= D * kSmallSlots / kSmallT, "one inverse pass");
  static_assert(kSmallMaxRows == 4 * kSmallSlots, "rows per thread: 1, 2 or 4");
  if (!commit_small_fits(p, rows, cols, batch)) return GRID_ERR_INVALID_PARAMETERS;
  const size_t head = (2 * TWN + 4) * sizeof(uint32_t);  // twiddles
  const size_t smem = head + (cols + rows) * PS * sizeof(uint32_t);
  // the shared-memory limit is set once per device: set it for the largest shape
  constexpr size_t kSmemMax =
      (2 * TWN + 4) * sizeof(uint32_t) + (size_t)(kSmallMaxCols + kSmallMaxRows) * PS * 4;
  // rows per thread: 1, 2 or 4
  auto run = [&](auto kernel, int* cache) -> int {
    int bps = 0;
    const int rc = prepare_kernel(kernel, kSmemMax, D * kSmallSlots, p->device, cache, &bps);
    if (rc) return rc;
    kernel<<<(unsigned)batch, D * kSmallSlots, smem, st>>>(A_evals, (int)rows, (int)cols, (int)ld,
                                                           s, t, p->d_tw, p->f);
    return cuda_status(cudaGetLastError());
  };
  static int cache1[kMaxDevices] = {}, cache2[kMaxDevices] = {}, cache4[kMaxDevices] = {};
  if (rows <= (size_t)kSmallSlots) return run(commit_small_kernel<D, 1>, cache1);
  if (rows <= 2 * (size_t)kSmallSlots) return run(commit_small_kernel<D, 2>, cache2);
  return run(commit_small_kernel<D, 4>, cache4);
}

}  // namespace grid
