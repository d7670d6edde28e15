// Tensor-core negacyclic products for d = 256 (tcgen05, kind::i8):
// out = INTT(NTT(a) (.) b), b given in the evaluation domain (natural slots),
// the product a Montgomery product as in every other path.
//
// Reference path replaced: the "NTT -> Montgomery pointwise -> INTT" chain of a
// negacyclic product over TwistedNttPlan (algebra/src/poly/ntt.rs:75-126,
// forward slot j = x(psi^(2j+1)), inverse with d^-1), bit-exact.
//
// Split 256 = 4 x 64. With coefficient n = 64 a + b and slot j = 4 j2 + j1
// (a, j1 < 4; b, j2 < 64), psi a primitive 512th root, zeta = psi^64 and
// omega = psi^8:
//   X_{4 j2 + j1} = sum_b omega^(j2 b) Y_{j1}[b],
//   Y_{j1}[b]     = psi^((2 j1 + 1) b) sum_a zeta^(a (2 j1 + 1)) x_{64 a + b}.
// The 4-point step and the twist run on CUDA cores; the four 64-point cyclic
// transforms of a polynomial are four rows of one tensor-core product against
// the single matrix omega^(j2 b), by the byte-plane method of the d = 64
// kernel (ntt_tc_common.cuh). The inverse mirrors it:
//   V_{j1}[b] = sum_j2 omega^(-j2 b) Z_{4 j2 + j1}
// is the same matrix read at output column j' = -b mod 64, and
//   out_{64 a + b} = sum_j1 zeta^(-a (2 j1 + 1)) 256^-1 psi^(-(2 j1 + 1) b) V_{j1}[b].
// One matrix in shared memory serves both directions, which leaves room for
// two input buffers and a staged tile of b.
//
// A tile is 32 polynomials = 128 rows (row 32 j1 + p), so epilogue warp w
// (tensor-memory lanes 32 (w % 4) ..) holds block j1 = w % 4 of every
// polynomial. Per tile j of a CTA (one persistent CTA per SM):
//   loader (warp 17): bulk-loads input tile j into buffer j % 2 once output
//     tile j - 2 has been stored from it, and b's tile j into padded rows once
//     F(j-1) has read the previous one; L2 prefetch of a and b 3 tiles ahead
//   epilogue (warps 0-15): P(j) 4-point + twist -> forward A operand;
//     E(j-1) inverse results -> 4-point inverse in buffer (j-1) % 2 -> staged;
//     F(j) forward results (x) b -> inverse A operand
//   MMA (warp 16): fwd(j) after P(j) and F(j-1) read columns 0-255;
//     inv(j) after F(j) and E(j-1) read columns 256-511.
// The epilogue warps agree on every wait's outcome through a named barrier,
// so a timed-out wait ends all of them together; every wait is bounded.
#include <cuda_runtime.h>

#include <cstring>
#include <vector>

#include "grid_async.cuh"
#include "grid_field.cuh"
#include "grid_internal.h"
#include "grid_tc.cuh"
#include "ntt_tc_common.cuh"

namespace grid {
namespace {

using namespace tcx;

constexpr int D = 256;
constexpr int PT = ROWS / 4;                // polys per tile
constexpr int EPI_THREADS = EPI_WARPS * 32;
constexpr int NX = 2;                       // natural-order tile buffers
constexpr uint32_t XT = PT * D * 4;         // 32 KB
// b rows padded to 260 words: the 32 rows of one gather start 4 banks apart
constexpr uint32_t BROW = (D + 4) * 4;

// Offsets from the 1 KB-aligned base of dynamic shared memory.
constexpr uint32_t OFF_W = 0;               // the 64-point matrix (B of both transforms)
constexpr uint32_t OFF_AF = OFF_W + WMAT;   // forward A operand
constexpr uint32_t OFF_AI = OFF_AF + TILE;  // inverse A operand (pointwise products)
constexpr uint32_t OFF_X = OFF_AI + TILE;   // input tiles, then inverse results
constexpr uint32_t OFF_B = OFF_X + NX * XT;  // b's tile, padded rows
constexpr uint32_t OFF_BAR = OFF_B + PT * BROW;
constexpr uint32_t OFF_TADDR = OFF_BAR + 16 * 8;
constexpr uint32_t SMEM_BYTES = OFF_TADDR + 16 + 1024;  // + alignment slack
static_assert(SMEM_BYTES <= 232448, "shared memory budget");

// Device table: the matrix image (WMAT bytes), then {w, w q^-1 mod 2^32}
// Montgomery constants: forward twists psi^((2 j1 + 1) b) [4][64], inverse
// twists 256^-1 psi^(-(2 j1 + 1) b) [4][64], and zeta^2, zeta, zeta^3,
// zeta^-1, zeta^-2, zeta^-3.
constexpr uint32_t TW_F = WMAT / 8;  // in uint2 units
constexpr uint32_t TW_I = TW_F + 256;
constexpr uint32_t TW_C = TW_I + 256;
constexpr size_t TABLE_BYTES = WMAT + (256 + 256 + 8) * 8;

enum Bar : int {
  AFULL0 = 0,               // input tile landed in buffer i
  STAGED0 = AFULL0 + NX,    // output tile written into buffer i
  BFULL = STAGED0 + NX,     // b's tile landed
  BFREE,                    // F has read b's tile
  PREP, FDONE, FREAD, PREADY, IDONE, EREAD, NBARS
};
static_assert(NBARS <= 16, "barrier slots");

// All epilogue warps: true iff every one of them passes ok (named barrier 1).
__device__ __forceinline__ bool epi_all(bool ok) {
  uint32_t r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\tsetp.ne.u32 q, %1, 0;\n\t"
      "bar.red.and.pred p, 1, %2, q;\n\tselp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(r)
      : "r"((uint32_t)ok), "n"(EPI_THREADS)
      : "memory");
  return r != 0;
}

__device__ __forceinline__ void epi_sync() {
  asm volatile("bar.sync 1, %0;" ::"n"(EPI_THREADS) : "memory");
}

__device__ __forceinline__ uint32_t mulc(uint32_t x, uint2 w, uint32_t q) {
  return mont_c(x, w.x, w.y, q);
}

__global__ void __launch_bounds__(THREADS, 1)
    ntt256_tc_mulinv_kernel(const uint32_t* __restrict__ a, const uint32_t* __restrict__ b,
                            uint32_t* out, unsigned long long npolys,
                            const unsigned char* __restrict__ table, const TcConsts k,
                            uint32_t r1, int* __restrict__ err) {
  extern __shared__ __align__(1024) unsigned char sm_raw[];
  const uint32_t raw = smem_addr(sm_raw);
  unsigned char* sm = sm_raw + (((raw + 1023u) & ~1023u) - raw);
  const uint32_t s0 = smem_addr(sm);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  uint64_t* bars = reinterpret_cast<uint64_t*>(sm + OFF_BAR);
  uint32_t* taddr_slot = reinterpret_cast<uint32_t*>(sm + OFF_TADDR);
  const uint2* tw = reinterpret_cast<const uint2*>(table);

  {
    const uint4* src = reinterpret_cast<const uint4*>(table);
    uint4* w = reinterpret_cast<uint4*>(sm + OFF_W);
    for (int i = threadIdx.x; i < (int)(WMAT / 16); i += THREADS) w[i] = src[i];
  }
  if (warp == MMA_WARP) {
    tc::tmem_alloc(taddr_slot, 512);
    tc::tmem_relinquish();
    if (lane == 0) {
      for (int i = 0; i < NX; ++i) {
        mbar_init(&bars[AFULL0 + i], 1);
        mbar_init(&bars[STAGED0 + i], EPI_WARPS);
      }
      mbar_init(&bars[BFULL], 1);
      mbar_init(&bars[BFREE], EPI_WARPS);
      mbar_init(&bars[PREP], EPI_WARPS);
      mbar_init(&bars[FDONE], 1);
      mbar_init(&bars[FREAD], EPI_WARPS);
      mbar_init(&bars[PREADY], EPI_WARPS);
      mbar_init(&bars[IDONE], 1);
      mbar_init(&bars[EREAD], EPI_WARPS);
      fence_mbar_init();
    }
  }
  tc::fence_async_smem();
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tbase = *taddr_slot;
  const uint32_t R0 = tbase, R1 = tbase + 256;

  const unsigned long long ntiles = (npolys + PT - 1) / PT;
  const uint32_t n = blockIdx.x < ntiles
                         ? (uint32_t)((ntiles - 1 - blockIdx.x) / gridDim.x + 1)
                         : 0u;  // tiles of this CTA
  auto poly0 = [&](uint32_t j) -> unsigned long long {
    return ((unsigned long long)blockIdx.x + (unsigned long long)j * gridDim.x) * PT;
  };
  auto tile_bytes = [&](uint32_t j) -> uint32_t {
    const unsigned long long left = npolys - poly0(j);
    return (uint32_t)(left < PT ? left : PT) * D * 4;
  };

  if (warp == LOAD_WARP) {
    // ------------------------------------------------------------ loader
    uint32_t armed[NX] = {}, barmed = 0;
    bool ok = true;
    auto prefetch = [&](uint32_t j) {
      if (lane == 0 && j < n) {
        prefetch_l2(a + poly0(j) * D, tile_bytes(j));
        prefetch_l2(b + poly0(j) * D, tile_bytes(j));
      }
    };
    for (uint32_t j = 0; j < 3; ++j) prefetch(j);
    for (uint32_t t = 0; ok && t < n + NX; ++t) {
      const uint32_t buf = t % NX;
      unsigned char* xb = sm + OFF_X + buf * XT;
      if (t >= (uint32_t)NX) {  // store output tile t - 2, which frees the buffer
        const uint32_t js = t - NX;
        ok = warp_wait_fast(&bars[STAGED0 + buf], (js / NX) & 1, err);
        if (ok && lane == 0) {
          bulk_store(out + poly0(js) * D, xb, tile_bytes(js));
          bulk_commit();
          bulk_wait_read_all();
        }
        __syncwarp();
      }
      if (ok && t < n) {
        ++armed[buf];
        if (lane == 0) {
          mbar_arrive_expect_tx(&bars[AFULL0 + buf], tile_bytes(t));
          bulk_load(xb, a + poly0(t) * D, tile_bytes(t), &bars[AFULL0 + buf]);
        }
        __syncwarp();
        // b's tile t, one row per lane, once F(t-1) has read tile t-1
        if (t >= 1) ok = warp_wait_fast(&bars[BFREE], (t - 1) & 1, err);
        if (ok) {
          ++barmed;
          if (lane == 0) mbar_arrive_expect_tx(&bars[BFULL], tile_bytes(t));
          __syncwarp();
          if ((uint32_t)lane * D * 4 < tile_bytes(t))
            bulk_load(sm + OFF_B + lane * BROW, b + (poly0(t) + lane) * D, D * 4, &bars[BFULL]);
          __syncwarp();
        }
      }
      prefetch(t + 3);
    }
    if (lane == 0) bulk_wait_all();
    if (!ok) {
      for (int i = 0; i < NX; ++i)
        if (armed[i]) mbar_wait_sleep(&bars[AFULL0 + i], (armed[i] - 1) & 1, err);
      if (barmed) mbar_wait_sleep(&bars[BFULL], (barmed - 1) & 1, err);
    }
  } else if (warp == MMA_WARP) {
    // ------------------------------------------------------------ MMA issue
    uint32_t armed[NBARS] = {};
    auto issue = [&](uint32_t dcol, uint32_t abase, int bar) {
      tc::fence_after_sync();
      if (lane == 0) {
        issue_transform(dcol, abase, s0 + OFF_W);
        tc::mma_commit(&bars[bar]);
      }
      ++armed[bar];
      __syncwarp();
    };
    bool ok = true;
    for (uint32_t j = 0; ok && j < n; ++j) {
      ok = warp_wait_fast(&bars[PREP], j & 1, err);
      if (ok && j >= 1) ok = warp_wait_fast(&bars[FREAD], (j - 1) & 1, err);
      if (!ok) break;
      issue(R0, s0 + OFF_AF, FDONE);
      ok = warp_wait_fast(&bars[PREADY], j & 1, err);
      if (ok && j >= 1) ok = warp_wait_fast(&bars[EREAD], (j - 1) & 1, err);
      if (!ok) break;
      issue(R1, s0 + OFF_AI, IDONE);
    }
    // the last results must be read before the columns are freed
    if (ok && n > 0) warp_wait(&bars[EREAD], (n - 1) & 1, err);
    if (!ok) {
      const int started[2] = {FDONE, IDONE};
      for (int bar : started)
        if (armed[bar]) mbar_wait_sleep(&bars[bar], (armed[bar] - 1) & 1, err);
    }
  } else {
    // ------------------------------------------------------------ epilogue
    const uint32_t wl = warp & 3, cq = warp >> 2;  // block j1 = wl, columns 16 cq .. + 15
    const uint32_t p = lane;                       // polynomial of this thread's row
    const uint32_t row = 32 * wl + lane;
    const uint32_t lane_off = ((32 * wl) << 16) + 16 * cq;
    const int tid = threadIdx.x;  // 0 .. 511
    const uint32_t q = k.q;
    bool ok = true;
    // The 4-point steps give this thread coefficient / slot index bb = tid % 64
    // of polynomials tid / 64 + 8 it: its twists are fixed. Montgomery words
    // only; the Shoup companions are recomputed at use.
    const uint32_t bb = tid & 63;
    uint32_t twf[4], twi[4];
#pragma unroll
    for (int j1 = 0; j1 < 4; ++j1) {
      twf[j1] = tw[TW_F + 64 * j1 + bb].x;
      twi[j1] = tw[TW_I + 64 * j1 + bb].x;
    }
    const uint2 ci = tw[TW_C + 0], cz = tw[TW_C + 1], cz3 = tw[TW_C + 2];
    const uint2 czi1 = tw[TW_C + 3], czi2 = tw[TW_C + 4], czi3 = tw[TW_C + 5];
    auto mulw = [&](uint32_t x, uint32_t w) { return mont_c(x, w, w * k.qinv, q); };

    // P(j): Y_{j1}[bb] for 4 polynomials per thread, into the forward A operand
    auto prep = [&](uint32_t j) {
      const uint32_t* x = reinterpret_cast<const uint32_t*>(sm + OFF_X + (j % NX) * XT);
      unsigned char* af = sm + OFF_AF;
#pragma unroll
      for (int it = 0; it < 4; ++it) {
        const uint32_t pp = (it * EPI_THREADS + tid) >> 6;
        const uint32_t* xr = x + pp * D + bb;
        const uint32_t x0 = xr[0], x1 = xr[64], x2 = xr[128], x3 = xr[192];
        const uint32_t t2 = mulc(x2, ci, q), t3 = mulc(x3, ci, q);  // zeta^2 x2, zeta^2 x3
        const uint32_t e0 = add_lazy(x0, t2, r1), e1 = sub_lazy(x0, t2, q);
        const uint32_t o0 = add_lazy(x1, t3, r1), o1 = sub_lazy(x1, t3, q);
        const uint32_t s = mulc(o0, cz, q), s1 = mulc(o1, cz3, q);
        uint32_t z[4];
        z[0] = add_lazy(e0, s, r1);   // j1 = 0: zeta^(a)
        z[2] = sub_lazy(e0, s, q);    // j1 = 2: zeta^(5a)
        z[1] = add_lazy(e1, s1, r1);  // j1 = 1: zeta^(3a)
        z[3] = sub_lazy(e1, s1, q);   // j1 = 3: zeta^(7a)
#pragma unroll
        for (int j1 = 0; j1 < 4; ++j1) {
          const uint32_t y = mulw(z[j1], twf[j1]);
          *reinterpret_cast<uint32_t*>(af + sw128(32 * j1 + pp, bb >> 5, (bb & 31) >> 2, BOX) +
                                       4 * (bb & 3)) = y;
        }
      }
    };
    // F(j): forward results (x) b -> inverse A operand
    auto forward_out = [&](uint32_t j) -> bool {
      bool got = warp_wait_fast(&bars[FDONE], j & 1, err);
      got = got && warp_wait_fast(&bars[BFULL], j & 1, err);
      if (!epi_all(got)) return false;
      tc::fence_after_sync();
      uint32_t res[16];
      reduce16(R0 + lane_off, k, res);
      tc::fence_before_sync();
      __syncwarp();
      if (lane == 0) mbar_arrive(&bars[FREAD]);  // columns 0-255 free for fwd(j+1)
      // b at slots 4 (16 cq + t) + wl of polynomial p
      const uint32_t* brow = reinterpret_cast<const uint32_t*>(sm + OFF_B + p * BROW) + 64 * cq + wl;
      uint32_t bv[16];
#pragma unroll
      for (int t = 0; t < 16; ++t) bv[t] = brow[4 * t];
      __syncwarp();
      if (lane == 0) mbar_arrive(&bars[BFREE]);
#pragma unroll
      for (int t = 0; t < 16; ++t) res[t] = redc64(mad_wide(res[t], bv[t], 0ull), q, k.qinv);
      unsigned char* ai = sm + OFF_AI;
#pragma unroll
      for (int c = 0; c < 4; ++c)
        *reinterpret_cast<uint4*>(ai + sw128(row, cq >> 1, (cq & 1) * 4 + c, BOX)) =
            make_uint4(res[4 * c], res[4 * c + 1], res[4 * c + 2], res[4 * c + 3]);
      tc::fence_async_smem();
      __syncwarp();
      if (lane == 0) mbar_arrive(&bars[PREADY]);
      return true;
    };
    // E(j): inverse results -> 4-point inverse -> output tile in buffer j % 3
    auto inverse_out = [&](uint32_t j) -> bool {
      if (!epi_all(warp_wait_fast(&bars[IDONE], j & 1, err))) return false;
      tc::fence_after_sync();
      uint32_t res[16];
      reduce16(R1 + lane_off, k, res);
      tc::fence_before_sync();
      __syncwarp();
      if (lane == 0) mbar_arrive(&bars[EREAD]);  // columns 256-511 free for inv(j+1)
      uint32_t* x = reinterpret_cast<uint32_t*>(sm + OFF_X + (j % NX) * XT);
      // column 16 cq + t is V_{wl}[c] with c = -(16 cq + t) mod 64; word 64 wl + c of
      // polynomial p, its low 5 bits XORed with p (the 32 lanes hit 32 banks)
#pragma unroll
      for (int t = 0; t < 16; ++t) {
        const uint32_t c = (64u - (16u * cq + t)) & 63u;
        x[p * D + ((64 * wl + c) ^ p)] = res[t];
      }
      epi_sync();
      uint32_t o[4][4];
#pragma unroll
      for (int it = 0; it < 4; ++it) {
        const uint32_t pp = (it * EPI_THREADS + tid) >> 6;
        const uint32_t* xr = x + pp * D;
        uint32_t v[4];
#pragma unroll
        for (int j1 = 0; j1 < 4; ++j1) v[j1] = mulw(xr[(64 * j1 + bb) ^ pp], twi[j1]);
        const uint32_t p0 = add_canon(v[0], v[2], q), q0 = sub_lazy(v[0], v[2], q);
        const uint32_t p1 = add_canon(v[1], v[3], q), q1 = sub_lazy(v[1], v[3], q);
        const uint32_t tq = mulc(q1, czi2, q);
        o[it][0] = add_canon(p0, p1, q);
        o[it][1] = mulc(add_canon(q0, tq, q), czi1, q);
        o[it][2] = mulc(sub_lazy(p0, p1, q), czi2, q);
        o[it][3] = mulc(sub_lazy(q0, tq, q), czi3, q);
      }
      epi_sync();  // every swizzled word read before the tile is rewritten in order
#pragma unroll
      for (int it = 0; it < 4; ++it) {
        const uint32_t pp = (it * EPI_THREADS + tid) >> 6;
#pragma unroll
        for (int aa = 0; aa < 4; ++aa) x[pp * D + 64 * aa + bb] = o[it][aa];
      }
      tc::fence_async_smem();
      __syncwarp();
      if (lane == 0) mbar_arrive(&bars[STAGED0 + j % NX]);
      return true;
    };

    for (uint32_t j = 0; ok && j < n; ++j) {
      ok = epi_all(warp_wait_fast(&bars[AFULL0 + j % NX], (j / NX) & 1, err));
      if (!ok) break;
      prep(j);  // the forward A operand is free: F(j-1) saw fwd(j-1) complete
      tc::fence_async_smem();
      __syncwarp();
      if (lane == 0) mbar_arrive(&bars[PREP]);
      if (j >= 1 && !(ok = inverse_out(j - 1))) break;  // also frees the inverse A operand
      if (!(ok = forward_out(j))) break;
    }
    if (ok && n > 0) inverse_out(n - 1);
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == MMA_WARP) {
    tc::fence_after_sync();
    tc::tmem_dealloc(tbase, 512);
  }
}

}  // namespace

bool ntt256_tc_available(const grid_gpu_plan* p) { return p->d == 256 && p->d_tcw != nullptr; }

int launch_ntt256_tc(const grid_gpu_plan* p, const uint32_t* a, const uint32_t* b, uint32_t* out,
                     size_t npolys, cudaStream_t s) {
  if (npolys == 0) return GRID_OK;
  static int bps_cache[kMaxDevices] = {};
  int bps = 0;
  const int st =
      prepare_kernel(ntt256_tc_mulinv_kernel, SMEM_BYTES, THREADS, p->device, bps_cache, &bps);
  if (st) return st;
  const unsigned long long tiles = (npolys + PT - 1) / PT;
  const unsigned long long grid =
      tiles < (unsigned long long)p->num_sms ? tiles : (unsigned long long)p->num_sms;
  TcConsts k;
  k.q = p->f.q;
  k.qinv = p->f.qinv;
  ntt256_tc_mulinv_kernel<<<(unsigned)grid, THREADS, SMEM_BYTES, s>>>(
      a, b, out, (unsigned long long)npolys, static_cast<const unsigned char*>(p->d_tcw), k,
      p->f.r1, p->d_err);
  return cuda_status(cudaGetLastError());
}

// The 64-point matrix image (row 64 l + j, K byte 4k + i = byte l of
// 2^(8i) omega^(jk) 2^32 mod q, 128-byte-swizzled K-major), then the twist and
// 4-point constants as {Montgomery word, word * q^-1 mod 2^32}.
void build_tc256_tables(uint32_t q, uint64_t psi, std::vector<unsigned char>& out) {
  out.assign(TABLE_BYTES, 0);
  auto mulm = [q](uint64_t x, uint64_t y) { return (uint64_t)((unsigned __int128)x * y % q); };
  auto powm = [&](uint64_t x, uint64_t e) {
    uint64_t r = 1;
    x %= q;
    while (e) {
      if (e & 1) r = mulm(r, x);
      x = mulm(x, x);
      e >>= 1;
    }
    return r;
  };
  uint32_t qinv = 1;
  for (int i = 0; i < 5; ++i) qinv *= 2u - q * qinv;
  const uint64_t R = ((uint64_t)1 << 32) % q;
  const uint64_t omega = powm(psi, 8);
  for (uint32_t j = 0; j < 64; ++j)
    for (uint32_t kk = 0; kk < 64; ++kk) {
      uint64_t w = mulm(powm(omega, (j * kk) % 64), R);
      for (uint32_t i = 0; i < 4; ++i) {
        const uint32_t kb = 4 * kk + i, h = kb / 128, kc = kb % 128;
        for (uint32_t l = 0; l < 4; ++l)
          out[sw128(64 * l + j, h, kc / 16, WMAT / 2) + kc % 16] = (unsigned char)(w >> (8 * l));
        w = mulm(w, 256);  // next byte of x_k: times 2^8
      }
    }
  auto put = [&](uint32_t idx, uint64_t value) {
    const uint32_t wm = (uint32_t)mulm(value, R);
    const uint32_t pair[2] = {wm, wm * qinv};
    std::memcpy(out.data() + (size_t)idx * 8, pair, 8);
  };
  const uint64_t psi_inv = powm(psi, 2 * D - 1);
  const uint64_t dinv = powm(D, q - 2);
  for (uint32_t j1 = 0; j1 < 4; ++j1)
    for (uint32_t bb = 0; bb < 64; ++bb) {
      const uint64_t e = ((2 * j1 + 1) * bb) % (2 * D);
      put(TW_F + 64 * j1 + bb, powm(psi, e));
      put(TW_I + 64 * j1 + bb, mulm(dinv, powm(psi_inv, e)));
    }
  const uint64_t zeta = powm(psi, 64), zeta_inv = powm(psi_inv, 64);
  put(TW_C + 0, powm(zeta, 2));
  put(TW_C + 1, zeta);
  put(TW_C + 2, powm(zeta, 3));
  put(TW_C + 3, zeta_inv);
  put(TW_C + 4, powm(zeta_inv, 2));
  put(TW_C + 5, powm(zeta_inv, 3));
}

}  // namespace grid
