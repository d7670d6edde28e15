// Tensor-core twisted negacyclic NTT / INTT for d = 64 (tcgen05, kind::i8).
//
// Reference path replaced: TwistedNttPlan::{forward,inverse}_in_place_trusted
// (algebra/src/poly/ntt.rs:75-104) and the NTT -> Montgomery pointwise -> INTT
// chain of a negacyclic product, bit-exact.
//
// The transform is a linear map over Z_q: natural-order slot j of the forward
// output is sum_k x_k psi^((2j+1) k) and the inverse is its inverse matrix
// (d^-1 folded in). Both run as exact integer matrix products on the 8-bit
// tensor cores:
//  * a tile of 128 polynomials is read as a 128 x 256 byte matrix in its
//    natural memory order, byte 4k + i = byte i of word x_k;
//  * with W' = W * 2^32 mod q (Montgomery form) and W^(i) = 2^(8i) W' mod q,
//    B[64 l + j][4k + i] = byte l of W^(i)[j][k]. Then the MMA product
//    E[64 l + j] = sum_{k,i} byte_i(x_k) byte_l(W^(i)[j][k]) satisfies
//    sum_k W'[j][k] x_k = sum_l 2^(8l) E_l[j] (mod q), each E entry
//    < 256 * 255^2 < 2^24 (exact in int32): eight MMAs (M = 128, N = 256,
//    K = 32) per transform, straight from the TMA-loaded tile;
//  * the epilogue forms v = E_0 + 2^8 E_1 + 2^16 E_2 + 2^24 E_3 < 2^49 and
//    one Montgomery reduction returns the canonical word.
// Operands use the 128-byte-swizzled K-major layout that TMA writes: a 128 x
// 256 byte tile is two boxes (K bytes 0-127, 128-255) of 128-byte rows, row r
// of a box at 128 r with 16-byte chunk c at position c ^ (r % 8).
// One persistent CTA per SM: warp 17 moves data (TMA loads of input tiles
// into two buffers, TMA stores of result tiles, L2 prefetch two tiles
// ahead), warp 16 issues the MMAs, warps 0-15 reduce, multiply by b (read
// straight from global memory one tile ahead) and write result tiles. The
// forward transform of tile j+1 (tensor-memory columns 0-255) runs while the
// epilogue finishes the inverse of tile j-1 (columns 256-511). Epilogue warp
// w owns tensor-memory lanes 32 (w % 4) .. + 31 (its rows) and columns
// 16 (w / 4) .. + 15 of each E_l block. Every wait is bounded.
#include <cuda.h>
#include <cuda_runtime.h>

#include <mutex>

#include "grid_async.cuh"
#include "grid_field.cuh"
#include "grid_internal.h"
#include "grid_tc.cuh"
#include "ntt_tc_common.cuh"

namespace grid {
namespace {

using namespace tcx;

constexpr int D = 64;
// Offsets from the 1 KB-aligned base of dynamic shared memory.
constexpr uint32_t OFF_XA = 0;                  // two input tiles / staged results
constexpr uint32_t OFF_PP = OFF_XA + 2 * TILE;  // pointwise products (inverse's A)
constexpr uint32_t OFF_W = OFF_PP + TILE;       // forward, inverse B matrices
constexpr uint32_t OFF_BAR = OFF_W + 2 * WMAT;
constexpr uint32_t OFF_TADDR = OFF_BAR + 16 * 8;
constexpr uint32_t SMEM_BYTES = OFF_TADDR + 16 + 1024;  // + alignment slack
static_assert(SMEM_BYTES <= 232448, "shared memory budget");

enum Bar : int {
  AFULL0 = 0, AFULL1,  // input tile landed in buffer 0 / 1
  STAGED0, STAGED1,    // result tile written into buffer 0 / 1
  FDONE, FREAD, PREADY, IDONE, EREAD, NBARS
};

// MODE_FWD / MODE_INV: one transform per tile, results written by phase F.
// MODE_MULINV: F = forward + Montgomery product with b -> product tile;
// E = inverse -> results. Per tile j of this CTA:
//   MMA warp: fwd(j) once tile j is loaded and F(j-1) has read columns
//             0-255 (FREAD); then inv(j-1) once F(j-1) has written the
//             product tile (PREADY) and E(j-2) has read columns 256-511
//   epilogue: F(j), then E(j-1)
//   loader:   buffer t & 1 holds input tile t until fwd(t) is done, then a
//             result tile (single transform: tile t; two: tile t-1), which it
//             stores before loading tile t + 2.
template <int MODE>
__global__ void __launch_bounds__(THREADS, 1)
    ntt_tc_kernel(const __grid_constant__ CUtensorMap tmap_a,
                  const __grid_constant__ CUtensorMap tmap_out, const uint32_t* __restrict__ a,
                  const uint32_t* __restrict__ b, unsigned long long npolys,
                  const uint4* __restrict__ wtab, const TcConsts k, int* __restrict__ err,
                  const uint4* __restrict__ ptiles, unsigned long long nptiles) {
  constexpr bool kTwo = MODE == MODE_MULINV;
  constexpr bool kPm = MODE == MODE_FWD_PM;
  extern __shared__ __align__(1024) unsigned char sm_raw[];
  const uint32_t raw = smem_addr(sm_raw);
  unsigned char* sm = sm_raw + (((raw + 1023u) & ~1023u) - raw);
  const uint32_t s0 = smem_addr(sm);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  uint64_t* bars = reinterpret_cast<uint64_t*>(sm + OFF_BAR);
  uint32_t* taddr_slot = reinterpret_cast<uint32_t*>(sm + OFF_TADDR);

  {
    // forward matrix then inverse matrix; MODE_INV's only transform is the inverse
    const uint4* w1 = wtab + (MODE == MODE_INV ? WMAT / 16 : 0);
    uint4* w = reinterpret_cast<uint4*>(sm + OFF_W);
    const int n16 = (kTwo ? 2 : 1) * WMAT / 16;
    for (int i = threadIdx.x; i < n16; i += THREADS) w[i] = w1[i];
  }
  if (warp == MMA_WARP) {
    tc::tmem_alloc(taddr_slot, 512);
    tc::tmem_relinquish();
    if (lane == 0) {
      mbar_init(&bars[AFULL0], 1);
      mbar_init(&bars[AFULL1], 1);
      mbar_init(&bars[STAGED0], EPI_WARPS);
      mbar_init(&bars[STAGED1], EPI_WARPS);
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

  // Point-major mode with a tile list (ptiles): tile t reads 128 polys from
  // row x, stores them at column y, and rows from z on (past an instance) as 0.
  const bool listed = kPm && ptiles != nullptr;
  const unsigned long long ntiles = listed ? nptiles : (npolys + ROWS - 1) / ROWS;
  const uint32_t n = blockIdx.x < ntiles
                         ? (uint32_t)((ntiles - 1 - blockIdx.x) / gridDim.x + 1)
                         : 0u;  // tiles of this CTA
  auto tile_index = [&](uint32_t j) -> unsigned long long {
    return (unsigned long long)blockIdx.x + (unsigned long long)j * gridDim.x;
  };
  // first source row / destination row (point-major: column) of tile j
  auto tile_row0 = [&](uint32_t j) -> unsigned long long {
    return listed ? (unsigned long long)ptiles[tile_index(j)].x : tile_index(j) * ROWS;
  };
  auto tile_out0 = [&](uint32_t j) -> unsigned long long {
    return listed ? (unsigned long long)ptiles[tile_index(j)].y : tile_index(j) * ROWS;
  };
  auto tile_valid = [&](uint32_t j) -> uint32_t {
    return listed ? ptiles[tile_index(j)].z : (uint32_t)ROWS;
  };

  if (warp == LOAD_WARP) {
    // ------------------------------------------------------------ loader
    const uint32_t lag = kTwo ? 3u : 2u;  // result staged in buffer t & 1: tile t - lag
    uint32_t armed[2] = {}, staged_seen[2] = {};
    bool ok = true;
    auto prefetch = [&](uint32_t j) {
      if (lane == 0 && j < n) {
        const unsigned long long r0 = tile_row0(j);
        const unsigned long long left = npolys - r0;
        const uint32_t bytes = (uint32_t)((left < ROWS ? left : ROWS) * D * 4);
        prefetch_l2(a + r0 * D, bytes);
        if (kTwo) prefetch_l2(b + r0 * D, bytes);
      }
    };
    prefetch(0);
    prefetch(1);
    prefetch(2);
    for (uint32_t t = 0; ok && t < n + lag; ++t) {
      const uint32_t buf = t & 1;
      const uint32_t dst = s0 + OFF_XA + buf * TILE;
      // Buffer t & 1 is free for tile t once fwd(t - 2) has read it. For t >= lag
      // the STAGED wait below implies that (the epilogue stages tile t - lag
      // only after F(t - 2)). A parity wait on FDONE itself could alias: with
      // load t - 1 issued, fwd(t - 1) may complete too, and a barrier two phases
      // past the awaited one reads as not yet there. The two-transform mode
      // needs fwd(0) before load 2: it waits for it before issuing load 1, when
      // no second phase can complete.
      if (kTwo && t == 1 && n > 0) ok = warp_wait_fast(&bars[FDONE], 0, err);
      if (ok && t >= lag) {
        const uint32_t js = t - lag;
        ok = warp_wait_fast(&bars[STAGED0 + buf], staged_seen[buf]++ & 1, err);
        if (ok && lane == 0) {
          if constexpr (kPm) {  // [64 points][128 polys] -> columns row0.. of the [d][npolys] output
            tma_store_2d(&tmap_out, (int)tile_out0(js), 0, dst);
          } else {
            tma_store_2d(&tmap_out, 0, (int)tile_row0(js), dst);
            tma_store_2d(&tmap_out, 32, (int)tile_row0(js), dst + BOX);
          }
          bulk_commit();
          bulk_wait_read_all();  // the buffer may be refilled once the store has read it
        }
        __syncwarp();
      }
      if (ok && t < n) {
        ++armed[buf];
        if (lane == 0) {
          uint64_t* bar = &bars[AFULL0 + buf];
          mbar_arrive_expect_tx(bar, TILE);
          tma_load_2d(dst, &tmap_a, 0, (int)tile_row0(t), smem_addr(bar));
          tma_load_2d(dst + BOX, &tmap_a, 32, (int)tile_row0(t), smem_addr(bar));
        }
        __syncwarp();
      }
      prefetch(t + 2);
    }
    if (lane == 0) bulk_wait_all();
    if (!ok)
      for (int i = 0; i < 2; ++i)
        if (armed[i]) mbar_wait_sleep(&bars[AFULL0 + i], (armed[i] - 1) & 1, err);
  } else if (warp == MMA_WARP) {
    // ------------------------------------------------------------ MMA issue
    uint32_t armed[NBARS] = {};
    auto issue = [&](uint32_t dcol, uint32_t abase, uint32_t w, int bar) {
      tc::fence_after_sync();
      if (lane == 0) {
        issue_transform(dcol, abase, w);
        tc::mma_commit(&bars[bar]);
      }
      ++armed[bar];
      __syncwarp();
    };
    auto inverse = [&](uint32_t j) -> bool {  // inv(j): after F(j) and E(j-1)
      if (!warp_wait_fast(&bars[PREADY], j & 1, err)) return false;
      if (j >= 1 && !warp_wait_fast(&bars[EREAD], (j - 1) & 1, err)) return false;
      issue(R1, s0 + OFF_PP, s0 + OFF_W + WMAT, IDONE);
      return true;
    };
    bool ok = true;
    for (uint32_t j = 0; ok && j < n; ++j) {
      ok = warp_wait_fast(&bars[AFULL0 + (j & 1)], (j >> 1) & 1, err);
      if (ok && j >= 1) ok = warp_wait_fast(&bars[FREAD], (j - 1) & 1, err);  // F(j-1) read R0
      if (!ok) break;
      issue(R0, s0 + OFF_XA + (j & 1) * TILE, s0 + OFF_W, FDONE);
      if (kTwo && j >= 1) ok = inverse(j - 1);
    }
    if (ok && n > 0) {
      if (kTwo) ok = inverse(n - 1);
      // the last results must be read before the columns are freed
      if (ok) warp_wait(&bars[kTwo ? EREAD : FREAD], (n - 1) & 1, err);
    }
    if (!ok) {
      const int started[2] = {FDONE, IDONE};
      for (int bar : started)
        if (armed[bar]) mbar_wait_sleep(&bars[bar], (armed[bar] - 1) & 1, err);
    }
  } else {
    // ------------------------------------------------------------ epilogue
    const uint32_t wl = warp & 3, cq = warp >> 2;
    const uint32_t row = 32 * wl + lane;
    const uint32_t lane_off = ((32 * wl) << 16) + 16 * cq;
    bool ok = true;

    // 16 words (columns 16 cq .. + 15 of this row) into a swizzled tile; the
    // point-major mode writes the tile transposed, [point][row] (a warp's 32
    // rows of one point are 32 consecutive words: no bank conflict)
    auto put_row = [&](unsigned char* tile, const uint32_t* res, uint32_t valid) {
      if constexpr (kPm) {
        uint32_t* t = reinterpret_cast<uint32_t*>(tile);
        const bool keep = row < valid;
#pragma unroll
        for (int c = 0; c < 16; ++c) t[(16 * cq + c) * ROWS + row] = keep ? res[c] : 0u;
      } else {
#pragma unroll
        for (int c = 0; c < 4; ++c)
          *reinterpret_cast<uint4*>(tile + sw128(row, cq >> 1, (cq & 1) * 4 + c, BOX)) =
              make_uint4(res[4 * c], res[4 * c + 1], res[4 * c + 2], res[4 * c + 3]);
      }
    };
    // Result tile j -> buffer (j + off) & 1 (a tile whose forward is done)
    auto stage = [&](uint32_t j, const uint32_t* res) {
      const uint32_t buf = (j + (kTwo ? 1u : 0u)) & 1;
      put_row(sm + OFF_XA + buf * TILE, res, tile_valid(j));
      tc::fence_async_smem();
      __syncwarp();
      if (lane == 0) mbar_arrive(&bars[STAGED0 + buf]);
    };
    auto load_b = [&](uint32_t j, uint4 (&bv)[4]) {
      const unsigned long long r = tile_row0(j) + row;
#pragma unroll
      for (int c = 0; c < 4; ++c) bv[c] = make_uint4(0, 0, 0, 0);
      if (r < npolys) {
        const uint4* src = reinterpret_cast<const uint4*>(b + r * D + 16 * cq);
#pragma unroll
        for (int c = 0; c < 4; ++c) bv[c] = __ldg(src + c);
      }
    };
    // E(j): inverse results of tile j
    auto inverse_out = [&](uint32_t j) {
      ok = ok && warp_wait_fast(&bars[IDONE], j & 1, err);
      if (!ok) return;
      tc::fence_after_sync();
      uint32_t res[16];
      reduce16(R1 + lane_off, k, res);
      tc::fence_before_sync();
      __syncwarp();
      if (lane == 0) mbar_arrive(&bars[EREAD]);
      stage(j, res);
    };

    uint4 bv[4];
    if (kTwo && n > 0) load_b(0, bv);
    for (uint32_t j = 0; ok && j < n; ++j) {
      // F(j)
      ok = warp_wait_fast(&bars[FDONE], j & 1, err);
      if (!ok) break;
      tc::fence_after_sync();
      uint32_t res[16];
      reduce16(R0 + lane_off, k, res);
      tc::fence_before_sync();
      __syncwarp();
      if (lane == 0) mbar_arrive(&bars[FREAD]);  // columns 0-255 free for fwd(j+1)
      if (kTwo) {
#pragma unroll
        for (int c = 0; c < 4; ++c) {  // Montgomery product with b: t * b < q * 2^32
          res[4 * c] = redc64(mad_wide(res[4 * c], bv[c].x, 0ull), k.q, k.qinv);
          res[4 * c + 1] = redc64(mad_wide(res[4 * c + 1], bv[c].y, 0ull), k.q, k.qinv);
          res[4 * c + 2] = redc64(mad_wide(res[4 * c + 2], bv[c].z, 0ull), k.q, k.qinv);
          res[4 * c + 3] = redc64(mad_wide(res[4 * c + 3], bv[c].w, 0ull), k.q, k.qinv);
        }
        // inv(j-1) must be done reading the product tile
        if (j >= 1) ok = warp_wait_fast(&bars[IDONE], (j - 1) & 1, err);
        if (!ok) break;
        put_row(sm + OFF_PP, res, (uint32_t)ROWS);
        tc::fence_async_smem();
        __syncwarp();
        if (lane == 0) mbar_arrive(&bars[PREADY]);
        if (j + 1 < n) load_b(j + 1, bv);
        if (j >= 1) inverse_out(j - 1);
      } else {
        stage(j, res);
      }
    }
    if (kTwo && ok && n > 0) inverse_out(n - 1);
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == MMA_WARP) {
    tc::fence_after_sync();
    tc::tmem_dealloc(tbase, 512);
  }
}

// ptiles / nptiles / ps_out: the point-major mode's tile list and row length
// (defaults: consecutive tiles, npolys rounded up to a multiple of 4).
template <int MODE>
int run_tc(const grid_gpu_plan* p, const uint32_t* a, const uint32_t* b, uint32_t* out,
           size_t npolys, cudaStream_t s, const uint4* ptiles = nullptr,
           unsigned long long nptiles = 0, unsigned long long ps_out = 0) {
  EncodeTiled enc = encoder();
  if (!enc) return GRID_ERR_CUDA;
  // Rows of 64 words, boxes of 32 words x 128 rows with 128-byte swizzle.
  CUtensorMap map_a, map_out;
  const cuuint64_t dims[2] = {64, (cuuint64_t)npolys};
  const cuuint64_t strides[1] = {256};
  const cuuint32_t box[2] = {32, ROWS};
  const cuuint32_t estr[2] = {1, 1};
  for (int m = 0; m < 2; ++m)
    if (enc(m ? &map_out : &map_a, CU_TENSOR_MAP_DATA_TYPE_UINT32, 2,
            m ? (void*)out : (void*)const_cast<uint32_t*>(a), dims, strides, box, estr,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
            CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
      return GRID_ERR_CUDA;
  if (MODE == MODE_FWD_PM) {
    // output [64 points][ps], ps = npolys rounded up to a multiple of 4 (rows
    // of whole 16-byte units); one box of 128 polys x 64 points per tile, the
    // pad polys transformed from the zero fill past the input
    const cuuint64_t ps = ps_out ? ps_out : ((cuuint64_t)npolys + 3) / 4 * 4;
    const cuuint64_t pdims[2] = {ps, 64};
    const cuuint64_t pstrides[1] = {ps * 4};
    const cuuint32_t pbox[2] = {ROWS, 64};
    if (enc(&map_out, CU_TENSOR_MAP_DATA_TYPE_UINT32, 2, (void*)out, pdims, pstrides, pbox, estr,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
            CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
      return GRID_ERR_CUDA;
  }
  static int bps_cache[kMaxDevices] = {};
  int bps = 0;
  const int st =
      prepare_kernel(ntt_tc_kernel<MODE>, SMEM_BYTES, THREADS, p->device, bps_cache, &bps);
  if (st) return st;
  const unsigned long long tiles = ptiles ? nptiles : (npolys + ROWS - 1) / ROWS;
  const unsigned long long grid =
      tiles < (unsigned long long)p->num_sms ? tiles : (unsigned long long)p->num_sms;
  TcConsts k;
  k.q = p->f.q;
  k.qinv = p->f.qinv;
  ntt_tc_kernel<MODE><<<(unsigned)grid, THREADS, SMEM_BYTES, s>>>(
      map_a, map_out, a, b, (unsigned long long)npolys, reinterpret_cast<const uint4*>(p->d_tcw), k,
      p->d_err, ptiles, nptiles);
  return cuda_status(cudaGetLastError());
}

}  // namespace

// The driver's tensor-map encoder, looked up once through the runtime (the
// library does not link the driver library directly).
tcx::EncodeTiled tcx::encoder() {
  static EncodeTiled fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiled>(p);
  });
  return fn;
}

bool ntt_tc_available(const grid_gpu_plan* p) { return p->d == 64 && p->d_tcw != nullptr; }

int launch_ntt_tc_pm_tiles(const grid_gpu_plan* p, const uint32_t* a, size_t npolys,
                           uint32_t* out, unsigned long long ps_out, const uint4* ptiles,
                           unsigned long long nptiles, cudaStream_t s) {
  if (nptiles == 0) return GRID_OK;
  if (!ptiles || a == out) return GRID_ERR_INVALID_PARAMETERS;
  // TMA coordinates (source rows, destination columns) are 32-bit; the row
  // stride of the [64][ps_out] output is a multiple of 16 bytes
  if (npolys > (size_t)INT32_MAX - ROWS || ps_out > (unsigned long long)INT32_MAX - ROWS ||
      ps_out % 4)
    return GRID_ERR_INVALID_PARAMETERS;
  return run_tc<MODE_FWD_PM>(p, a, nullptr, out, npolys, s, ptiles, nptiles, ps_out);
}

int launch_ntt_tc(const grid_gpu_plan* p, int mode, const uint32_t* a, const uint32_t* b,
                  uint32_t* out, size_t npolys, cudaStream_t s) {
  if (npolys == 0) return GRID_OK;
  if (npolys > (size_t)INT32_MAX - ROWS) return GRID_ERR_INVALID_PARAMETERS;  // TMA row coordinate
  switch (mode) {
    case MODE_FWD: return run_tc<MODE_FWD>(p, a, nullptr, out, npolys, s);
    case MODE_INV: return run_tc<MODE_INV>(p, a, nullptr, out, npolys, s);
    case MODE_MULINV: return run_tc<MODE_MULINV>(p, a, b, out, npolys, s);
    case MODE_FWD_PM:
      // tiles of other CTAs still read the input while a tile's columns land
      if (a == out) return GRID_ERR_INVALID_PARAMETERS;
      return run_tc<MODE_FWD_PM>(p, a, nullptr, out, npolys, s);
    default: return GRID_ERR_INVALID_PARAMETERS;
  }
}

// B matrices in the tiles' 128-byte-swizzled K-major layout, 64 KB per
// transform (256 rows x 256 K bytes, two boxes of 128 K bytes): row
// n = 64 l + j, K byte 4k + i holds byte l of W^(i)[j][k] = 2^(8i) W'[j][k]
// mod q, W' the transform matrix in Montgomery form. Forward, then inverse.
void build_tc_tables(uint32_t q, uint32_t d, uint64_t psi, uint64_t ninv,
                     std::vector<unsigned char>& out) {
  out.assign(2 * WMAT, 0);
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
  const uint64_t R = ((uint64_t)1 << 32) % q;
  const uint64_t psi_inv = powm(psi, q - 2);
  for (uint32_t j = 0; j < d; ++j)
    for (uint32_t kk = 0; kk < d; ++kk) {
      // forward: slot j <- x_k psi^((2j+1)k); inverse: out_j <- X_k d^-1 psi^-((2k+1)j)
      const uint64_t ef = ((uint64_t)(2 * j + 1) * kk) % (2 * d);
      const uint64_t ei = ((uint64_t)(2 * kk + 1) * j) % (2 * d);
      uint64_t w[2] = {mulm(powm(psi, ef), R), mulm(mulm(powm(psi_inv, ei), ninv), R)};
      for (uint32_t i = 0; i < 4; ++i) {
        const uint32_t kb = 4 * kk + i, h = kb / 128, kc = kb % 128;
        for (uint32_t l = 0; l < 4; ++l) {
          const uint32_t n = 64 * l + j;
          const uint32_t off = sw128(n, h, kc / 16, WMAT / 2) + kc % 16;
          for (int t = 0; t < 2; ++t) out[t * WMAT + off] = (unsigned char)(w[t] >> (8 * l));
        }
        for (int t = 0; t < 2; ++t) w[t] = mulm(w[t], 256);  // next byte: times 2^8
      }
    }
}

}  // namespace grid
