// Tensor-core twisted negacyclic NTT / INTT for d = 64 (tcgen05, kind::i8).
//
// Reference path replaced: TwistedNttPlan::{forward,inverse}_in_place_trusted
// (algebra/src/poly/ntt.rs:75-104) and the NTT -> Montgomery pointwise -> INTT
// chain of a negacyclic product, bit-exact.
//
// The transform is a linear map over Z_q: natural-order slot j of the forward
// output is sum_k x_k psi^((2j+1) k) and the inverse is its inverse matrix
// (d^-1 folded in). Both run as 64 x 64 matrix products with exact integer
// arithmetic on the 8-bit tensor cores:
//  * every 32-bit input word x = sum_i 2^(8i) x_i is split into byte planes
//    x_i (a 128 poly x 64 byte matrix per plane);
//  * with W' = W * 2^32 mod q (Montgomery form), plane i is multiplied by
//    W^(i) = 2^(8i) W' mod q, split into byte planes W^(i)_l. Then
//    sum_k W'[j][k] x_k = sum_l 2^(8l) E_l (mod q) with
//    E_l = sum_i x_i * W^(i)_l: four MMAs (M = 128, N = 256, one per input
//    plane and 32-byte K step) accumulate E_0..E_3 side by side in 256
//    tensor-memory columns, each entry < 4 * 64 * 255^2 < 2^24 (exact);
//  * the epilogue forms v = E_0 + 2^8 E_1 + 2^16 E_2 + 2^24 E_3 < 2^49 and
//    one Montgomery reduction returns the canonical word.
// One persistent CTA per SM streams tiles of 128 polynomials: warp 16 issues
// the TMA tensor loads (two 32-word x 128-row boxes, 128-byte swizzle, two
// input buffers) and the MMAs; warps 0-15 transpose inputs into byte planes,
// reduce, multiply by b (read straight from global memory, one tile ahead)
// and store the result rows. The forward transform of a tile (columns
// 0-255) runs while the epilogue finishes the previous tile's inverse
// (columns 256-511), so the tensor core, the CUDA cores and HBM overlap.
// Epilogue warp w owns tensor-memory lanes 32 (w % 4) .. + 31 (its rows) and
// columns 16 (w / 4) .. + 15 of each E_l block. Every wait is bounded.
#include <cuda.h>
#include <cuda_runtime.h>

#include <mutex>

#include "grid_async.cuh"
#include "grid_field.cuh"
#include "grid_internal.h"
#include "grid_tc.cuh"

namespace grid {
namespace {

constexpr int D = 64;
constexpr int ROWS = 128;  // polys per tile (MMA M)
constexpr int EPI_WARPS = 16;
constexpr int THREADS = (EPI_WARPS + 1) * 32;
constexpr uint32_t PLANE = ROWS * 64;     // one byte plane: 128 rows x 64 bytes
constexpr uint32_t TILE = 4 * PLANE;      // 32 KB: a natural tile or its 4 planes
constexpr uint32_t LBO = 128, SBO = 512;  // core-matrix strides of the plane / W layouts
constexpr uint32_t WBLK = 16384;          // matrix planes for one input plane (256 x 64 B)

// Offsets from the 1 KB-aligned base of dynamic shared memory.
constexpr uint32_t OFF_XA = 0;               // two input tiles (TMA) / their planes
constexpr uint32_t OFF_PP = OFF_XA + 2 * TILE;  // pointwise-product planes
constexpr uint32_t OFF_W = OFF_PP + TILE;       // 4 (or 8) matrix blocks
constexpr uint32_t OFF_BAR = OFF_W + 8 * WBLK;
constexpr uint32_t OFF_TADDR = OFF_BAR + 16 * 8;
constexpr uint32_t SMEM_BYTES = OFF_TADDR + 16 + 1024;  // + alignment slack
static_assert(SMEM_BYTES <= 232448, "shared memory budget");

enum Bar : int { AFULL0 = 0, AFULL1, XREADY, FDONE, PREADY, IDONE, EREAD, NBARS };

struct TcConsts {
  uint32_t q, qinv;
};

// 4 words -> their byte planes: o[i] = bytes i of (a, b, c, d).
__device__ __forceinline__ void transpose4(uint32_t a, uint32_t b, uint32_t c, uint32_t d,
                                           uint32_t (&o)[4]) {
  const uint32_t p = __byte_perm(a, b, 0x5140), q = __byte_perm(a, b, 0x7362);
  const uint32_t r = __byte_perm(c, d, 0x5140), s = __byte_perm(c, d, 0x7362);
  o[0] = __byte_perm(p, r, 0x5410);
  o[1] = __byte_perm(p, r, 0x7632);
  o[2] = __byte_perm(q, s, 0x5410);
  o[3] = __byte_perm(q, s, 0x7632);
}

// 16 words (a row's 16-byte chunk of every plane) -> 4 plane chunks.
__device__ __forceinline__ void store_planes(unsigned char* planes, uint32_t row, uint32_t chunk,
                                             const uint32_t* w) {
  uint32_t pl[4][4];
#pragma unroll
  for (int g = 0; g < 4; ++g) {
    uint32_t o[4];
    transpose4(w[4 * g], w[4 * g + 1], w[4 * g + 2], w[4 * g + 3], o);
#pragma unroll
    for (int i = 0; i < 4; ++i) pl[i][g] = o[i];
  }
#pragma unroll
  for (int i = 0; i < 4; ++i)
    *reinterpret_cast<uint4*>(planes + i * PLANE + tc::core_offset(row, chunk, LBO, SBO)) =
        make_uint4(pl[i][0], pl[i][1], pl[i][2], pl[i][3]);
}

// a * b + c with a 64-bit addend: one wide integer multiply-add.
__device__ __forceinline__ uint64_t mad_wide(uint32_t a, uint32_t b, uint64_t c) {
  uint64_t d;
  asm("mad.wide.u32 %0, %1, %2, %3;" : "=l"(d) : "r"(a), "r"(b), "l"(c));
  return d;
}

// Montgomery reduction of v < q * 2^32: v * 2^-32 mod q, canonical.
__device__ __forceinline__ uint32_t redc64(uint64_t v, uint32_t q, uint32_t qinv) {
  const uint32_t m = (uint32_t)v * qinv;
  return sub_lazy((uint32_t)(v >> 32), __umulhi(m, q), q);
}

// 16 reduced results of this thread's row: columns col0 .. col0 + 15 of the
// four E_l blocks (64 columns apart) starting at taddr; four tensor-memory
// round trips of 4 columns x 4 blocks (wider loads cost more registers than
// this kernel has).
__device__ __forceinline__ void reduce16(uint32_t taddr, const TcConsts& k, uint32_t* out) {
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    uint32_t e[4][4];
#pragma unroll
    for (int l = 0; l < 4; ++l) tc::tmem_ld4(taddr + 64 * l + 4 * c, e[l]);
    tc::tmem_ld_wait();
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      uint64_t v = mad_wide(e[1][j], 256u, (uint64_t)e[0][j]);
      v = mad_wide(e[2][j], 65536u, v);
      v = mad_wide(e[3][j], 16777216u, v);
      out[4 * c + j] = redc64(v, k.q, k.qinv);
    }
  }
}

// One transform of a 128-row tile into 256 columns at dcol: E_l at dcol + 64 l.
__device__ __forceinline__ void issue_transform(uint32_t dcol, uint32_t planes, uint32_t w) {
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int h = 0; h < 2; ++h)
      tc::mma_u8(dcol, tc::smem_desc(planes + i * PLANE + h * 256, LBO, SBO),
                 tc::smem_desc(w + i * WBLK + h * 256, LBO, SBO), tc::idesc_u8(ROWS, 256),
                 (i | h) != 0);
}

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, int x, int y,
                                            uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3}], [%4];" ::"r"(dst),
      "l"(map), "r"(x), "r"(y), "r"(bar)
      : "memory");
}

// Barrier 1 over the 512 epilogue threads, AND-reducing a flag.
__device__ __forceinline__ bool epi_and(bool ok) {
  uint32_t r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\t"
      "setp.ne.u32 p, %1, 0;\n\t"
      "bar.red.and.pred q, 1, 512, p;\n\t"
      "selp.u32 %0, 1, 0, q;\n\t}"
      : "=r"(r)
      : "r"((uint32_t)ok)
      : "memory");
  return r != 0;
}

__device__ __forceinline__ bool warp_wait(uint64_t* bar, uint32_t parity, int* err) {
  const bool ok = mbar_wait_sleep(bar, parity, err);
  return __all_sync(0xffffffffu, ok);
}

// MODE_FWD / MODE_INV: one transform per tile, results stored by phase F.
// MODE_MULINV: F = forward + Montgomery product with b -> product planes;
// E = inverse -> stored. Per tile j (this CTA's j-th tile), in order:
//   producer: fwd(j) after planes(j); inv(j-1) after F(j-1) and E(j-2)
//   epilogue: F(j), T(j+1) (planes of the next tile), E(j-1)
// so the tensor core runs fwd(j+1) and inv(j) while the CUDA cores do
// T(j+1), E(j-1) and the arithmetic of F(j+1).
template <int MODE>
__global__ void __launch_bounds__(THREADS, 1)
    ntt_tc_kernel(const __grid_constant__ CUtensorMap tmap_a, const uint32_t* __restrict__ b,
                  uint32_t* __restrict__ out, unsigned long long npolys,
                  const uint4* __restrict__ wtab, const TcConsts k, int* __restrict__ err) {
  constexpr bool kTwo = MODE == MODE_MULINV;
  extern __shared__ __align__(1024) unsigned char sm_raw[];
  const uint32_t raw = smem_addr(sm_raw);
  unsigned char* sm = sm_raw + (((raw + 1023u) & ~1023u) - raw);
  const uint32_t s0 = smem_addr(sm);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  uint64_t* bars = reinterpret_cast<uint64_t*>(sm + OFF_BAR);
  uint32_t* taddr_slot = reinterpret_cast<uint32_t*>(sm + OFF_TADDR);

  {
    // forward blocks then inverse blocks; MODE_INV's only transform is the inverse
    const uint4* w1 = wtab + (MODE == MODE_INV ? 4 * WBLK / 16 : 0);
    uint4* w = reinterpret_cast<uint4*>(sm + OFF_W);
    const int n16 = (kTwo ? 8 : 4) * WBLK / 16;
    for (int i = threadIdx.x; i < n16; i += THREADS) w[i] = w1[i];
  }
  if (warp == EPI_WARPS) {
    tc::tmem_alloc(taddr_slot, 512);
    tc::tmem_relinquish();
    if (lane == 0) {
      mbar_init(&bars[AFULL0], 1);
      mbar_init(&bars[AFULL1], 1);
      mbar_init(&bars[XREADY], EPI_WARPS);
      mbar_init(&bars[FDONE], 1);
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

  const unsigned long long ntiles = (npolys + ROWS - 1) / ROWS;
  const uint32_t n = blockIdx.x < ntiles
                         ? (uint32_t)((ntiles - 1 - blockIdx.x) / gridDim.x + 1)
                         : 0u;  // tiles of this CTA
  auto tile_row0 = [&](uint32_t j) -> unsigned long long {
    return ((unsigned long long)blockIdx.x + (unsigned long long)j * gridDim.x) * ROWS;
  };

  if (warp == EPI_WARPS) {
    // ------------------------------------------------------------ producer
    uint32_t armed[NBARS] = {};
    auto load = [&](uint32_t j) {
      const int bar = AFULL0 + (j & 1);
      ++armed[bar];
      if (lane == 0) {
        const uint32_t dst = s0 + OFF_XA + (j & 1) * TILE;
        mbar_arrive_expect_tx(&bars[bar], TILE);
        tma_load_2d(dst, &tmap_a, 0, (int)tile_row0(j), smem_addr(&bars[bar]));
        tma_load_2d(dst + 2 * PLANE, &tmap_a, 32, (int)tile_row0(j), smem_addr(&bars[bar]));
      }
      __syncwarp();
    };
    auto issue = [&](uint32_t dcol, uint32_t planes, uint32_t w, int bar) {
      tc::fence_after_sync();
      if (lane == 0) {
        issue_transform(dcol, planes, w);
        tc::mma_commit(&bars[bar]);
      }
      ++armed[bar];
      __syncwarp();
    };
    auto inverse = [&](uint32_t j) -> bool {  // inv(j): after F(j) and E(j-1)
      if (!warp_wait(&bars[PREADY], j & 1, err)) return false;
      if (j >= 1 && !warp_wait(&bars[EREAD], (j - 1) & 1, err)) return false;
      issue(R1, s0 + OFF_PP, s0 + OFF_W + 4 * WBLK, IDONE);
      return true;
    };
    bool ok = true;
    if (n > 0) load(0);
    if (n > 1) load(1);
    for (uint32_t j = 0; ok && j < n; ++j) {
      ok = warp_wait(&bars[XREADY], j & 1, err);
      if (ok && j >= 1) {
        // fwd(j-1) is done with its input buffer: refill it with tile j+1
        ok = warp_wait(&bars[FDONE], (j - 1) & 1, err);
        if (ok && j + 1 < n) load(j + 1);
      }
      if (!ok) break;
      issue(R0, s0 + OFF_XA + (j & 1) * TILE, s0 + OFF_W, FDONE);
      if (kTwo && j >= 1) ok = inverse(j - 1);
    }
    if (ok && n > 0) {
      if (kTwo) ok = inverse(n - 1);
      // the last results must be read before the columns are freed
      if (ok) warp_wait(&bars[kTwo ? EREAD : PREADY], (n - 1) & 1, err);
    }
    if (!ok) {
      const int started[4] = {AFULL0, AFULL1, FDONE, IDONE};
      for (int bar : started)
        if (armed[bar]) mbar_wait_sleep(&bars[bar], (armed[bar] - 1) & 1, err);
    }
  } else {
    // ------------------------------------------------------------ epilogue
    const uint32_t wl = warp & 3, cq = warp >> 2;
    const uint32_t row = 32 * wl + lane;
    const uint32_t lane_off = ((32 * wl) << 16) + 16 * cq;
    bool ok = true;

    // T(j): this thread's 16 input words -> plane chunk cq of every plane
    auto transpose_tile = [&](uint32_t j) {
      unsigned char* xa = sm + OFF_XA + (j & 1) * TILE;
      ok = ok && warp_wait(&bars[AFULL0 + (j & 1)], (j >> 1) & 1, err);
      uint32_t w[16];
      if (ok) {
        const unsigned char* box = xa + (cq >> 1) * 2 * PLANE + row * 128;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          const uint32_t chunk = ((cq & 1) * 4 + c) ^ (row & 7);
          const uint4 v = *reinterpret_cast<const uint4*>(box + chunk * 16);
          w[4 * c] = v.x, w[4 * c + 1] = v.y, w[4 * c + 2] = v.z, w[4 * c + 3] = v.w;
        }
      }
      ok = epi_and(ok);  // every read of the tile done before planes overwrite it
      if (!ok) return;
      store_planes(xa, row, cq, w);
      tc::fence_async_smem();
      __syncwarp();
      if (lane == 0) mbar_arrive(&bars[XREADY]);
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
    auto store_row = [&](uint32_t j, const uint32_t* res) {
      const unsigned long long r = tile_row0(j) + row;
      if (r < npolys) {
        uint4* dst = reinterpret_cast<uint4*>(out + r * D + 16 * cq);
#pragma unroll
        for (int c = 0; c < 4; ++c)
          dst[c] = make_uint4(res[4 * c], res[4 * c + 1], res[4 * c + 2], res[4 * c + 3]);
      }
    };
    // E(j): inverse results of tile j
    auto inverse_out = [&](uint32_t j) {
      ok = ok && warp_wait(&bars[IDONE], j & 1, err);
      if (!ok) return;
      tc::fence_after_sync();
      uint32_t res[16];
      reduce16(R1 + lane_off, k, res);
      tc::fence_before_sync();
      __syncwarp();
      if (lane == 0) mbar_arrive(&bars[EREAD]);
      store_row(j, res);
    };

    uint4 bv[4];
    if (n > 0) {
      if (kTwo) load_b(0, bv);
      transpose_tile(0);
    }
    for (uint32_t j = 0; j < n; ++j) {
      // F(j)
      ok = ok && warp_wait(&bars[FDONE], j & 1, err);
      uint32_t res[16];
      if (ok) {
        tc::fence_after_sync();
        reduce16(R0 + lane_off, k, res);
        tc::fence_before_sync();
        if (kTwo) {
#pragma unroll
          for (int c = 0; c < 4; ++c) {  // Montgomery product with b: t * b < q * 2^32
            res[4 * c] = redc64(mad_wide(res[4 * c], bv[c].x, 0ull), k.q, k.qinv);
            res[4 * c + 1] = redc64(mad_wide(res[4 * c + 1], bv[c].y, 0ull), k.q, k.qinv);
            res[4 * c + 2] = redc64(mad_wide(res[4 * c + 2], bv[c].z, 0ull), k.q, k.qinv);
            res[4 * c + 3] = redc64(mad_wide(res[4 * c + 3], bv[c].w, 0ull), k.q, k.qinv);
          }
          // inv(j-1) must be done reading the product planes
          if (j >= 1) ok = warp_wait(&bars[IDONE], (j - 1) & 1, err);
          if (ok) {
            store_planes(sm + OFF_PP, row, cq, res);
            tc::fence_async_smem();
          }
        } else {
          store_row(j, res);
        }
        __syncwarp();
        if (ok && lane == 0) mbar_arrive(&bars[PREADY]);
      }
      if (kTwo && j + 1 < n) load_b(j + 1, bv);
      if (j + 1 < n) transpose_tile(j + 1);
      if (!ok) break;
      if (kTwo && j >= 1) inverse_out(j - 1);
    }
    if (kTwo && ok && n > 0) inverse_out(n - 1);
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == EPI_WARPS) {
    tc::fence_after_sync();
    tc::tmem_dealloc(tbase, 512);
  }
}

using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                 const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                 const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                 CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// The driver's tensor-map encoder, looked up once through the runtime (the
// library does not link the driver library directly).
EncodeTiled encoder() {
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

template <int MODE>
int run_tc(const grid_gpu_plan* p, const uint32_t* a, const uint32_t* b, uint32_t* out,
           size_t npolys, cudaStream_t s) {
  EncodeTiled enc = encoder();
  if (!enc) return GRID_ERR_CUDA;
  // Rows of 64 words, boxes of 32 words x 128 rows with 128-byte swizzle.
  CUtensorMap map;
  const cuuint64_t dims[2] = {64, (cuuint64_t)npolys};
  const cuuint64_t strides[1] = {256};
  const cuuint32_t box[2] = {32, ROWS};
  const cuuint32_t estr[2] = {1, 1};
  if (enc(&map, CU_TENSOR_MAP_DATA_TYPE_UINT32, 2, const_cast<uint32_t*>(a), dims, strides, box,
          estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
          CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
    return GRID_ERR_CUDA;
  static int bps_cache[kMaxDevices] = {};
  int bps = 0;
  const int st =
      prepare_kernel(ntt_tc_kernel<MODE>, SMEM_BYTES, THREADS, p->device, bps_cache, &bps);
  if (st) return st;
  const unsigned long long tiles = (npolys + ROWS - 1) / ROWS;
  const unsigned long long grid =
      tiles < (unsigned long long)p->num_sms ? tiles : (unsigned long long)p->num_sms;
  TcConsts k;
  k.q = p->f.q;
  k.qinv = p->f.qinv;
  ntt_tc_kernel<MODE><<<(unsigned)grid, THREADS, SMEM_BYTES, s>>>(
      map, b, out, (unsigned long long)npolys, reinterpret_cast<const uint4*>(p->d_tcw), k,
      p->d_err);
  return cuda_status(cudaGetLastError());
}

}  // namespace

bool ntt_tc_available(const grid_gpu_plan* p) { return p->d == 64 && p->d_tcw != nullptr; }

int launch_ntt_tc(const grid_gpu_plan* p, int mode, const uint32_t* a, const uint32_t* b,
                  uint32_t* out, size_t npolys, cudaStream_t s) {
  if (npolys == 0) return GRID_OK;
  if (npolys > (size_t)INT32_MAX - ROWS) return GRID_ERR_INVALID_PARAMETERS;  // TMA row coordinate
  switch (mode) {
    case MODE_FWD: return run_tc<MODE_FWD>(p, a, nullptr, out, npolys, s);
    case MODE_INV: return run_tc<MODE_INV>(p, a, nullptr, out, npolys, s);
    case MODE_MULINV: return run_tc<MODE_MULINV>(p, a, b, out, npolys, s);
    default: return GRID_ERR_INVALID_PARAMETERS;
  }
}

// Matrix byte planes in the MMA B layout (K-major, no swizzle), 16 KB per
// (transform, input plane i): row n = 64 l + j holds byte l of
// W^(i)[j][k] = 2^(8i) W'[j][k] mod q at K position k, W' the transform
// matrix in Montgomery form. Order: forward i = 0..3, then inverse i = 0..3.
void build_tc_tables(uint32_t q, uint32_t d, uint64_t psi, uint64_t ninv,
                     std::vector<unsigned char>& out) {
  out.assign(8 * WBLK, 0);
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
      uint64_t wf = mulm(powm(psi, ef), R);
      uint64_t wi = mulm(mulm(powm(psi_inv, ei), ninv), R);
      for (uint32_t i = 0; i < 4; ++i) {
        for (uint32_t l = 0; l < 4; ++l) {
          const uint32_t off = tc::core_offset(64 * l + j, kk / 16, LBO, SBO) + kk % 16;
          out[i * WBLK + off] = (unsigned char)(wf >> (8 * l));
          out[(4 + i) * WBLK + off] = (unsigned char)(wi >> (8 * l));
        }
        wf = mulm(wf, 256);  // next plane: times 2^8
        wi = mulm(wi, 256);
      }
    }
}

}  // namespace grid
