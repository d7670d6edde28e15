// Shared pieces of the tensor-core transforms (d = 64 in ntt_tc.cu, d = 256
// in ntt256_tc.cu): warp roles, the 128-byte-swizzled K-major operand layout
// that TMA writes, the byte-plane reduction of tensor-memory results, the MMA
// sequence of one transform and bounded barrier waits.
//
// A transform multiplies a 128-row tile of 64-word vectors (128 x 256 bytes,
// byte 4k + i = byte i of word k) by a 256 x 256-byte B matrix whose row
// 64 l + j, K byte 4k + i holds byte l of 2^(8i) W'[j][k] mod q (W' a 64 x 64
// matrix in Montgomery form): column 64 l + j of the result is E_l[j], and
// sum_l 2^(8l) E_l[j] = sum_k W'[j][k] x_k (mod q).
#pragma once
#include <cuda.h>
#include <stdint.h>

#include "grid_async.cuh"
#include "grid_field.cuh"
#include "grid_tc.cuh"

namespace grid {
namespace tcx {

constexpr int ROWS = 128;  // rows per tile (MMA M)
constexpr int EPI_WARPS = 16;
constexpr int MMA_WARP = EPI_WARPS;       // issues the MMAs
constexpr int LOAD_WARP = EPI_WARPS + 1;  // bulk / TMA loads and stores, L2 prefetch
constexpr int THREADS = (EPI_WARPS + 2) * 32;
constexpr uint32_t BOX = ROWS * 128;      // 16 KB: 128 rows x 128 bytes
constexpr uint32_t TILE = 2 * BOX;        // 32 KB: a 128 x 256 byte tile
constexpr uint32_t WMAT = 2 * 256 * 128;  // 64 KB: one transform's B matrix (256 x 256 B)

struct TcConsts {
  uint32_t q, qinv;
};

// cuTensorMapEncodeTiled, looked up once through the runtime (ntt_tc.cu); null
// if the driver does not provide it.
using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                 const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                 const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                 CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiled encoder();

// Byte offset of (row, 16-byte chunk c of K bytes 128h..128h+127) in a
// 128-byte-swizzled tile.
__host__ __device__ constexpr uint32_t sw128(uint32_t row, uint32_t h, uint32_t c,
                                             uint32_t box_bytes) {
  return h * box_bytes + (row >> 3) * 1024 + (row & 7) * 128 + ((c ^ (row & 7)) << 4);
}

// K-major, 128-byte swizzle, 8-row groups 1024 bytes apart.
__device__ __forceinline__ uint64_t desc_sw128(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | (1ull << 16) | ((uint64_t)(1024 >> 4) << 32) |
         (1ull << 46) | (2ull << 61);
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

// Whole warp: lane l receives 16 consecutive columns of tensor-memory lane
// (taddr.lane + l).
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
      "%12, %13, %14, %15}, [%16];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
                 "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]),
                 "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
               : "r"(taddr) : "memory");
}

// The four E_l blocks (64 columns apart) of 16 columns from taddr: loads
// issued, not waited for.
__device__ __forceinline__ void tmem_ld_planes(uint32_t taddr, uint32_t (&e)[4][16]) {
#pragma unroll
  for (int l = 0; l < 4; ++l) tmem_ld16(taddr + 64 * l, e[l]);
}

// Wait for this thread's tensor-memory loads, naming every loaded register so
// that no use is scheduled above the wait.
__device__ __forceinline__ void tmem_wait_planes(uint32_t (&e)[4][16]) {
  asm volatile("tcgen05.wait::ld.sync.aligned;"
               :
                 "+r"(e[0][0]), "+r"(e[0][1]), "+r"(e[0][2]), "+r"(e[0][3]), "+r"(e[0][4]), "+r"(e[0][5]), "+r"(e[0][6]), "+r"(e[0][7]),
                 "+r"(e[0][8]), "+r"(e[0][9]), "+r"(e[0][10]), "+r"(e[0][11]), "+r"(e[0][12]), "+r"(e[0][13]), "+r"(e[0][14]), "+r"(e[0][15]),
                 "+r"(e[1][0]), "+r"(e[1][1]), "+r"(e[1][2]), "+r"(e[1][3]), "+r"(e[1][4]), "+r"(e[1][5]), "+r"(e[1][6]), "+r"(e[1][7]),
                 "+r"(e[1][8]), "+r"(e[1][9]), "+r"(e[1][10]), "+r"(e[1][11]), "+r"(e[1][12]), "+r"(e[1][13]), "+r"(e[1][14]), "+r"(e[1][15]),
                 "+r"(e[2][0]), "+r"(e[2][1]), "+r"(e[2][2]), "+r"(e[2][3]), "+r"(e[2][4]), "+r"(e[2][5]), "+r"(e[2][6]), "+r"(e[2][7]),
                 "+r"(e[2][8]), "+r"(e[2][9]), "+r"(e[2][10]), "+r"(e[2][11]), "+r"(e[2][12]), "+r"(e[2][13]), "+r"(e[2][14]), "+r"(e[2][15]),
                 "+r"(e[3][0]), "+r"(e[3][1]), "+r"(e[3][2]), "+r"(e[3][3]), "+r"(e[3][4]), "+r"(e[3][5]), "+r"(e[3][6]), "+r"(e[3][7]),
                 "+r"(e[3][8]), "+r"(e[3][9]), "+r"(e[3][10]), "+r"(e[3][11]), "+r"(e[3][12]), "+r"(e[3][13]), "+r"(e[3][14]), "+r"(e[3][15])
               :
               : "memory");
}

// 16 canonical words from loaded planes: sum_l 2^(8l) E_l, one reduction.
__device__ __forceinline__ void combine16(const uint32_t (&e)[4][16], const TcConsts& k,
                                          uint32_t* out) {
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    uint64_t v = mad_wide(e[1][j], 256u, (uint64_t)e[0][j]);
    v = mad_wide(e[2][j], 65536u, v);
    v = mad_wide(e[3][j], 16777216u, v);
    out[j] = redc64(v, k.q, k.qinv);
  }
}

// 16 reduced results of this thread's row: columns col0 .. col0 + 15 of the
// four E_l blocks (64 columns apart) starting at taddr; one tensor-memory
// round trip of 16 columns x 4 blocks. after_load() runs once the loads have
// landed in registers, before the arithmetic (the columns may be reused from
// then on).
template <typename AfterLoad>
__device__ __forceinline__ void reduce16(uint32_t taddr, const TcConsts& k, uint32_t* out,
                                         AfterLoad&& after_load) {
  uint32_t e[4][16];
  tmem_ld_planes(taddr, e);
  tmem_wait_planes(e);
  after_load();
  combine16(e, k, out);
}

__device__ __forceinline__ void reduce16(uint32_t taddr, const TcConsts& k, uint32_t* out) {
  reduce16(taddr, k, out, [] {});
}

// One transform of a 128-row tile (A at `a`, B at `w`) into 256 columns.
__device__ __forceinline__ void issue_transform(uint32_t dcol, uint32_t a, uint32_t w) {
#pragma unroll
  for (int h = 0; h < 2; ++h)
#pragma unroll
    for (int s = 0; s < 4; ++s)
      tc::mma_u8(dcol, desc_sw128(a + h * BOX + 32 * s), desc_sw128(w + h * (WMAT / 2) + 32 * s),
                 tc::idesc_u8(ROWS, 256), (h | s) != 0);
}

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, int x, int y,
                                            uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3}], [%4];" ::"r"(dst),
      "l"(map), "r"(x), "r"(y), "r"(bar)
      : "memory");
}

__device__ __forceinline__ void tma_load_3d(uint32_t dst, const CUtensorMap* map, int x, int y,
                                            int z, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(dst),
      "l"(map), "r"(x), "r"(y), "r"(z), "r"(bar)
      : "memory");
}

__device__ __forceinline__ void tma_store_2d(const CUtensorMap* map, int x, int y, uint32_t src) {
  asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.tile.bulk_group [%0, {%1, %2}], [%3];" ::"l"(
                   map),
               "r"(x), "r"(y), "r"(src)
               : "memory");
}

// Contiguous global bytes -> L2 (no shared memory, no completion tracking).
__device__ __forceinline__ void prefetch_l2(const void* src, uint32_t bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool warp_wait(uint64_t* bar, uint32_t parity, int* err) {
  const bool ok = mbar_wait_sleep(bar, parity, err);
  return __all_sync(0xffffffffu, ok);
}

// The epilogue's waits on MMA results are on the critical path: poll
// without a suspend hint.
__device__ __forceinline__ bool warp_wait_fast(uint64_t* bar, uint32_t parity, int* err) {
  const bool ok = mbar_wait(bar, parity, err);
  return __all_sync(0xffffffffu, ok);
}

}  // namespace tcx
}  // namespace grid
