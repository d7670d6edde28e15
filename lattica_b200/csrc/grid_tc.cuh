// Inline-PTX wrappers for the sm_100a fifth-generation tensor cores
// (tcgen05): tensor-memory allocation, shared-memory matrix descriptors,
// unsigned 8-bit integer MMAs with 32-bit accumulators in tensor memory,
// completion through an mbarrier, and tensor-memory loads.
//
// Operand layout used throughout ("K-major, no swizzle"): a matrix of R rows
// by K bytes is stored as 8-row x 16-byte core matrices (128 contiguous
// bytes, row r of the core matrix at offset 16 r). The core matrix holding
// rows 8g..8g+7 and bytes 16c..16c+15 sits at g * SBO + c * LBO. One MMA
// consumes K = 32 bytes (two core matrices along K).
#pragma once
#include <stdint.h>

#include "grid_async.cuh"

namespace grid {
namespace tc {

// Byte offset of (row, 16-byte chunk) in the K-major no-swizzle layout.
__host__ __device__ constexpr uint32_t core_offset(uint32_t row, uint32_t chunk, uint32_t lbo,
                                                   uint32_t sbo) {
  return (row >> 3) * sbo + chunk * lbo + (row & 7u) * 16u;
}

// Shared-memory matrix descriptor: start address, leading (K) and stride
// (8-row) byte offsets, all in 16-byte units; descriptor version 1 (bits
// 46-47), no swizzle (bits 61-63 = 0), base offset 0.
__host__ __device__ constexpr uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor, kind::i8: unsigned 8-bit A and B (format 0), both
// K-major, signed 32-bit accumulator (format 2, bits 4-5), N / 8 at bits
// 17-22, M / 16 at bits 24-28.
__host__ __device__ constexpr uint32_t idesc_u8(uint32_t m, uint32_t n) {
  return (2u << 4) | ((n >> 3) << 17) | ((m >> 4) << 24);
}

// Tensor-memory address: lane in bits 16-31, column in bits 0-15.
__host__ __device__ constexpr uint32_t tmem_addr(uint32_t base, uint32_t lane, uint32_t col) {
  return base + (lane << 16) + col;
}

// Whole warp: allocate `ncols` columns (power of two >= 32); the base address
// is written to shared memory at dst.
__device__ __forceinline__ void tmem_alloc(uint32_t* dst, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                   smem_addr(dst)),
               "r"(ncols)
               : "memory");
}

__device__ __forceinline__ void tmem_relinquish() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

// Whole warp (the allocating one).
__device__ __forceinline__ void tmem_dealloc(uint32_t base, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(base), "r"(ncols)
               : "memory");
}

__device__ __forceinline__ void fence_before_sync() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}

__device__ __forceinline__ void fence_after_sync() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// Generic-proxy shared-memory writes -> visible to the tensor core's reads.
__device__ __forceinline__ void fence_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// One thread: D[tmem] (+)= A * B^T, M = 128 rows, N columns, K = 32 bytes.
__device__ __forceinline__ void mma_u8(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc,
                                       uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}

// One thread: arrive once on `bar` when every MMA it issued so far is done.
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_addr(bar))
               : "memory");
}

// Whole warp: lane l of the warp receives 4 consecutive columns of TMEM lane
// (taddr.lane + l). The warp may only touch lanes 32 * (warp % 4) .. + 31.
__device__ __forceinline__ void tmem_ld4(uint32_t taddr, uint32_t (&r)[4]) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0, %1, %2, %3}, [%4];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(taddr)
               : "memory");
}

// Whole warp: lane l of the warp receives 8 consecutive columns of TMEM lane
// (taddr.lane + l). The warp may only touch lanes 32 * (warp % 4) .. + 31.
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, uint32_t (&r)[8]) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
                 "=r"(r[6]), "=r"(r[7])
               : "r"(taddr)
               : "memory");
}

__device__ __forceinline__ void tmem_ld_wait32(uint32_t (&r)[4][8]) {
  asm volatile("tcgen05.wait::ld.sync.aligned;"
               : "+r"(r[0][0]), "+r"(r[0][1]), "+r"(r[0][2]), "+r"(r[0][3]), "+r"(r[0][4]), "+r"(r[0][5]), "+r"(r[0][6]), "+r"(r[0][7]),
                 "+r"(r[1][0]), "+r"(r[1][1]), "+r"(r[1][2]), "+r"(r[1][3]), "+r"(r[1][4]), "+r"(r[1][5]), "+r"(r[1][6]), "+r"(r[1][7]),
                 "+r"(r[2][0]), "+r"(r[2][1]), "+r"(r[2][2]), "+r"(r[2][3]), "+r"(r[2][4]), "+r"(r[2][5]), "+r"(r[2][6]), "+r"(r[2][7]),
                 "+r"(r[3][0]), "+r"(r[3][1]), "+r"(r[3][2]), "+r"(r[3][3]), "+r"(r[3][4]), "+r"(r[3][5]), "+r"(r[3][6]), "+r"(r[3][7])
               :
               : "memory");
}

__device__ __forceinline__ void tmem_ld_wait() {
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// Wait for this thread's tensor-memory loads, naming the 16 registers they
// fill so that no use of them can be scheduled above the wait.
__device__ __forceinline__ void tmem_ld_wait(uint32_t (&r)[4][4]) {
  asm volatile("tcgen05.wait::ld.sync.aligned;"
               : "+r"(r[0][0]), "+r"(r[0][1]), "+r"(r[0][2]), "+r"(r[0][3]), "+r"(r[1][0]),
                 "+r"(r[1][1]), "+r"(r[1][2]), "+r"(r[1][3]), "+r"(r[2][0]), "+r"(r[2][1]),
                 "+r"(r[2][2]), "+r"(r[2][3]), "+r"(r[3][0]), "+r"(r[3][1]), "+r"(r[3][2]),
                 "+r"(r[3][3])
               :
               : "memory");
}

}  // namespace tc
}  // namespace grid
