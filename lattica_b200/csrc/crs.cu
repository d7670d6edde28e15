// Uniform ring elements on the device, in the order and with the values of
// the reference's seeded commitment-key expansion.
//
// Reference path replaced: CommitKey::from_seed / generate_from_params /
// sample_uniform_mat (labrador/src/crs.rs:136-198, 308-326): the matrices A, B,
// C, D are ring elements drawn one after another from ChaCha20Rng(seed)
// (rand_chacha 0.10.0, Cargo.lock), every coefficient by PrimeField::rand
// (algebra/src/arith/prime.rs:730-743): a u64 sample s is accepted when
// s <= u64::MAX - ((u64::MAX % q + 1) % q) and maps to from_u64(s % q).
// The generator's u64 stream is the ChaCha20 keystream (64-bit block counter
// from 0, stream 0) read as consecutive little-endian word pairs, low word
// first (rand_core 0.10.1 block RNG).
//
// The sequence is sequential only through its rare rejections (probability
// below 2^-32 per sample for q < 2^32), so the device runs it as a compaction:
// every candidate is generated in parallel (one ChaCha20 block = 8 candidates
// per thread, 2048 per 256-thread segment); pass 1 counts each segment's
// rejections, pass 2 scans them, pass 3 regenerates the candidates and writes
// accepted sample k to position k - (rejections before k). Candidates beyond
// the requested count are a margin for rejections; running out of it is
// reported (GRID_ERR_SAMPLE_EXHAUSTED through the plan's error word).
#include <cuda_runtime.h>

#include "grid_async.cuh"
#include "grid_chacha.cuh"
#include "grid_field.cuh"
#include "grid_internal.h"

namespace grid {
namespace {

constexpr int kSegThreads = 256;
constexpr int kSegCands = kSegThreads * 8;  // candidates per segment
constexpr int kCrsFmaAdds = 0;              // keystream additions on the FMA pipe: 4 measured no faster

__device__ __forceinline__ void rng_block(const chacha::ChachaKey& key, unsigned long long blk,
                                          uint32_t (&w)[16]) {
  chacha::chacha20_block<kCrsFmaAdds>(key, (uint32_t)blk, (uint32_t)(blk >> 32), w);
}

__device__ __forceinline__ unsigned long long cand(const uint32_t (&w)[16], int c) {
  return (unsigned long long)w[2 * c] | ((unsigned long long)w[2 * c + 1] << 32);
}

// Exclusive prefix sum of v over the 256 threads of the CTA; *total gets the sum.
__device__ __forceinline__ unsigned cta_exclusive_scan(unsigned v, unsigned* total) {
  __shared__ unsigned warp_sums[kSegThreads / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  unsigned x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_sums[warp] = x;
  __syncthreads();
  unsigned before = 0, all = 0;
#pragma unroll
  for (int i = 0; i < kSegThreads / 32; ++i) {
    if (i < warp) before += warp_sums[i];
    all += warp_sums[i];
  }
  __syncthreads();  // warp_sums is reused by the next call
  *total = all;
  return before + x - v;
}

__global__ void __launch_bounds__(kSegThreads) crs_count_kernel(chacha::ChachaKey key,
                                                                unsigned long long nseg,
                                                                unsigned long long upper,
                                                                unsigned* __restrict__ seg_rej) {
  for (unsigned long long seg = blockIdx.x; seg < nseg; seg += gridDim.x) {
    uint32_t w[16];
    rng_block(key, seg * kSegThreads + threadIdx.x, w);
    unsigned rej = 0;
#pragma unroll
    for (int c = 0; c < 8; ++c) rej += cand(w, c) > upper ? 1u : 0u;
    unsigned total;
    cta_exclusive_scan(rej, &total);
    if (threadIdx.x == 0) seg_rej[seg] = total;
  }
}

// One CTA: seg_off[s] = rejections in segments before s; short = whether the
// accepted candidates fall below `count`.
__global__ void __launch_bounds__(kSegThreads) crs_scan_kernel(const unsigned* __restrict__ seg_rej,
                                                               unsigned long long nseg,
                                                               unsigned long long count,
                                                               unsigned long long* __restrict__ seg_off,
                                                               int* __restrict__ err) {
  unsigned long long carry = 0;
  for (unsigned long long base = 0; base < nseg; base += kSegThreads) {
    const unsigned long long i = base + threadIdx.x;
    const unsigned v = i < nseg ? seg_rej[i] : 0u;
    unsigned total;
    const unsigned ex = cta_exclusive_scan(v, &total);
    if (i < nseg) seg_off[i] = carry + ex;
    carry += total;
  }
  if (threadIdx.x == 0 && nseg * kSegCands - carry < count) atomicExch(err, GRID_DEV_SAMPLE_SHORT);
}

__global__ void __launch_bounds__(kSegThreads) crs_write_kernel(
    chacha::ChachaKey key, unsigned long long nseg, unsigned long long upper,
    const unsigned long long* __restrict__ seg_off, unsigned long long count,
    uint32_t* __restrict__ out, FieldParams f, uint32_t r3) {
  for (unsigned long long seg = blockIdx.x; seg < nseg; seg += gridDim.x) {
    const unsigned long long blk = seg * kSegThreads + threadIdx.x;
    uint32_t w[16];
    rng_block(key, blk, w);
    unsigned rej = 0;
#pragma unroll
    for (int c = 0; c < 8; ++c) rej += cand(w, c) > upper ? 1u : 0u;
    unsigned total;
    unsigned long long before = seg_off[seg] + cta_exclusive_scan(rej, &total);
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      const unsigned long long s = cand(w, c);
      if (s > upper) {
        ++before;
        continue;
      }
      const unsigned long long dest = blk * 8 + c - before;
      if (dest < count) {
        // from_u64(s % q) in Montgomery form: s * 2^32 mod q
        //   = hi * 2^64 + lo * 2^32 = mont(hi, 2^96 mod q) + mont(lo, 2^64 mod q)
        const uint32_t hi = (uint32_t)(s >> 32), lo = (uint32_t)s;
        out[dest] = add_mod(mont_mul(hi, r3, f.q, f.qinv), mont_mul(lo, f.r2, f.q, f.qinv), f.q);
      }
    }
  }
}

struct SampleGeometry {
  unsigned long long upper, nseg;
};

SampleGeometry sample_geometry(uint32_t q, unsigned long long count, unsigned long long accept_max) {
  SampleGeometry g;
  const unsigned long long reject = (~0ull % q + 1ull) % q;
  g.upper = accept_max ? accept_max : ~0ull - reject;
  // one spare segment covers the reference threshold's rejections (below 2^-32
  // per sample); a caller-chosen threshold gets a quarter more besides
  const unsigned long long cands = count + kSegCands + (accept_max ? count / 4 : 0);
  g.nseg = (cands + kSegCands - 1) / kSegCands;
  return g;
}

}  // namespace

size_t sample_uniform_workspace_bytes(uint32_t q, unsigned long long count,
                                      unsigned long long accept_max) {
  const SampleGeometry g = sample_geometry(q, count, accept_max);
  return ((g.nseg * 4 + 255) / 256) * 256 + g.nseg * 8;
}

int launch_sample_uniform(const grid_gpu_plan* p, const uint8_t seed[32], unsigned long long count,
                          unsigned long long accept_max, uint32_t* out, void* ws, size_t ws_bytes,
                          cudaStream_t s) {
  if (count == 0) return GRID_OK;
  const SampleGeometry g = sample_geometry(p->f.q, count, accept_max);
  if (ws_bytes < sample_uniform_workspace_bytes(p->f.q, count, accept_max))
    return GRID_ERR_INVALID_PARAMETERS;
  unsigned* seg_rej = static_cast<unsigned*>(ws);
  unsigned long long* seg_off = reinterpret_cast<unsigned long long*>(
      static_cast<char*>(ws) + ((g.nseg * 4 + 255) / 256) * 256);
  chacha::ChachaKey key;
  for (int i = 0; i < 8; ++i)
    key.k[i] = (uint32_t)seed[4 * i] | ((uint32_t)seed[4 * i + 1] << 8) |
               ((uint32_t)seed[4 * i + 2] << 16) | ((uint32_t)seed[4 * i + 3] << 24);
  const uint32_t r3 = (uint32_t)(((unsigned __int128)1 << 96) % p->f.q);
  unsigned long long grid = (unsigned long long)p->num_sms * 8;
  if (grid > g.nseg) grid = g.nseg;
  crs_count_kernel<<<(unsigned)grid, kSegThreads, 0, s>>>(key, g.nseg, g.upper, seg_rej);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_status(e);
  crs_scan_kernel<<<1, kSegThreads, 0, s>>>(seg_rej, g.nseg, count, seg_off, p->d_err);
  if ((e = cudaGetLastError()) != cudaSuccess) return cuda_status(e);
  crs_write_kernel<<<(unsigned)grid, kSegThreads, 0, s>>>(key, g.nseg, g.upper, seg_off, count,
                                                          out, p->f, r3);
  return cuda_status(cudaGetLastError());
}

}  // namespace grid
