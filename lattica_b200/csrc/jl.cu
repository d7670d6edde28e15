// Johnson-Lindenstrauss projection of the LaBRADOR prover on the GPU.
//
// Reference path replaced: JLMatrix::project_and_extract_jl_rows /
// project_and_extract_seq (labrador/src/jl.rs:267-303, 388-508). Part i of the
// witness uses the IETF ChaCha20 keystream (RFC 8439; the reference uses the
// chacha20 0.10 crate) with key = seed, nonce = (u32 i, little endian) || 0^8,
// block counter from 0. Column `col` consumes packed_len = ceil(rows/4) bytes
// at keystream offset col*packed_len; row r reads bits 2*(r%4) of byte r/4:
// 00 -> +1, 01 -> -1, 1x -> 0. p[row] = sum over parts and columns of
// entry * coeff (mod q), accumulated on Montgomery words (the map to
// Montgomery form is additive, so this is the reference's field sum).
//
// The keystream is regenerated on the fly (the reference materialises the
// whole [rows][parts][d][n] i8 matrix, 2 GiB at the LaBRADOR round size);
// the i8 extraction is a separate, optional kernel.
//
// Projection kernel: a warp takes 32 consecutive columns of one part; lane l
// computes the keystream bytes of column c0 + l into shared memory, then owns
// rows 8l .. 8l+7 and sweeps the 32 columns, adding the coefficient to a
// 64-bit "plus" or "minus" accumulator per row (exact while one warp sees
// fewer than 2^32 columns of 32-bit words). Per-lane totals are folded mod q and added to
// 64-bit global row sums with atomics; a final kernel reduces them mod q.
#include <cuda_runtime.h>

#include <algorithm>

#include "grid_async.cuh"
#include "grid_field.cuh"
#include "grid_internal.h"
#include "grid_chacha.cuh"
#include "grid_tc.cuh"

namespace grid {
namespace {

using chacha::ChachaKey;
using chacha::chacha20_block;

constexpr int kJlWarps = 8;
constexpr int kJlThreads = kJlWarps * 32;

// Keystream bytes [off, off + 64) of stream (key, nonce0) as 16 words
// (unused tail bytes are whatever the next block holds; callers mask rows).
__device__ __forceinline__ void keystream64(const ChachaKey& key, uint32_t nonce0, uint64_t off,
                                            uint32_t (&w)[16]) {
  const uint32_t blk = (uint32_t)(off >> 6);
  const uint32_t sh = (uint32_t)(off & 63);
  chacha20_block(key, blk, nonce0, w);
  if (sh != 0) {
    uint32_t nx[16];
    chacha20_block(key, blk + 1, nonce0, nx);
    // byte-shift the 128-byte window (w ++ nx) left by sh bytes
    const uint32_t ws = sh >> 2, bs = (sh & 3) * 8;
    uint32_t r[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) {
      const uint32_t j = i + ws;
      const uint32_t lo = j < 16 ? w[j] : nx[j - 16];
      const uint32_t j2 = j + 1;
      const uint32_t hi = j2 < 16 ? w[j2] : (j2 < 32 ? nx[j2 - 16] : 0u);
      r[i] = bs ? __funnelshift_r(lo, hi, bs) : lo;
    }
#pragma unroll
    for (int i = 0; i < 16; ++i) w[i] = r[i];
  }
}

template <bool kWholeBlocks>
__global__ void __launch_bounds__(kJlThreads) jl_project_kernel(
    const uint32_t* __restrict__ parts, unsigned long long cols, int num_parts, int rows,
    int packed_len, ChachaKey key, unsigned long long* __restrict__ gsum_pos,
    unsigned long long* __restrict__ gsum_neg, uint32_t q) {
  __shared__ uint32_t ks[kJlWarps][32][17];
  __shared__ uint32_t xs[kJlWarps][32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const unsigned long long chunks_per_part = (cols + 31) / 32;
  const unsigned long long total = chunks_per_part * (unsigned long long)num_parts;
  const unsigned long long stride = (unsigned long long)gridDim.x * kJlWarps;
  unsigned long long pos[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  unsigned long long neg[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  const int word = lane >> 1, shift = (lane & 1) * 16;

  for (unsigned long long ch = (unsigned long long)blockIdx.x * kJlWarps + warp; ch < total;
       ch += stride) {
    const uint32_t part = (uint32_t)(ch / chunks_per_part);
    const unsigned long long c = (ch % chunks_per_part) * 32 + lane;
    uint32_t w[16];
    uint32_t x = 0;
    if (c < cols) {
      if constexpr (kWholeBlocks)
        chacha20_block(key, (uint32_t)c, part, w);  // 256 rows: column c is block c
      else
        keystream64(key, part, c * (unsigned long long)packed_len, w);
      x = parts[(unsigned long long)part * cols + c];
    } else {
#pragma unroll
      for (int i = 0; i < 16; ++i) w[i] = 0xFFFFFFFFu;  // code 11 -> 0
    }
    __syncwarp();
#pragma unroll
    for (int i = 0; i < 16; ++i) ks[warp][lane][i] = w[i];
    xs[warp][lane] = x;
    __syncwarp();
#pragma unroll 4
    for (int cc = 0; cc < 32; ++cc) {
      const uint32_t h = ks[warp][cc][word] >> shift;
      const uint32_t xc = xs[warp][cc];
      const uint32_t lo = h & 0x5555u, hi = (h >> 1) & 0x5555u;
      const uint32_t plus = ~(lo | hi) & 0x5555u;  // code 00
      const uint32_t minus = lo & ~hi;             // code 01
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        pos[k] += (unsigned long long)(xc & (0u - ((plus >> (2 * k)) & 1u)));
        neg[k] += (unsigned long long)(xc & (0u - ((minus >> (2 * k)) & 1u)));
      }
    }
  }
  // Fold to residues and publish. Rows beyond `rows` only saw code 11.
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const int row = lane * 8 + k;
    if (row < rows && (pos[k] | neg[k])) {
      atomicAdd(&gsum_pos[row], pos[k] % q);
      atomicAdd(&gsum_neg[row], neg[k] % q);
    }
  }
}

__global__ void jl_finish_kernel(const unsigned long long* __restrict__ gsum_pos,
                                 const unsigned long long* __restrict__ gsum_neg, uint32_t* p_out,
                                 int rows, uint32_t q) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r < rows) {
    const uint32_t a = (uint32_t)(gsum_pos[r] % q), b = (uint32_t)(gsum_neg[r] % q);
    p_out[r] = sub_mod(a, b, q);
  }
}

// ---------------------------------------------------------------------------
// Tensor-core projection. A CTA takes chunks of 256 columns of one part:
// thread t computes the keystream of column c0 + t and writes its 256
// entries shifted by one, M' = M + 1 in {0, 1, 2}, as column t of an
// MN-major u8 A tile (rows contiguous), and the column's word as a
// zero-padded 16-byte column of an MN-major u8 B tile (bytes = N). One u8
// MMA per (128-row half, 32-column step) accumulates
// D'[r][i] = sum_c M'[r][c] * byte_i(x_c) in tensor memory across all of the
// CTA's chunks; then p_r = sum_i 2^(8i) (D'[r][i] - sum_c byte_i(x_c)) mod q.
// D' < 2 * 255 * (columns per CTA) stays below 2^31 (the host bounds the
// columns per CTA).
// ---------------------------------------------------------------------------
constexpr int kTcThreads = 256;
constexpr int kTcCols = 256;                      // columns (K) per chunk
// Keystream additions issued on the FMA pipe per quarter round (chacha20_block).
// Measured: the projection 0.552 / 0.532 / 0.524 ms with 0 / 2 / 4, the
// evaluations (whose FMA pipe is busier) 0.795 / 0.828 / 0.829 ms.
constexpr int kTcFmaAdds = 4;
constexpr int kEvFmaAdds = 0;
constexpr uint32_t kTcA = 256u * kTcCols;         // A tile: 256 rows x 256 columns
constexpr uint32_t kTcB = 16u * kTcCols;          // B tile: 16 bytes x 256 columns
constexpr uint32_t kTcSmem = kTcA + kTcB + 1024 + 64 + 1024;  // + LUT, barrier, slack
constexpr unsigned long long kTcMaxColsPerCta = 1ull << 22;    // 2 * 255 * 2^22 < 2^31

// row m, column k of the A tile: 16-row x 8-column core matrices
__device__ __forceinline__ uint32_t jl_a_off(uint32_t m, uint32_t k) {
  return (k >> 3) * 2048u + (m >> 4) * 128u + (k & 7u) * 16u + (m & 15u);
}

// M' = M + 1 for the 4 codes of one keystream byte: 00 -> 2, 01 -> 0, 1x -> 1.
__device__ __forceinline__ uint32_t shifted_entries_of_byte(uint32_t byte) {
  uint32_t out = 0;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const uint32_t c = (byte >> (2 * i)) & 3u;
    const uint32_t v = c == 0 ? 2u : (c == 1 ? 0u : 1u);
    out |= v << (8 * i);
  }
  return out;
}

// kFlat (whole blocks, d % 8 == 0, n % 32 == 0): the kernel also writes the
// int8 entries flat[row][part][k][j] (col = j d + k) from the words it builds
// for the A tile, so the keystream is generated once. A chunk is then 32
// consecutive polynomials x 8 coefficient indices: warp w takes coefficient
// 8 kg + w and lane l polynomial 32 jg + l. For each keystream byte, the four
// lanes of a quad swap bytes (a 4 x 4 transpose: two shuffles, two byte
// permutes) so that lane 4 g + r holds row 4 b + r of polynomials 4 g .. 4 g + 3,
// and the warp's stores fill whole 32-byte sectors of four rows.
template <bool kWholeBlocks, bool kFlat = false>
__global__ void __launch_bounds__(kTcThreads) jl_tc_kernel(
    const uint32_t* __restrict__ parts, unsigned long long cols, int rows, int packed_len,
    ChachaKey key, unsigned long long nchunks, unsigned long long per_part, int d,
    unsigned long long plane, int8_t* __restrict__ flat,
    unsigned long long* __restrict__ gsum_pos, uint32_t q, int* __restrict__ err) {
  extern __shared__ __align__(1024) unsigned char sm_raw[];
  const uint32_t raw = smem_addr(sm_raw);
  unsigned char* sm = sm_raw + (((raw + 1023u) & ~1023u) - raw);
  const uint32_t s0 = smem_addr(sm);
  uint32_t* lut = reinterpret_cast<uint32_t*>(sm + kTcA + kTcB);
  uint64_t* bar = reinterpret_cast<uint64_t*>(sm + kTcA + kTcB + 1024);
  uint32_t* taddr_slot = reinterpret_cast<uint32_t*>(bar + 1);
  uint32_t* colsum = taddr_slot + 2;  // [4]
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  for (int i = tid; i < 256; i += kTcThreads) lut[i] = shifted_entries_of_byte(i);
  if (tid < 4) colsum[tid] = 0;
  if (warp == 0) {
    tc::tmem_alloc(taddr_slot, 32);
    tc::tmem_relinquish();
  }
  if (tid == 0) {
    mbar_init(bar, 1);
    fence_mbar_init();
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tbase = *taddr_slot;
  // kind::i8, u8 x u8 -> s32, A and B MN-major, M = 128, N = 16
  const uint32_t idesc = tc::idesc_u8(128, 16) | (1u << 15) | (1u << 16);

  const unsigned long long npoly = cols / (unsigned long long)d;
  // byte selectors of the quad transpose (step 1: lanes l, l ^ 1; step 2: l, l ^ 2)
  const uint32_t sel1 = (lane & 1) ? 0x3715u : 0x6240u;
  const uint32_t sel2 = (lane & 2) ? 0x3276u : 0x5410u;
  uint32_t bsum[4] = {0, 0, 0, 0};
  bool ok = true;
  uint32_t it = 0;
  for (unsigned long long ch = blockIdx.x; ch < nchunks; ch += gridDim.x, ++it) {
    const uint32_t part = (uint32_t)(ch / per_part);
    const unsigned long long ci = ch % per_part;
    unsigned long long c, jj = 0;
    uint32_t kk = 0;
    if constexpr (kFlat) {
      const unsigned long long kgroups = (unsigned long long)d / 8;
      jj = (ci / kgroups) * 32 + lane;
      kk = (uint32_t)(ci % kgroups) * 8 + warp;
      c = jj * d + kk;
    } else {
      c = ci * kTcCols + tid;
    }
    uint32_t w[16];
    uint32_t x = 0;
    if (c < cols) {
      if constexpr (kWholeBlocks)
        chacha20_block<kTcFmaAdds>(key, (uint32_t)c, part, w);
      else
        keystream64(key, part, c * (unsigned long long)packed_len, w);
      x = parts[(unsigned long long)part * cols + c];
    } else {
#pragma unroll
      for (int i = 0; i < 16; ++i) w[i] = 0xFFFFFFFFu;  // padding column: x = 0
    }
    // the previous chunk's MMAs must be done reading the tiles
    if (it > 0) ok = __syncthreads_and(mbar_wait(bar, (it - 1) & 1, err));
    if (!ok) break;
    // kFlat: this lane's row 4 b + (lane & 3) of polynomials jj - (lane & 3) .. + 3,
    // keystream byte b = 0, 1, ...: one pointer advanced by 4 rows per byte
    int8_t* rowp = nullptr;
    if constexpr (kFlat)
      rowp = flat + (unsigned long long)(lane & 3) * plane +
             ((unsigned long long)part * d + kk) * npoly + (jj - (lane & 3));
    const unsigned long long step4 = 4 * plane;
#pragma unroll
    for (int g = 0; g < 16; ++g) {
      const uint32_t v[4] = {lut[w[g] & 0xFFu], lut[(w[g] >> 8) & 0xFFu],
                             lut[(w[g] >> 16) & 0xFFu], lut[w[g] >> 24]};
      *reinterpret_cast<uint4*>(sm + jl_a_off(16 * g, tid)) = make_uint4(v[0], v[1], v[2], v[3]);
      if constexpr (kFlat) {
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          const uint32_t m = (v[i] + 0x7F7F7F7Fu) ^ 0x80808080u;  // M = M' - 1 per byte
          const uint32_t a = __byte_perm(m, __shfl_xor_sync(0xffffffffu, m, 1), sel1);
          const uint32_t o = __byte_perm(a, __shfl_xor_sync(0xffffffffu, a, 2), sel2);
          if (4 * (4 * g + i) + (lane & 3) < rows) *reinterpret_cast<uint32_t*>(rowp) = o;
          rowp += step4;
        }
      }
    }
    *reinterpret_cast<uint4*>(sm + kTcA + (tid >> 3) * 128 + (tid & 7) * 16) =
        make_uint4(x, 0, 0, 0);
#pragma unroll
    for (int i = 0; i < 4; ++i) bsum[i] += (x >> (8 * i)) & 0xFFu;
    tc::fence_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    if (tid == 0) {
      tc::fence_after_sync();
#pragma unroll
      for (int h = 0; h < 2; ++h)
#pragma unroll
        for (int ks = 0; ks < kTcCols / 32; ++ks)
          tc::mma_u8(tbase + 16 * h, tc::smem_desc(s0 + h * 1024 + ks * 8192, 2048, 128),
                     tc::smem_desc(s0 + kTcA + ks * 512, 128, 256), idesc,
                     (it | (uint32_t)ks) != 0);
      tc::mma_commit(bar);
    }
  }
  if (ok && it > 0) ok = mbar_wait(bar, (it - 1) & 1, err);
  ok = __syncthreads_and(ok);
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    uint32_t v = bsum[i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) atomicAdd(&colsum[i], v);
  }
  __syncthreads();
  tc::fence_after_sync();
  if (ok && it > 0 && warp < 4) {
    uint32_t d0[4], d1[4];
    tc::tmem_ld4(tc::tmem_addr(tbase, 32 * warp, 0), d0);
    tc::tmem_ld4(tc::tmem_addr(tbase, 32 * warp, 16), d1);
    tc::tmem_ld_wait();
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int row = 128 * h + 32 * warp + lane;
      const uint32_t* dv = h ? d1 : d0;
      long long v = 0;
#pragma unroll
      for (int i = 0; i < 4; ++i) v += ((long long)dv[i] - (long long)colsum[i]) << (8 * i);
      long long r = v % (long long)q;
      if (r < 0) r += q;
      if (row < rows) atomicAdd(&gsum_pos[row], (unsigned long long)r);
    }
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tbase, 32);
}

// Entry -> int8 table for one keystream byte: 4 rows, 2 bits each.
__device__ __forceinline__ uint32_t entries_of_byte(uint32_t byte) {
  uint32_t out = 0;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const uint32_t c = (byte >> (2 * i)) & 3u;
    const uint32_t v = c == 0 ? 0x01u : (c == 1 ? 0xFFu : 0x00u);
    out |= v << (8 * i);
  }
  return out;
}

// flat[row][part][k][j] (int8) for col = j*d + k. A warp handles one (part, k)
// and 128 consecutive j, 4 per lane, so each row store is a 4-byte word and
// a warp writes 128 contiguous bytes per row.
template <bool kWholeBlocks>
__global__ void __launch_bounds__(kJlThreads) jl_flat_kernel(unsigned long long cols, int d,
                                                             int num_parts, int rows,
                                                             int packed_len, ChachaKey key,
                                                             int8_t* __restrict__ flat) {
  __shared__ uint32_t lut[256];
  for (int i = threadIdx.x; i < 256; i += blockDim.x) lut[i] = entries_of_byte(i);
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const unsigned long long n = cols / d;
  const unsigned long long jchunks = (n + 127) / 128;
  const unsigned long long total = (unsigned long long)num_parts * d * jchunks;
  const unsigned long long plane = (unsigned long long)num_parts * cols;  // bytes per row
  const unsigned long long stride = (unsigned long long)gridDim.x * kJlWarps;
  const bool vec_ok = (n % 4) == 0;
  for (unsigned long long wk = (unsigned long long)blockIdx.x * kJlWarps + warp; wk < total;
       wk += stride) {
    const unsigned long long jc = wk % jchunks;
    const unsigned long long pk = wk / jchunks;  // part * d + k
    const uint32_t part = (uint32_t)(pk / d);
    const uint32_t k = (uint32_t)(pk % d);
    const unsigned long long j0 = jc * 128 + lane * 4;
    uint32_t w[4][16];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const unsigned long long j = j0 + u;
      if (j < n) {
        if constexpr (kWholeBlocks)
          chacha20_block(key, (uint32_t)(j * d + k), part, w[u]);
        else
          keystream64(key, part, (j * d + k) * (unsigned long long)packed_len, w[u]);
      } else {
#pragma unroll
        for (int i = 0; i < 16; ++i) w[u][i] = 0xFFFFFFFFu;
      }
    }
    int8_t* base = flat + pk * n + j0;
#pragma unroll
    for (int b = 0; b < 64; ++b) {
      if (b >= packed_len) break;
      uint32_t e[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) e[u] = lut[(w[u][b >> 2] >> ((b & 3) * 8)) & 0xFFu];
      // transpose 4 columns x 4 rows of bytes: out[r] = (e0.r, e1.r, e2.r, e3.r)
      const uint32_t t01l = __byte_perm(e[0], e[1], 0x5140);
      const uint32_t t23l = __byte_perm(e[2], e[3], 0x5140);
      const uint32_t t01h = __byte_perm(e[0], e[1], 0x7362);
      const uint32_t t23h = __byte_perm(e[2], e[3], 0x7362);
      uint32_t o[4];
      o[0] = __byte_perm(t01l, t23l, 0x5410);
      o[1] = __byte_perm(t01l, t23l, 0x7632);
      o[2] = __byte_perm(t01h, t23h, 0x5410);
      o[3] = __byte_perm(t01h, t23h, 0x7632);
#pragma unroll
      for (int r4 = 0; r4 < 4; ++r4) {
        const int row = b * 4 + r4;
        if (row >= rows) break;
        int8_t* dst = base + (unsigned long long)row * plane;
        if (vec_ok && j0 + 3 < n) {
          *reinterpret_cast<uint32_t*>(dst) = o[r4];
        } else {
          for (int u = 0; u < 4; ++u)
            if (j0 + u < n) dst[u] = (int8_t)((o[r4] >> (8 * u)) & 0xFFu);
        }
      }
    }
  }
}


// ---------------------------------------------------------------------------
// JL evaluations (aggregation side): evals[m] = sum_{i,j} conj(pi_{m,i,j}) s_{i,j}
// (jl_rows_flat_to_conjugated_polys + the jl_evals loop of prove_step,
// main_protocol/mod.rs:885-923, step_prover.rs:185-206), without the int8
// entries ever being stored. Coefficient t of conj(pi) * s is
// sum_u pi_u s'[u + t] with s' the negacyclic extension (s'[v] = -s[v - d] for
// v >= d), so coefficient t of evals[m] is the JL projection of the witness
// with every polynomial multiplied by X^-t. One keystream therefore serves all
// d = 64 coefficients: column (j, u) of the B tile holds the 64 words
// s'_j[u + t], t = 0 .. 63, as 256 bytes (N = 256), and D'[r][4t + i] =
// sum_c M'[r][c] byte_i(s'[u_c + t]) accumulates in all 512 tensor-memory
// columns (two 128-row halves). The M' = M + 1 correction
// S[t][i] = sum_c byte_i(s'[u_c + t]) comes from per-position byte sums of each
// coefficient and its negation: sum_{v >= t} P_i[v] + sum_{v < t} N_i[v].
// ---------------------------------------------------------------------------
constexpr uint32_t kEvB = 256u * kTcCols;                  // B tile: 256 bytes x 256 columns
// M' table in 32 bank-rotated copies (entry e of copy c at word 32 e + c; lane
// l reads copy l), so the 32 random lookups of a warp never share a bank
constexpr uint32_t kEvOffLut = kTcA + kEvB;
constexpr uint32_t kEvOffPoly = kEvOffLut + 32 * 1024;     // the chunk's 4 polys (1 KB)
constexpr uint32_t kEvOffSums = kEvOffPoly + 1024;         // P[64][4], N[64][4] (2 KB)
constexpr uint32_t kEvOffS = kEvOffSums + 2048;            // S[64][4] (1 KB)
constexpr uint32_t kEvOffBar = kEvOffS + 1024;
constexpr uint32_t kEvSmem = kEvOffBar + 64 + 1024;        // + alignment slack
constexpr int kEvD = 64, kEvRows = 256;

__global__ void __launch_bounds__(kTcThreads, 1) jl_eval_tc_kernel(
    const uint32_t* __restrict__ parts, unsigned long long cols, ChachaKey key,
    unsigned long long nchunks, unsigned long long* __restrict__ gsum, uint32_t q,
    int* __restrict__ err) {
  extern __shared__ __align__(1024) unsigned char sm_raw[];
  const uint32_t raw = smem_addr(sm_raw);
  unsigned char* sm = sm_raw + (((raw + 1023u) & ~1023u) - raw);
  const uint32_t s0 = smem_addr(sm);
  uint32_t* lut = reinterpret_cast<uint32_t*>(sm + kEvOffLut);
  uint32_t* poly = reinterpret_cast<uint32_t*>(sm + kEvOffPoly);
  uint32_t* sums = reinterpret_cast<uint32_t*>(sm + kEvOffSums);  // [0,256): P, [256,512): N
  uint32_t* corr = reinterpret_cast<uint32_t*>(sm + kEvOffS);
  uint64_t* bar = reinterpret_cast<uint64_t*>(sm + kEvOffBar);
  uint32_t* taddr_slot = reinterpret_cast<uint32_t*>(bar + 1);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  for (int i = tid; i < 256 * 32; i += kTcThreads) lut[i] = shifted_entries_of_byte(i >> 5);
  for (int i = tid; i < 512; i += kTcThreads) sums[i] = 0;
  if (warp == 0) {
    tc::tmem_alloc(taddr_slot, 512);
    tc::tmem_relinquish();
  }
  if (tid == 0) {
    mbar_init(bar, 1);
    fence_mbar_init();
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tbase = *taddr_slot;
  // kind::i8, u8 x u8 -> s32, A and B MN-major, M = 128, N = 256
  const uint32_t idesc = tc::idesc_u8(128, 256) | (1u << 15) | (1u << 16);

  const unsigned long long per_part = (cols + kTcCols - 1) / kTcCols;
  const uint32_t u = tid & (kEvD - 1);  // this thread's coefficient position in its poly
  uint32_t psum[4] = {0, 0, 0, 0}, nsum[4] = {0, 0, 0, 0};
  bool ok = true;
  uint32_t it = 0;
  for (unsigned long long ch = blockIdx.x; ch < nchunks; ch += gridDim.x, ++it) {
    const uint32_t part = (uint32_t)(ch / per_part);
    const unsigned long long c = (ch % per_part) * kTcCols + tid;
    uint32_t w[16];
    uint32_t x = 0;
    if (c < cols) {
      chacha20_block<kEvFmaAdds>(key, (uint32_t)c, part, w);  // 256 rows: column c is block c
      x = parts[(unsigned long long)part * cols + c];
    } else {
#pragma unroll
      for (int i = 0; i < 16; ++i) w[i] = 0xFFFFFFFFu;  // padding column: x = 0
    }
    const uint32_t xn = x == 0 ? 0u : q - x;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      psum[i] += (x >> (8 * i)) & 0xFFu;
      nsum[i] += (xn >> (8 * i)) & 0xFFu;
    }
    // the previous chunk's MMAs must be done reading the tiles
    if (it > 0) ok = __syncthreads_and(mbar_wait(bar, (it - 1) & 1, err));
    if (!ok) break;
    poly[tid] = x;
    const uint32_t* lt = lut + lane;
#pragma unroll
    for (int g = 0; g < 16; ++g)
      *reinterpret_cast<uint4*>(sm + jl_a_off(16 * g, tid)) =
          make_uint4(lt[(w[g] & 0xFFu) << 5], lt[((w[g] >> 8) & 0xFFu) << 5],
                     lt[((w[g] >> 16) & 0xFFu) << 5], lt[(w[g] >> 24) << 5]);
    __syncthreads();  // the chunk's polys are staged
    // B column tid: s'[u + t] for t = 0 .. 63, 16 bytes per group of 4 t
    const uint32_t* pw = poly + (tid & ~(kEvD - 1));
#pragma unroll
    for (int g = 0; g < 16; ++g) {
      uint32_t v4[4];
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const uint32_t pos = u + 4 * g + k;
        const uint32_t s = pw[pos & (kEvD - 1)];
        v4[k] = pos < (uint32_t)kEvD ? s : (s == 0 ? 0u : q - s);
      }
      *reinterpret_cast<uint4*>(sm + kTcA + (tid >> 3) * 2048 + g * 128 + (tid & 7) * 16) =
          make_uint4(v4[0], v4[1], v4[2], v4[3]);
    }
    tc::fence_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    if (tid == 0) {
      tc::fence_after_sync();
#pragma unroll
      for (int h = 0; h < 2; ++h)
#pragma unroll
        for (int ks = 0; ks < kTcCols / 32; ++ks)
          tc::mma_u8(tbase + 256 * h, tc::smem_desc(s0 + h * 1024 + ks * 8192, 2048, 128),
                     tc::smem_desc(s0 + kTcA + ks * 8192, 2048, 128), idesc,
                     (it | (uint32_t)ks) != 0);
      tc::mma_commit(bar);
    }
  }
  if (ok && it > 0) ok = mbar_wait(bar, (it - 1) & 1, err);
  ok = __syncthreads_and(ok);
  // per-position byte sums of the coefficients and of their negations
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    atomicAdd(&sums[4 * u + i], psum[i]);
    atomicAdd(&sums[256 + 4 * u + i], nsum[i]);
  }
  __syncthreads();
  {
    // S[t][i] = sum_{v >= t} P[v][i] + sum_{v < t} N[v][i], thread (t, i) = (tid / 4, tid % 4)
    const int t = tid >> 2, i = tid & 3;
    uint32_t acc = 0;
    for (int v = 0; v < kEvD; ++v) acc += v >= t ? sums[4 * v + i] : sums[256 + 4 * v + i];
    corr[tid] = acc;
  }
  __syncthreads();
  tc::fence_after_sync();
  if (ok && it > 0) {
    const int h = warp >> 2, wl = warp & 3;
    const int row = 128 * h + 32 * wl + lane;
    const uint32_t base = tc::tmem_addr(tbase, 32 * wl, 256 * h);
#pragma unroll 1
    for (int t0 = 0; t0 < kEvD; t0 += 2) {
      uint32_t dv[8];
      tc::tmem_ld8(base + 4 * t0, dv);
      tc::tmem_ld_wait();
#pragma unroll
      for (int k = 0; k < 2; ++k) {
        const int t = t0 + k;
        long long v = 0;
#pragma unroll
        for (int i = 0; i < 4; ++i)
          v += ((long long)dv[4 * k + i] - (long long)corr[4 * t + i]) << (8 * i);
        long long r = v % (long long)q;
        if (r < 0) r += q;
        atomicAdd(&gsum[(size_t)row * kEvD + t], (unsigned long long)r);
      }
    }
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tbase, 512);
}

__global__ void jl_eval_finish_kernel(const unsigned long long* __restrict__ gsum,
                                      uint32_t* __restrict__ evals, size_t n, uint32_t q) {
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
    evals[i] = (uint32_t)(gsum[i] % q);
}

}  // namespace

size_t jl_scratch_bytes(size_t rows, size_t, int) { return 2 * rows * sizeof(unsigned long long); }

int launch_jl_project(const FieldParams& f, const uint8_t seed[32], size_t rows,
                      const uint32_t* parts, size_t num_parts, size_t cols, size_t d,
                      uint32_t* p_out, int8_t* flat_out, void* scratch, size_t scratch_bytes,
                      int num_sms, int* err, cudaStream_t s) {
  if (rows == 0 || rows > 256 || d == 0 || cols % d != 0 || num_parts == 0 ||
      num_parts > 0xFFFFFFFFull)
    return GRID_ERR_INVALID_PARAMETERS;
  if (scratch_bytes < jl_scratch_bytes(rows, num_parts, num_sms)) return GRID_ERR_INVALID_PARAMETERS;
  ChachaKey key;
  for (int i = 0; i < 8; ++i)
    key.k[i] = (uint32_t)seed[4 * i] | ((uint32_t)seed[4 * i + 1] << 8) |
               ((uint32_t)seed[4 * i + 2] << 16) | ((uint32_t)seed[4 * i + 3] << 24);
  const int packed_len = (int)((rows + 3) / 4);
  unsigned long long* gpos = static_cast<unsigned long long*>(scratch);
  unsigned long long* gneg = gpos + rows;
  cudaError_t e = cudaMemsetAsync(gpos, 0, 2 * rows * sizeof(unsigned long long), s);
  if (e != cudaSuccess) return cuda_status(e);
  static int tc_bps_whole[kMaxDevices] = {}, tc_bps_part[kMaxDevices] = {},
             tc_bps_flat[kMaxDevices] = {};
  int dev = 0, bps = 0;
  // the int8 entries come out of the projection kernel itself when the
  // columns split into 32 polynomials x 8 coefficients and rows fill the blocks
  const unsigned long long npoly = cols / d;
  const bool fused_flat = flat_out && packed_len == 64 && d % 8 == 0 && npoly % 32 == 0 &&
                          (reinterpret_cast<uintptr_t>(flat_out) & 3u) == 0;
  const unsigned long long tc_per_part =
      fused_flat ? npoly / 32 * (d / 8) : (cols + kTcCols - 1) / kTcCols;
  const unsigned long long tc_chunks = tc_per_part * num_parts;
  bool use_tc = cols > 0 && cudaGetDevice(&dev) == cudaSuccess &&
                (fused_flat ? prepare_kernel(jl_tc_kernel<true, true>, kTcSmem, kTcThreads, dev,
                                             tc_bps_flat, &bps)
                 : packed_len == 64
                     ? prepare_kernel(jl_tc_kernel<true>, kTcSmem, kTcThreads, dev, tc_bps_whole,
                                      &bps)
                     : prepare_kernel(jl_tc_kernel<false>, kTcSmem, kTcThreads, dev, tc_bps_part,
                                      &bps)) == GRID_OK;
  // Resident CTAs per SM: the occupancy query has reported 1 for this kernel
  // where shared memory admits 3 (measured 20 % slower), so take the larger of
  // it and what the SM's shared memory holds. The grid-stride chunk loop makes
  // any count correct.
  static int smem_bps[kMaxDevices] = {};
  if (use_tc && smem_bps[dev] == 0) {
    int per_sm = 0, reserved = 0;
    if (cudaDeviceGetAttribute(&per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev) !=
            cudaSuccess ||
        cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev) !=
            cudaSuccess)
      per_sm = 0;
    const int fit = per_sm / (int)(kTcSmem + (uint32_t)reserved);
    smem_bps[dev] = std::max(1, std::min(fit, 2048 / kTcThreads));
  }
  if (use_tc) bps = std::max(bps, smem_bps[dev]);
  unsigned long long tc_grid = (unsigned long long)num_sms * (unsigned long long)(bps > 0 ? bps : 1);
  if (tc_grid > tc_chunks) tc_grid = tc_chunks;
  // exactness bound of the int32 accumulators: columns per CTA
  if (use_tc && tc_grid > 0 &&
      (tc_chunks + tc_grid - 1) / tc_grid * (unsigned long long)kTcCols > kTcMaxColsPerCta)
    use_tc = false;
  const unsigned long long plane = (unsigned long long)num_parts * cols;  // flat bytes per row
  if (use_tc) {
    if (fused_flat)
      jl_tc_kernel<true, true><<<(unsigned)tc_grid, kTcThreads, kTcSmem, s>>>(
          parts, cols, (int)rows, packed_len, key, tc_chunks, tc_per_part, (int)d, plane,
          flat_out, gpos, f.q, err);
    else if (packed_len == 64)
      jl_tc_kernel<true><<<(unsigned)tc_grid, kTcThreads, kTcSmem, s>>>(
          parts, cols, (int)rows, packed_len, key, tc_chunks, tc_per_part, (int)d, plane,
          nullptr, gpos, f.q, err);
    else
      jl_tc_kernel<false><<<(unsigned)tc_grid, kTcThreads, kTcSmem, s>>>(
          parts, cols, (int)rows, packed_len, key, tc_chunks, tc_per_part, (int)d, plane,
          nullptr, gpos, f.q, err);
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_status(e);
  } else if (cols > 0) {
    const unsigned long long chunks = (cols + 31) / 32 * num_parts;
    unsigned long long blocks = (chunks + kJlWarps - 1) / kJlWarps;
    const unsigned long long cap = (unsigned long long)num_sms * 8;
    if (blocks > cap) blocks = cap;
    if (packed_len == 64)
      jl_project_kernel<true><<<(unsigned)blocks, kJlThreads, 0, s>>>(
          parts, cols, (int)num_parts, (int)rows, packed_len, key, gpos, gneg, f.q);
    else
      jl_project_kernel<false><<<(unsigned)blocks, kJlThreads, 0, s>>>(
          parts, cols, (int)num_parts, (int)rows, packed_len, key, gpos, gneg, f.q);
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_status(e);
  }
  jl_finish_kernel<<<(unsigned)((rows + 255) / 256), 256, 0, s>>>(gpos, gneg, p_out, (int)rows, f.q);
  e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_status(e);
  if (flat_out && cols > 0 && !(use_tc && fused_flat)) {
    const unsigned long long n = cols / d;
    const unsigned long long work = (unsigned long long)num_parts * d * ((n + 127) / 128);
    unsigned long long blocks = (work + kJlWarps - 1) / kJlWarps;
    const unsigned long long cap = (unsigned long long)num_sms * 8;
    if (blocks > cap) blocks = cap;
    if (packed_len == 64)
      jl_flat_kernel<true><<<(unsigned)blocks, kJlThreads, 0, s>>>(
          cols, (int)d, (int)num_parts, (int)rows, packed_len, key, flat_out);
    else
      jl_flat_kernel<false><<<(unsigned)blocks, kJlThreads, 0, s>>>(
          cols, (int)d, (int)num_parts, (int)rows, packed_len, key, flat_out);
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_status(e);
  }
  return GRID_OK;
}


size_t jl_evals_scratch_bytes() { return (size_t)kEvRows * kEvD * sizeof(unsigned long long); }

// evals: kEvRows x d words. Only the LaBRADOR shape (256 rows, d = 64) has a
// kernel; other shapes return GRID_ERR_UNSUPPORTED_SIZE.
int launch_jl_evals(const FieldParams& f, const uint8_t seed[32], size_t rows,
                    const uint32_t* parts, size_t num_parts, size_t cols, size_t d,
                    uint32_t* evals, void* scratch, size_t scratch_bytes, int num_sms, int* err,
                    cudaStream_t s) {
  if (rows != (size_t)kEvRows || d != (size_t)kEvD) return GRID_ERR_UNSUPPORTED_SIZE;
  if (cols == 0 || cols % d != 0 || num_parts == 0 || num_parts > 0xFFFFFFFFull)
    return GRID_ERR_INVALID_PARAMETERS;
  if (scratch_bytes < jl_evals_scratch_bytes()) return GRID_ERR_INVALID_PARAMETERS;
  ChachaKey key;
  for (int i = 0; i < 8; ++i)
    key.k[i] = (uint32_t)seed[4 * i] | ((uint32_t)seed[4 * i + 1] << 8) |
               ((uint32_t)seed[4 * i + 2] << 16) | ((uint32_t)seed[4 * i + 3] << 24);
  unsigned long long* gsum = static_cast<unsigned long long*>(scratch);
  cudaError_t e = cudaMemsetAsync(gsum, 0, jl_evals_scratch_bytes(), s);
  if (e != cudaSuccess) return cuda_status(e);
  const unsigned long long nchunks = (cols + kTcCols - 1) / kTcCols * num_parts;
  // one CTA per SM (all 512 tensor-memory columns); more CTAs only where a CTA
  // would see more than kTcMaxColsPerCta columns (they queue for an SM)
  unsigned long long grid = (unsigned long long)num_sms;
  const unsigned long long need = (nchunks * kTcCols + kTcMaxColsPerCta - 1) / kTcMaxColsPerCta;
  if (grid < need) grid = need;
  if (grid > nchunks) grid = nchunks;
  if (grid > 0x7FFFFFFFull) return GRID_ERR_INVALID_PARAMETERS;
  int dev = 0;
  if ((e = cudaGetDevice(&dev)) != cudaSuccess) return cuda_status(e);
  static int bps_cache[kMaxDevices] = {};
  int bps = 0;
  int rc = prepare_kernel(jl_eval_tc_kernel, kEvSmem, kTcThreads, dev, bps_cache, &bps);
  if (rc) return rc;
  jl_eval_tc_kernel<<<(unsigned)grid, kTcThreads, kEvSmem, s>>>(parts, cols, key, nchunks, gsum,
                                                               f.q, err);
  if ((e = cudaGetLastError()) != cudaSuccess) return cuda_status(e);
  const size_t n = (size_t)kEvRows * kEvD;
  jl_eval_finish_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(gsum, evals, n, f.q);
  return cuda_status(cudaGetLastError());
}

}  // namespace grid
