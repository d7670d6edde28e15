// Evaluation-domain pieces of the LaBRADOR garbage h and the amortized
// witness.
//
// Reference paths replaced:
//   compute_garbage_h (labrador/src/main_protocol/garbage.rs:101-133):
//     h_ij = (<phi_i, s_j> + <phi_j, s_i>) * 2^-1 for i <= j, garbage_index order
//     (main_protocol/mod.rs:664-670). With C = Phi S^T from the evaluation-domain
//     product (commit.cu), symmetrize_half_kernel forms (C_ij + C_ji) * 2^-1 on
//     the upper triangle before one INTT per output.
//   compute_amortized_witness (labrador/src/main_protocol/amortization.rs:61-84),
//     z[k] = sum_i c_i s_i[k]; the challenges c_i come from the host's
//     transcript. amortize_kernel sums c_hat_i (.) s_hat_i[k] per evaluation
//     point with an exact 96-bit accumulator and reduces once.
// Both kernels are memory bound and tiny next to the transforms around them.
#include <cuda_runtime.h>

#include "grid_field.cuh"
#include "grid_internal.h"

namespace grid {
namespace {

// C: dense [r][r][d]; H: packed upper triangle [r(r+1)/2][d]. two_inv: the
// Montgomery word of 2^-1 = (q + 1) / 2.
__global__ void symmetrize_half_kernel(const uint32_t* __restrict__ C, uint32_t* __restrict__ H,
                                       int r, int d, uint32_t two_inv, FieldParams f) {
  const size_t total = (size_t)r * r * d;
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  for (size_t w = (size_t)blockIdx.x * blockDim.x + threadIdx.x; w < total; w += stride) {
    const int e = (int)(w % d);
    const size_t ij = w / d;
    const int i = (int)(ij / r), j = (int)(ij % r);
    if (j < i) continue;
    const uint32_t s = add_mod(C[ij * d + e], C[((size_t)j * r + i) * d + e], f.q);
    const size_t idx = (size_t)i * r - ((size_t)i * (i - 1)) / 2 + (size_t)(j - i);
    H[idx * d + e] = mont_mul(s, two_inv, f.q, f.qinv);
  }
}

// z_hat[k][e] = sum_i c_hat[i][e] s_hat[i][k][e] (Montgomery words).
__global__ void amortize_kernel(const uint32_t* __restrict__ c_hat,
                                const uint32_t* __restrict__ s_hat, uint32_t* __restrict__ z_hat,
                                int r, size_t n, int d, FieldParams f) {
  const size_t total = n * d;
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  for (size_t w = (size_t)blockIdx.x * blockDim.x + threadIdx.x; w < total; w += stride) {
    const int e = (int)(w % d);
    Acc96 acc;
    acc96_zero(acc);
    for (int i = 0; i < r; ++i) acc96_mad(acc, c_hat[(size_t)i * d + e], s_hat[(size_t)i * total + w]);
    z_hat[w] = acc96_reduce(acc, f);
  }
}

unsigned blocks_for(const grid_gpu_plan* p, size_t work) {
  size_t b = (work + 255) / 256;
  const size_t cap = (size_t)p->num_sms * 8;
  if (b > cap) b = cap;
  return b ? (unsigned)b : 1u;
}

}  // namespace

int launch_symmetrize_half(const grid_gpu_plan* p, const uint32_t* C, int r, uint32_t* H,
                           cudaStream_t s) {
  // (q + 1) / 2 in Montgomery form: ((q + 1) / 2) * 2^32 mod q
  const uint32_t two_inv =
      (uint32_t)(((unsigned __int128)((p->f.q + 1ull) / 2) << 32) % p->f.q);
  symmetrize_half_kernel<<<blocks_for(p, (size_t)r * r * p->d), 256, 0, s>>>(C, H, r, (int)p->d,
                                                                            two_inv, p->f);
  return cuda_status(cudaGetLastError());
}

int launch_amortize(const grid_gpu_plan* p, const uint32_t* c_hat, const uint32_t* s_hat, int r,
                    size_t n, uint32_t* z_hat, cudaStream_t s) {
  amortize_kernel<<<blocks_for(p, n * p->d), 256, 0, s>>>(c_hat, s_hat, z_hat, r, n, (int)p->d,
                                                          p->f);
  return cuda_status(cudaGetLastError());
}

}  // namespace grid
