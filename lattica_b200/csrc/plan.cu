// Plans, host-side field arithmetic and the NTT entry points of the C ABI.
//
// Plan construction restates the reference's parameter derivation so the
// device twiddles are exactly the reference's roots:
//   PrimeField modulus checks      algebra/src/arith/prime.rs:31-46
//   Montgomery constants           algebra/src/arith/prime.rs:60-91
//   find_generator (smallest g)    algebra/src/arith/prime.rs:645-687
//   root_of_unity / max_ntt_size   algebra/src/arith/prime.rs:566-607
//   NttPlan::build error order     algebra/src/arith/ntt.rs:124-154
//   TwistedNttPlan::build (psi)    algebra/src/poly/ntt.rs:139-154
#include <cuda_runtime.h>

#include <cstdlib>
#include <cstring>
#include <new>
#include <vector>

#include "grid_async.cuh"
#include "grid_internal.h"

namespace grid {

// ---------------------------------------------------------------------------
// Host field arithmetic (exact, 128-bit intermediates)
// ---------------------------------------------------------------------------
namespace {

uint64_t mulmod(uint64_t a, uint64_t b, uint64_t m) {
  return (uint64_t)((unsigned __int128)a * b % m);
}

uint64_t powmod(uint64_t b, uint64_t e, uint64_t m) {
  uint64_t r = 1 % m;
  b %= m;
  while (e) {
    if (e & 1) r = mulmod(r, b, m);
    b = mulmod(b, b, m);
    e >>= 1;
  }
  return r;
}

// Deterministic Miller-Rabin for 64-bit n (same small-prime screen and base
// set as the reference's const-eval primality check).
bool is_prime(uint64_t n) {
  static const uint64_t small[] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37};
  static const uint64_t bases[] = {2, 325, 9375, 28178, 450775, 9780504, 1795265022};
  if (n < 2) return false;
  for (uint64_t p : small) {
    if (n == p) return true;
    if (n % p == 0) return false;
  }
  uint64_t d = n - 1;
  int s = 0;
  while (!(d & 1)) {
    d >>= 1;
    ++s;
  }
  for (uint64_t a0 : bases) {
    const uint64_t a = a0 % n;
    if (a == 0) continue;
    uint64_t x = powmod(a, d, n);
    if (x == 1 || x == n - 1) continue;
    bool comp = true;
    for (int r = 1; r < s; ++r) {
      x = mulmod(x, x, n);
      if (x == n - 1) {
        comp = false;
        break;
      }
    }
    if (comp) return false;
  }
  return true;
}

// Canonical integers are used on the host; Montgomery words are produced at
// the end with to_mont.
struct HostField {
  uint64_t q;
  uint32_t to_mont(uint64_t v) const { return (uint32_t)(((unsigned __int128)(v % q) << 32) % q); }
  uint64_t mul(uint64_t a, uint64_t b) const { return mulmod(a, b, q); }
  uint64_t pow(uint64_t a, uint64_t e) const { return powmod(a, e, q); }
  uint64_t inv(uint64_t a) const { return powmod(a, q - 2, q); }
};

uint64_t smallest_generator(uint64_t q) {
  std::vector<uint64_t> factors;
  uint64_t n = q - 1;
  for (uint64_t d = 2; d <= n / d; ++d) {
    if (n % d == 0) {
      factors.push_back(d);
      while (n % d == 0) n /= d;
    }
  }
  if (n > 1) factors.push_back(n);
  for (uint64_t g = 2; g < q; ++g) {
    bool ok = true;
    for (uint64_t f : factors)
      if (powmod(g, (q - 1) / f, q) == 1) {
        ok = false;
        break;
      }
    if (ok) return g;
  }
  return 0;
}

// root_of_unity(n) as an integer, 0 when the reference returns None.
uint64_t root_of_unity(uint64_t q, uint64_t g, uint64_t n) {
  if (n == 0 || (q - 1) % n != 0 || g == 0) return 0;
  const uint64_t r = powmod(g, (q - 1) / n, q);
  if (powmod(r, n, q) != 1) return 0;
  if (n > 1 && powmod(r, n / 2, q) == 1) return 0;
  return r;
}

uint32_t bit_reverse(uint32_t x, uint32_t bits) {
  uint32_t r = 0;
  for (uint32_t i = 0; i < bits; ++i) r |= ((x >> i) & 1u) << (bits - 1 - i);
  return r;
}

uint32_t shoup(uint32_t w, uint32_t qinv) { return w * qinv; }

__global__ void pointwise_kernel(uint32_t* __restrict__ dst, const uint32_t* __restrict__ rhs,
                                 size_t n, FieldParams f) {
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
    dst[i] = mont_mul(dst[i], rhs[i], f.q, f.qinv);
}

__global__ void add_kernel(uint32_t* __restrict__ dst, const uint32_t* __restrict__ rhs, size_t n,
                           uint32_t q) {
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
    dst[i] = add_mod(dst[i], rhs[i], q);
}

}  // namespace

int cuda_status(cudaError_t e) {
  if (e == cudaSuccess) return GRID_OK;
  if (e == cudaErrorMemoryAllocation) return GRID_ERR_OUT_OF_MEMORY;
  if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return GRID_ERR_NO_DEVICE;
  if (e == cudaErrorMisalignedAddress) return GRID_ERR_MISALIGNED;
  return GRID_ERR_CUDA;
}

int ensure_scratch(grid_gpu_plan* p, int slot, size_t bytes) {
  DeviceScratch& s = p->scratch[slot];
  if (s.bytes >= bytes) return GRID_OK;
  if (s.ptr) {
    cudaError_t e = cudaFree(s.ptr);
    s.ptr = nullptr;
    s.bytes = 0;
    if (e != cudaSuccess) return cuda_status(e);
  }
  void* ptr = nullptr;
  cudaError_t e = cudaMalloc(&ptr, bytes);
  if (e != cudaSuccess) return cuda_status(e);
  s.ptr = ptr;
  s.bytes = bytes;
  return GRID_OK;
}

int launch_pointwise(const grid_gpu_plan* p, uint32_t* dst, const uint32_t* rhs, size_t words,
                     cudaStream_t s) {
  if (words == 0) return GRID_OK;
  const int threads = 256;
  size_t blocks = (words + threads - 1) / threads;
  const size_t cap = (size_t)p->num_sms * 8;
  if (blocks > cap) blocks = cap;
  pointwise_kernel<<<(unsigned)blocks, threads, 0, s>>>(dst, rhs, words, p->f);
  return cuda_status(cudaGetLastError());
}

int launch_add(const grid_gpu_plan* p, uint32_t* dst, const uint32_t* rhs, size_t words,
               cudaStream_t s) {
  if (words == 0) return GRID_OK;
  const int threads = 256;
  size_t blocks = (words + threads - 1) / threads;
  const size_t cap = (size_t)p->num_sms * 8;
  if (blocks > cap) blocks = cap;
  add_kernel<<<(unsigned)blocks, threads, 0, s>>>(dst, rhs, words, p->f.q);
  return cuda_status(cudaGetLastError());
}

// ---------------------------------------------------------------------------
// Host-buffer pipeline: chunked H2D -> op -> D2H over two streams so copies in
// both directions overlap the kernels of the neighbouring chunk.
// ---------------------------------------------------------------------------
int host_pipeline(grid_gpu_plan* p, const uint32_t* const* ins, int nin, uint32_t* out,
                  size_t nunits, size_t unit_words,
                  int (*op)(grid_gpu_plan*, const uint32_t* const*, uint32_t*, size_t,
                            cudaStream_t, void*),
                  void* ctx) {
  if (nunits == 0) return GRID_OK;
  constexpr size_t kChunkBytes = 32u << 20;
  size_t chunk = kChunkBytes / (unit_words * 4);
  if (chunk < 1) chunk = 1;
  if (chunk > nunits) chunk = nunits;
  const size_t chunk_bytes = chunk * unit_words * 4;
  // Scratch slots: stream j uses slots [j*3, j*3 + nin] for inputs and output.
  for (int j = 0; j < 2; ++j)
    for (int k = 0; k <= nin; ++k) {
      int st = ensure_scratch(p, j * 3 + k, chunk_bytes);
      if (st) return st;
    }
  cudaStream_t streams[2] = {p->stream, p->stream2};
  int status = GRID_OK;
  size_t ci = 0;
  for (size_t off = 0; off < nunits; off += chunk, ++ci) {
    const size_t n = (nunits - off) < chunk ? (nunits - off) : chunk;
    const int j = (int)(ci & 1);
    cudaStream_t s = streams[j];
    const uint32_t* din[4];
    for (int k = 0; k < nin; ++k) {
      uint32_t* dptr = static_cast<uint32_t*>(p->scratch[j * 3 + k].ptr);
      cudaError_t e = cudaMemcpyAsync(dptr, ins[k] + off * unit_words, n * unit_words * 4,
                                      cudaMemcpyHostToDevice, s);
      if (e != cudaSuccess) { status = cuda_status(e); break; }
      din[k] = dptr;
    }
    if (status) break;
    uint32_t* dout = static_cast<uint32_t*>(p->scratch[j * 3 + nin].ptr);
    status = op(p, din, dout, n, s, ctx);
    if (status) break;
    cudaError_t e = cudaMemcpyAsync(out + off * unit_words, dout, n * unit_words * 4,
                                    cudaMemcpyDeviceToHost, s);
    if (e != cudaSuccess) { status = cuda_status(e); break; }
  }
  cudaError_t e1 = cudaStreamSynchronize(p->stream2);
  const int fin = finish_host_call(p, p->stream);
  if (status) return status;
  if (e1 != cudaSuccess) return cuda_status(e1);
  return fin;
}

// Synchronise `s`, then read and clear the plan's device error word (and, on
// a ring plan, those of the auxiliary primes' plans).
int finish_host_call(grid_gpu_plan* p, cudaStream_t s) {
  cudaError_t e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_status(e);
  int derr = 0;
  e = cudaMemcpy(&derr, p->d_err, sizeof(int), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_status(e);
  int status = GRID_OK;
  if (derr) {
    cudaMemset(p->d_err, 0, sizeof(int));
    status = derr == GRID_DEV_SAMPLE_SHORT ? GRID_ERR_SAMPLE_EXHAUSTED : GRID_ERR_TIMEOUT;
  }
  // a ring plan's products run on the auxiliary primes' plans: their words too
  for (grid_gpu_plan* sub : p->crt) {
    if (!sub) continue;
    const int sst = grid_gpu_plan_check(sub, s);
    if (!status) status = sst;
  }
  return status;
}

}  // namespace grid

using namespace grid;

namespace {

bool aligned16(const void* p) { return ((uintptr_t)p & 15u) == 0; }

int ntt_op_fwd(grid_gpu_plan* p, const uint32_t* const* in, uint32_t* out, size_t n,
               cudaStream_t s, void*) {
  return launch_ntt(p, MODE_FWD, in[0], nullptr, out, n, s);
}
int ntt_op_inv(grid_gpu_plan* p, const uint32_t* const* in, uint32_t* out, size_t n,
               cudaStream_t s, void*) {
  return launch_ntt(p, MODE_INV, in[0], nullptr, out, n, s);
}
int ntt_op_mulinv(grid_gpu_plan* p, const uint32_t* const* in, uint32_t* out, size_t n,
                  cudaStream_t s, void*) {
  return launch_ntt(p, MODE_MULINV, in[0], in[1], out, n, s);
}
int ntt_op_polymul(grid_gpu_plan* p, const uint32_t* const* in, uint32_t* out, size_t n,
                   cudaStream_t s, void*) {
  // NTT(b) into the output buffer, then out = INTT(NTT(a) (.) NTT(b)) in place.
  int st = launch_ntt(p, MODE_FWD, in[1], nullptr, out, n, s);
  if (st) return st;
  return launch_ntt(p, MODE_MULINV, in[0], out, out, n, s);
}

size_t crt_poly_words(const grid_gpu_plan* p, size_t npolys) {
  return round_up(npolys * p->d, 64);  // 256-byte aligned sub-buffers
}

// Negacyclic products on a ring plan without an NTT for q: per auxiliary
// prime, lift a and b, transform b, multiply and invert; then reconstruct.
// scratch: 4 * crt_poly_words words.
int crt_poly_mul(const grid_gpu_plan* p, const uint32_t* a, const uint32_t* b, uint32_t* out,
                 uint32_t* scratch, size_t npolys, cudaStream_t s) {
  if (!crt_bound_ok(p, 1)) return GRID_ERR_INVALID_PARAMETERS;
  const size_t w = npolys * p->d, stride = crt_poly_words(p, npolys);
  uint32_t* aj[3] = {scratch, scratch + stride, scratch + 2 * stride};
  uint32_t* bt = scratch + 3 * stride;
  int rc = GRID_OK;
  for (int j = 0; j < 3 && !rc; ++j) {
    const grid_gpu_plan* sub = p->crt[j];
    rc = crt_lift(p, a, w, j == 0 ? aj[0] : nullptr, j == 1 ? aj[1] : nullptr,
                  j == 2 ? aj[2] : nullptr, s);
    if (!rc)
      rc = crt_lift(p, b, w, j == 0 ? bt : nullptr, j == 1 ? bt : nullptr, j == 2 ? bt : nullptr,
                    s);
    if (!rc) rc = launch_ntt(sub, MODE_FWD, bt, nullptr, bt, npolys, s);
    if (!rc) rc = launch_ntt(sub, MODE_MULINV, aj[j], bt, aj[j], npolys, s);
  }
  if (rc) return rc;
  return crt_combine(p, aj[0], aj[1], aj[2], w, out, s);
}

}  // namespace

extern "C" {

const char* grid_gpu_status_string(int status) {
  switch (status) {
    case GRID_OK: return "ok";
    case GRID_ERR_LENGTH_MISMATCH: return "length mismatch";
    case GRID_ERR_LENGTH_NOT_POW2: return "length is not a power of two";
    case GRID_ERR_UNSUPPORTED_SIZE: return "unsupported NTT size for this modulus";
    case GRID_ERR_UNSUPPORTED_TWIST: return "modulus has no 2d-th root of unity (twist)";
    case GRID_ERR_INVALID_PARAMETERS: return "invalid parameters";
    case GRID_ERR_DIMENSION_MISMATCH: return "dimension mismatch";
    case GRID_ERR_INVALID_MODULUS: return "modulus is not an odd prime below 2^32";
    case GRID_ERR_NULL_POINTER: return "null pointer";
    case GRID_ERR_OUT_OF_MEMORY: return "out of device memory";
    case GRID_ERR_CUDA: return "CUDA error";
    case GRID_ERR_TIMEOUT: return "bounded device wait timed out";
    case GRID_ERR_UNSUPPORTED_DEGREE: return "no kernel compiled for this ring degree";
    case GRID_ERR_MISALIGNED: return "device buffer not 16-byte aligned";
    case GRID_ERR_NO_DEVICE: return "no CUDA device";
    case GRID_ERR_SCRATCH_LIMIT: return "problem exceeds the no-alloc entry point's fixed scratch buffer";
    default: return "unknown status";
  }
}

uint32_t grid_gpu_abi_version(void) { return (1u << 16) | 1u; }

uint32_t grid_gpu_max_degree(void) { return kMaxDegree; }

}  // extern "C"

namespace {

// d = 64 transforms run on the tensor cores unless the environment variable
// GRID_GPU_NTT_ENGINE is "cuda_core" when the plan is created (the CUDA-core
// kernels serve every degree; both give identical words).
bool use_tensor_cores() {
  const char* v = std::getenv("GRID_GPU_NTT_ENGINE");
  return !(v && std::strcmp(v, "cuda_core") == 0);
}

// Contractions over point-major evaluations (TMA-fed) unless
// GRID_GPU_CONTRACTION=gather selects the poly-major kernels that gather
// their operands.
bool use_point_major() {
  const char* v = std::getenv("GRID_GPU_CONTRACTION");
  return !(v && std::strcmp(v, "gather") == 0);
}

// Device state every plan owns: SM count, error word, the host-buffer
// pipeline's streams and the fork streams of *_dev calls (on the current device).
cudaError_t init_device_state(grid_gpu_plan* p) {
  cudaError_t e;
  int sms = 0;
  if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, p->device)) != cudaSuccess)
    return e;
  p->num_sms = sms;
  if ((e = cudaMalloc(&p->d_err, sizeof(int))) != cudaSuccess) return e;
  if ((e = cudaMemset(p->d_err, 0, sizeof(int))) != cudaSuccess) return e;
  if ((e = cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking)) != cudaSuccess) return e;
  if ((e = cudaStreamCreateWithFlags(&p->stream2, cudaStreamNonBlocking)) != cudaSuccess) return e;
  int least = 0, greatest = 0;
  if ((e = cudaDeviceGetStreamPriorityRange(&least, &greatest)) != cudaSuccess) return e;
  if ((e = cudaStreamCreateWithPriority(&p->fork_hi, cudaStreamNonBlocking, greatest)) !=
      cudaSuccess)
    return e;
  return cudaStreamCreateWithPriority(&p->fork_lo, cudaStreamNonBlocking, least);
}

// Validation and every host-side table of a plan (no device work).
int fill_plan_host(uint64_t q, uint64_t d, grid_gpu_plan* p) {
  if (q < 3 || (q & 1) == 0 || q >= (1ull << 32) || !is_prime(q)) return GRID_ERR_INVALID_MODULUS;
  if (d == 0 || (d & (d - 1)) != 0) return GRID_ERR_LENGTH_NOT_POW2;
  const uint64_t g = smallest_generator(q);
  const uint64_t omega = root_of_unity(q, g, d);
  if (omega == 0) return GRID_ERR_UNSUPPORTED_SIZE;
  const uint64_t psi = root_of_unity(q, g, 2 * d);
  if (psi == 0) return GRID_ERR_UNSUPPORTED_TWIST;
  if (d > kMaxDegree || d < 8) return GRID_ERR_UNSUPPORTED_DEGREE;

  HostField hf{q};
  p->q = (uint32_t)q;
  p->d = (uint32_t)d;
  p->log_d = 0;
  while ((1u << p->log_d) < d) ++p->log_d;
  uint32_t qinv = 1;
  for (int i = 0; i < 5; ++i) qinv *= 2u - (uint32_t)q * qinv;
  p->f.q = (uint32_t)q;
  p->f.qinv = qinv;
  p->f.r1 = (uint32_t)((1ull << 32) % q);
  p->f.r2 = (uint32_t)(((unsigned __int128)1 << 64) % q);
  p->generator = hf.to_mont(g);
  p->psi = hf.to_mont(psi);
  p->psi_value = psi;
  p->omega = hf.to_mont(omega);
  const uint64_t ninv = hf.inv(d % q);
  p->n_inv = hf.to_mont(ninv);
  p->n_inv_value = ninv;

  // Merged twiddles psi^brv(k), k in [1, d).
  TwiddleTable& tw = p->tw;
  tw.zeta.assign(d, 0);
  tw.zeta_q.assign(d, 0);
  tw.izeta.assign(d, 0);
  tw.izeta_q.assign(d, 0);
  const uint64_t psi_inv = hf.inv(psi);
  for (uint32_t k = 1; k < d; ++k) {
    const uint32_t e_k = bit_reverse(k, p->log_d);
    tw.zeta[k] = hf.to_mont(hf.pow(psi, e_k));
    tw.izeta[k] = hf.to_mont(hf.pow(psi_inv, e_k));
    tw.zeta_q[k] = shoup(tw.zeta[k], qinv);
    tw.izeta_q[k] = shoup(tw.izeta[k], qinv);
  }
  tw.ninv = hf.to_mont(ninv);
  tw.ninv_q = shoup(tw.ninv, qinv);
  tw.izeta1_ninv = hf.to_mont(hf.mul(hf.pow(psi_inv, bit_reverse(1, p->log_d)), ninv));
  tw.izeta1_ninv_q = shoup(tw.izeta1_ninv, qinv);
  return GRID_OK;
}

}  // namespace

extern "C" {

int grid_gpu_plan_describe(uint64_t q, uint64_t d, grid_gpu_plan_info* info, uint32_t* zeta,
                           uint32_t* izeta) {
  grid_gpu_plan tmp;
  const int st = fill_plan_host(q, d, &tmp);
  if (st) return st;
  if (info) grid_gpu_plan_get_info(&tmp, info);
  if (zeta && izeta) grid_gpu_plan_get_twiddles(&tmp, zeta, izeta);
  return GRID_OK;
}

int grid_gpu_plan_create(uint64_t q, uint64_t d, grid_gpu_plan** out) {
  if (!out) return GRID_ERR_NULL_POINTER;
  *out = nullptr;
  grid_gpu_plan* p = new (std::nothrow) grid_gpu_plan();
  if (!p) return GRID_ERR_OUT_OF_MEMORY;
  int st = fill_plan_host(q, d, p);
  if (st) {
    delete p;
    return st;
  }
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    delete p;
    return cuda_status(e);
  }
  p->device = dev;
  const TwiddleTable& tw = p->tw;
  std::vector<uint2> dev_tw(2 * d + 2);
  for (uint32_t k = 0; k < d; ++k) {
    dev_tw[k] = make_uint2(tw.zeta[k], tw.zeta_q[k]);
    dev_tw[d + k] = make_uint2(tw.izeta[k], tw.izeta_q[k]);
  }
  dev_tw[2 * d] = make_uint2(tw.ninv, tw.ninv_q);
  dev_tw[2 * d + 1] = make_uint2(tw.izeta1_ninv, tw.izeta1_ninv_q);

  int status = GRID_OK;
  do {
    if ((e = init_device_state(p)) != cudaSuccess) break;
    if ((e = cudaMalloc(&p->d_tw, dev_tw.size() * sizeof(uint2))) != cudaSuccess) break;
    if ((e = cudaMemcpy(p->d_tw, dev_tw.data(), dev_tw.size() * sizeof(uint2),
                        cudaMemcpyHostToDevice)) != cudaSuccess) break;
    p->tc_emm = use_tensor_cores();
    p->pm_emm = p->tc_emm && use_point_major();
    if ((d == 64 || d == 256) && use_tensor_cores()) {
      std::vector<unsigned char> tcw;
      if (d == 64)
        build_tc_tables(p->q, p->d, p->psi_value, p->n_inv_value, tcw);
      else
        build_tc256_tables(p->q, p->psi_value, tcw);
      if ((e = cudaMalloc(&p->d_tcw, tcw.size())) != cudaSuccess) break;
      if ((e = cudaMemcpy(p->d_tcw, tcw.data(), tcw.size(), cudaMemcpyHostToDevice)) !=
          cudaSuccess)
        break;
    }
  } while (0);
  if (e != cudaSuccess) status = cuda_status(e);
  if (status) {
    grid_gpu_plan_destroy(p);
    return status;
  }
  *out = p;
  return GRID_OK;
}

int grid_gpu_ring_plan_create(uint64_t q, uint64_t d, grid_gpu_plan** out) {
  if (!out) return GRID_ERR_NULL_POINTER;
  *out = nullptr;
  int st;
  {
    grid_gpu_plan probe;
    st = fill_plan_host(q, d, &probe);
  }
  // An NTT-friendly (q, d) gets the ordinary plan, like the reference's
  // dispatch in negacyclic_mul_coeffs (algebra/src/poly/ring.rs:79-102).
  if (st != GRID_ERR_UNSUPPORTED_SIZE && st != GRID_ERR_UNSUPPORTED_TWIST)
    return st ? st : grid_gpu_plan_create(q, d, out);
  if (d > kMaxDegree || d < 8) return GRID_ERR_UNSUPPORTED_DEGREE;
  grid_gpu_plan* p = new (std::nothrow) grid_gpu_plan();
  if (!p) return GRID_ERR_OUT_OF_MEMORY;
  HostField hf{q};
  p->q = (uint32_t)q;
  p->d = (uint32_t)d;
  p->log_d = 0;
  while ((1u << p->log_d) < d) ++p->log_d;
  crt_consts((uint32_t)q, &p->crt_c);
  p->f = p->crt_c.fq;
  p->generator = hf.to_mont(smallest_generator(q));
  p->ntt_status = st;
  cudaError_t e = cudaGetDevice(&p->device);
  if (e == cudaSuccess) e = init_device_state(p);
  int status = e == cudaSuccess ? GRID_OK : cuda_status(e);
  for (int j = 0; j < 3 && !status; ++j) status = grid_gpu_plan_create(crt_moduli()[j], d, &p->crt[j]);
  if (status) {
    grid_gpu_plan_destroy(p);
    return status;
  }
  *out = p;
  return GRID_OK;
}

int grid_gpu_plan_ring_kind(const grid_gpu_plan* p, int* kind, uint32_t* aux_moduli) {
  if (!p || !kind) return GRID_ERR_NULL_POINTER;
  *kind = is_crt(p) ? 1 : 0;
  if (aux_moduli && is_crt(p))
    for (int j = 0; j < 3; ++j) aux_moduli[j] = p->crt[j]->q;
  return GRID_OK;
}

int grid_gpu_plan_destroy(grid_gpu_plan* p) {
  if (!p) return GRID_ERR_NULL_POINTER;
  for (grid_gpu_plan*& sub : p->crt)
    if (sub) {
      grid_gpu_plan_destroy(sub);
      sub = nullptr;
    }
  int prev = -1;
  cudaGetDevice(&prev);
  if (prev != p->device) cudaSetDevice(p->device);
  if (p->stream) cudaStreamSynchronize(p->stream);
  if (p->stream2) cudaStreamSynchronize(p->stream2);
  if (p->fork_hi) cudaStreamSynchronize(p->fork_hi);
  if (p->fork_lo) cudaStreamSynchronize(p->fork_lo);
  for (auto& s : p->scratch)
    if (s.ptr) cudaFree(s.ptr);
  if (p->d_tw) cudaFree(p->d_tw);
  if (p->d_tcw) cudaFree(p->d_tcw);
  if (p->d_err) cudaFree(p->d_err);
  if (p->stream) cudaStreamDestroy(p->stream);
  if (p->stream2) cudaStreamDestroy(p->stream2);
  if (p->fork_hi) cudaStreamDestroy(p->fork_hi);
  if (p->fork_lo) cudaStreamDestroy(p->fork_lo);
  if (prev >= 0 && prev != p->device) cudaSetDevice(prev);
  delete p;
  return GRID_OK;
}

int grid_gpu_plan_get_info(const grid_gpu_plan* p, grid_gpu_plan_info* out) {
  if (!p || !out) return GRID_ERR_NULL_POINTER;
  out->q = p->q;
  out->d = p->d;
  out->generator = p->generator;
  out->psi = p->psi;
  out->omega = p->omega;
  out->n_inv = p->n_inv;
  out->r_mod_q = p->f.r1;
  out->r2_mod_q = p->f.r2;
  uint64_t v = (uint64_t)p->q - 1, m = 1;
  while (!(v & 1)) {
    v >>= 1;
    m <<= 1;
  }
  out->max_ntt_size = m;
  return GRID_OK;
}

int grid_gpu_plan_get_twiddles(const grid_gpu_plan* p, uint32_t* zeta, uint32_t* izeta) {
  if (!p || !zeta || !izeta) return GRID_ERR_NULL_POINTER;
  if (is_crt(p)) return p->ntt_status;  // no 2d-th root: no twiddles
  std::memcpy(zeta, p->tw.zeta.data(), p->d * sizeof(uint32_t));
  std::memcpy(izeta, p->tw.izeta.data(), p->d * sizeof(uint32_t));
  return GRID_OK;
}

int grid_gpu_plan_check(grid_gpu_plan* p, void* stream) {
  if (!p) return GRID_ERR_NULL_POINTER;
  cudaError_t e = cudaStreamSynchronize((cudaStream_t)stream);
  if (e != cudaSuccess) return cuda_status(e);
  int derr = 0;
  e = cudaMemcpy(&derr, p->d_err, sizeof(int), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_status(e);
  int status = GRID_OK;
  if (derr) {
    cudaMemset(p->d_err, 0, sizeof(int));
    status = derr == GRID_DEV_SAMPLE_SHORT ? GRID_ERR_SAMPLE_EXHAUSTED : GRID_ERR_TIMEOUT;
  }
  // a ring plan's products run on the auxiliary primes' plans: their words too
  for (grid_gpu_plan* sub : p->crt) {
    if (!sub) continue;
    const int sst = grid_gpu_plan_check(sub, stream);
    if (!status) status = sst;
  }
  return status;
}

int grid_gpu_ntt_forward_dev(const grid_gpu_plan* p, uint32_t* polys, size_t npolys,
                             void* stream) {
  if (!p || (!polys && npolys)) return GRID_ERR_NULL_POINTER;
  if (!aligned16(polys)) return GRID_ERR_MISALIGNED;
  return launch_ntt(p, MODE_FWD, polys, nullptr, polys, npolys, (cudaStream_t)stream);
}

int grid_gpu_ntt_inverse_dev(const grid_gpu_plan* p, uint32_t* polys, size_t npolys,
                             void* stream) {
  if (!p || (!polys && npolys)) return GRID_ERR_NULL_POINTER;
  if (!aligned16(polys)) return GRID_ERR_MISALIGNED;
  return launch_ntt(p, MODE_INV, polys, nullptr, polys, npolys, (cudaStream_t)stream);
}

int grid_gpu_ntt_mul_inverse_dev(const grid_gpu_plan* p, const uint32_t* a,
                                 const uint32_t* b_evals, uint32_t* out, size_t npolys,
                                 void* stream) {
  if (!p || ((!a || !b_evals || !out) && npolys)) return GRID_ERR_NULL_POINTER;
  if (!aligned16(a) || !aligned16(b_evals) || !aligned16(out)) return GRID_ERR_MISALIGNED;
  return launch_ntt(p, MODE_MULINV, a, b_evals, out, npolys, (cudaStream_t)stream);
}

size_t grid_gpu_poly_mul_scratch_words(const grid_gpu_plan* p, size_t npolys) {
  if (!p) return 0;
  return is_crt(p) ? 4 * crt_poly_words(p, npolys) : npolys * p->d;
}

int grid_gpu_poly_mul_dev(const grid_gpu_plan* p, const uint32_t* a, const uint32_t* b,
                          uint32_t* out, uint32_t* b_scratch, size_t npolys, void* stream) {
  if (!p || ((!a || !b || !out || !b_scratch) && npolys)) return GRID_ERR_NULL_POINTER;
  if (!aligned16(a) || !aligned16(b) || !aligned16(out) || !aligned16(b_scratch))
    return GRID_ERR_MISALIGNED;
  cudaStream_t s = (cudaStream_t)stream;
  if (is_crt(p)) return npolys ? crt_poly_mul(p, a, b, out, b_scratch, npolys, s) : GRID_OK;
  int st = launch_ntt(p, MODE_FWD, b, nullptr, b_scratch, npolys, s);
  if (st) return st;
  return launch_ntt(p, MODE_MULINV, a, b_scratch, out, npolys, s);
}

int grid_gpu_pointwise_mul_dev(const grid_gpu_plan* p, uint32_t* dst, const uint32_t* rhs,
                               size_t nwords, void* stream) {
  if (!p || ((!dst || !rhs) && nwords)) return GRID_ERR_NULL_POINTER;
  return launch_pointwise(p, dst, rhs, nwords, (cudaStream_t)stream);
}

int grid_gpu_ntt_forward(grid_gpu_plan* p, uint32_t* polys, size_t npolys) {
  if (!p || (!polys && npolys)) return GRID_ERR_NULL_POINTER;
  std::lock_guard<std::mutex> lk(p->mu);
  const uint32_t* ins[1] = {polys};
  return host_pipeline(p, ins, 1, polys, npolys, p->d, ntt_op_fwd, nullptr);
}

int grid_gpu_ntt_inverse(grid_gpu_plan* p, uint32_t* polys, size_t npolys) {
  if (!p || (!polys && npolys)) return GRID_ERR_NULL_POINTER;
  std::lock_guard<std::mutex> lk(p->mu);
  const uint32_t* ins[1] = {polys};
  return host_pipeline(p, ins, 1, polys, npolys, p->d, ntt_op_inv, nullptr);
}

int grid_gpu_ntt_mul_inverse(grid_gpu_plan* p, const uint32_t* a, const uint32_t* b_evals,
                             uint32_t* out, size_t npolys) {
  if (!p || ((!a || !b_evals || !out) && npolys)) return GRID_ERR_NULL_POINTER;
  std::lock_guard<std::mutex> lk(p->mu);
  const uint32_t* ins[2] = {a, b_evals};
  return host_pipeline(p, ins, 2, out, npolys, p->d, ntt_op_mulinv, nullptr);
}

int grid_gpu_poly_mul(grid_gpu_plan* p, const uint32_t* a, const uint32_t* b, uint32_t* out,
                      size_t npolys) {
  if (!p || ((!a || !b || !out) && npolys)) return GRID_ERR_NULL_POINTER;
  std::lock_guard<std::mutex> lk(p->mu);
  if (is_crt(p)) {
    if (npolys == 0) return GRID_OK;
    const size_t bytes = npolys * p->d * 4;
    const size_t sbytes = grid_gpu_poly_mul_scratch_words(p, npolys) * 4;
    int rc;
    if ((rc = ensure_scratch(p, 6, bytes)) || (rc = ensure_scratch(p, 7, bytes)) ||
        (rc = ensure_scratch(p, 8, bytes)) || (rc = ensure_scratch(p, 9, sbytes)))
      return rc;
    cudaStream_t st = p->stream;
    uint32_t* da = static_cast<uint32_t*>(p->scratch[6].ptr);
    uint32_t* db = static_cast<uint32_t*>(p->scratch[7].ptr);
    uint32_t* dout = static_cast<uint32_t*>(p->scratch[8].ptr);
    rc = cuda_status(cudaMemcpyAsync(da, a, bytes, cudaMemcpyHostToDevice, st));
    if (!rc) rc = cuda_status(cudaMemcpyAsync(db, b, bytes, cudaMemcpyHostToDevice, st));
    if (!rc)
      rc = crt_poly_mul(p, da, db, dout, static_cast<uint32_t*>(p->scratch[9].ptr), npolys, st);
    if (!rc) rc = cuda_status(cudaMemcpyAsync(out, dout, bytes, cudaMemcpyDeviceToHost, st));
    const int fin = finish_host_call(p, st);
    return rc ? rc : fin;
  }
  const uint32_t* ins[2] = {a, b};
  return host_pipeline(p, ins, 2, out, npolys, p->d, ntt_op_polymul, nullptr);
}

int grid_gpu_host_register(void* ptr, size_t bytes) {
  if (!ptr) return GRID_ERR_NULL_POINTER;
  return cuda_status(cudaHostRegister(ptr, bytes, cudaHostRegisterDefault));
}

int grid_gpu_host_unregister(void* ptr) {
  if (!ptr) return GRID_ERR_NULL_POINTER;
  return cuda_status(cudaHostUnregister(ptr));
}

}  // extern "C"
