// C ABI for prepared matrices, commitments, the Gram matrix, the JL
// projection, decompositions and the fused LaBRADOR prover round.
#include <cuda_runtime.h>

#include <cstring>
#include <new>

#include "grid_internal.h"

using namespace grid;

namespace {

bool aligned16(const void* p) { return ((uintptr_t)p & 15u) == 0; }

// The forward transform stores the evaluations of M x K witness polys
// point-major and the product with Y (N rows of row stride ldy) runs on the
// TMA-fed tensor-core kernel (emm_pm.cu).
bool pm_fits(const grid_gpu_plan* p, size_t M, size_t N, size_t K, size_t ldy, int mode) {
  EmmPmGeometry g;
  return ntt_tc_available(p) && emm_pm_geometry(p, (int)M, (int)N, (int)K, (int)ldy, mode, &g);
}

// Workspace layouts. On a ring plan without an NTT for q (is_crt) a call
// lifts its inputs into one residue buffer per auxiliary prime in turn (reused),
// keeps the three residue results, and runs the prime's own call in the rest of
// the workspace (reused across the primes); the reconstruction writes the output.
size_t commit_ws_bytes(const grid_gpu_plan* p, size_t rows, size_t cols, size_t batch) {
  if (is_crt(p))
    return words_bytes(batch * cols * p->d) + 3 * words_bytes(batch * rows * p->d) +
           commit_ws_bytes(p->crt[0], rows, cols, batch);
  return words_bytes(batch * cols * p->d) +
         words_bytes(emm_workspace_words(p, (int)batch, (int)rows, (int)cols, EMM_DENSE));
}

size_t gram_ws_bytes(const grid_gpu_plan* p, size_t r, size_t n) {
  const grid_gpu_plan* e = is_crt(p) ? p->crt[0] : p;
  const size_t base = words_bytes(r * n * p->d) +
                      words_bytes(emm_workspace_words(e, (int)r, (int)r, (int)n, EMM_UPPER));
  return is_crt(p) ? base + 3 * words_bytes(r * (r + 1) / 2 * p->d) : base;
}

size_t garbage_h_ws_bytes(const grid_gpu_plan* p, size_t r, size_t n) {
  const grid_gpu_plan* e = is_crt(p) ? p->crt[0] : p;
  const size_t base = 2 * words_bytes(r * n * p->d) + words_bytes(r * r * p->d) +
                      words_bytes(emm_workspace_words(e, (int)r, (int)r, (int)n, EMM_DENSE));
  return is_crt(p) ? base + 3 * words_bytes(r * r * p->d) : base;
}

size_t amortize_ws_bytes(const grid_gpu_plan* p, size_t r, size_t n) {
  const size_t base = words_bytes(r * n * p->d) + words_bytes(r * p->d);
  return is_crt(p) ? base + 3 * words_bytes(n * p->d) : base;
}

size_t round_ws_bytes(const grid_gpu_plan* p, size_t r, size_t n, size_t kappa, size_t jl_rows) {
  const grid_gpu_plan* e = is_crt(p) ? p->crt[0] : p;
  const size_t d = p->d;
  const size_t e1 = emm_workspace_words(e, (int)r, (int)kappa, (int)n, EMM_DENSE);
  const size_t e2 = emm_workspace_words(e, (int)r, (int)r, (int)n, EMM_UPPER);
  const size_t base = words_bytes(r * n * d) + words_bytes(e1 > e2 ? e1 : e2) +
                      words_bytes(r * kappa * d) +
                      round_up(jl_scratch_bytes(jl_rows ? jl_rows : 1, 0, 0), 256);
  return is_crt(p) ? base + 3 * (words_bytes(r * kappa * d) + words_bytes(r * (r + 1) / 2 * d))
                   : base;
}

// x mod p_j into dst (the j-th auxiliary prime only)
int lift_one(const grid_gpu_plan* p, int j, const uint32_t* x, size_t words, uint32_t* dst,
             cudaStream_t st) {
  return crt_lift(p, x, words, j == 0 ? dst : nullptr, j == 1 ? dst : nullptr,
                  j == 2 ? dst : nullptr, st);
}

bool dims_ok(size_t a, size_t b, size_t c) {
  // all kernels index rows/cols/K with int
  return a > 0 && b > 0 && c > 0 && a < (1u << 30) && b < (1u << 30) && c < (1u << 30);
}

// a * b * c words of 4 bytes stay far below SIZE_MAX (no wrap in any size sum).
bool words_fit(size_t a, size_t b, size_t c) {
  size_t x;
  return !__builtin_mul_overflow(a, b, &x) && !__builtin_mul_overflow(x, c, &x) &&
         x < (1ull << 56);
}

// r x n witness polys and the r x r products over them (Gram, garbage h, amortization).
bool square_dims_ok(const grid_gpu_plan* p, size_t r, size_t n) {
  return dims_ok(r, n, 1) && words_fit(r, n, p->d) && words_fit(r, r, p->d);
}

// t = A * s for `batch` vectors, into t (coefficients). ws from a Carver.
int commit_core(const grid_gpu_matrix* A, const uint32_t* s, size_t batch, uint32_t* t,
                Carver& cv, cudaStream_t st) {
  const grid_gpu_plan* p = A->plan;
  if (is_crt(p)) {
    if (!crt_bound_ok(p, A->cols)) return GRID_ERR_INVALID_PARAMETERS;
    const size_t sw = batch * A->cols * p->d, tw = batch * A->rows * p->d;
    uint32_t* sj = cv.take<uint32_t>(sw);
    uint32_t* tj[3] = {cv.take<uint32_t>(tw), cv.take<uint32_t>(tw), cv.take<uint32_t>(tw)};
    if (!cv.ok) return GRID_ERR_INVALID_PARAMETERS;
    const size_t mark = cv.used;
    for (int j = 0; j < 3; ++j) {
      int rc = lift_one(p, j, s, sw, sj, st);
      if (!rc) rc = commit_core(A->crt[j], sj, batch, tj[j], cv, st);
      if (rc) return rc;
      cv.used = mark;  // the next prime reuses the same workspace
    }
    return crt_combine(p, tj[0], tj[1], tj[2], tw, t, st);
  }
  if (commit_small_fits(p, A->rows, A->cols, batch))
    return launch_commit_small(p, A->d_evals, A->rows, A->cols, A->ld, s, batch, t, st);
  uint32_t* s_hat = cv.take<uint32_t>(batch * A->cols * p->d);
  const size_t ew = emm_workspace_words(p, (int)batch, (int)A->rows, (int)A->cols, EMM_DENSE);
  uint32_t* work = ew ? cv.take<uint32_t>(ew) : nullptr;
  if (!cv.ok) return GRID_ERR_INVALID_PARAMETERS;
  int rc;
  if (A->d_evals_pm && pm_fits(p, batch, A->rows, A->cols, A->ld, EMM_DENSE)) {
    rc = launch_ntt_tc(p, MODE_FWD_PM, s, nullptr, s_hat, batch * A->cols, st);
    if (!rc)
      rc = launch_emm_pm(p, s_hat, A->d_evals_pm, (int)batch, (int)A->rows, (int)A->cols,
                         (int)A->ld, EMM_DENSE, t, work, st);
  } else {
    rc = launch_ntt(p, MODE_FWD, s, nullptr, s_hat, batch * A->cols, st);
    if (!rc)
      rc = launch_emm(p, s_hat, A->d_evals, (int)batch, (int)A->rows, (int)A->cols, (int)A->ld,
                      EMM_DENSE, t, work, st);
  }
  if (rc) return rc;
  return launch_ntt(p, MODE_INV, t, nullptr, t, batch * A->rows, st);
}

}  // namespace

extern "C" {

/* ---- prepared matrices ------------------------------------------------- */

int grid_gpu_matrix_create_dev(grid_gpu_plan* p, const uint32_t* A, size_t rows, size_t cols,
                               int a_is_evals, grid_gpu_matrix** out, void* stream) {
  if (!p || !out || !A) return GRID_ERR_NULL_POINTER;
  *out = nullptr;
  if (!dims_ok(rows, cols, 1)) return GRID_ERR_INVALID_PARAMETERS;
  if (!aligned16(A)) return GRID_ERR_MISALIGNED;
  if (!words_fit(rows, cols, p->d)) return GRID_ERR_INVALID_PARAMETERS;
  if (is_crt(p) && a_is_evals) return p->ntt_status;  // q has no evaluation domain
  grid_gpu_matrix* m = new (std::nothrow) grid_gpu_matrix();
  if (!m) return GRID_ERR_OUT_OF_MEMORY;
  m->plan = p;
  m->rows = rows;
  m->cols = cols;
  m->ld = cols;
  cudaStream_t st = (cudaStream_t)stream;
  if (is_crt(p)) {
    // residues mod each auxiliary prime, prepared (transformed) on its plan
    const size_t words = rows * cols * p->d;
    int rc = GRID_OK;
    for (int j = 0; j < 3 && !rc; ++j) {
      grid_gpu_matrix* sub = new (std::nothrow) grid_gpu_matrix();
      if (!sub) {
        rc = GRID_ERR_OUT_OF_MEMORY;
        break;
      }
      m->crt[j] = sub;
      sub->plan = p->crt[j];
      sub->rows = rows;
      sub->cols = cols;
      sub->ld = cols;
      rc = cuda_status(cudaMalloc(&sub->d_evals, words * 4));
      if (!rc) rc = lift_one(p, j, A, words, sub->d_evals, st);
      if (!rc) rc = launch_ntt(sub->plan, MODE_FWD, sub->d_evals, nullptr, sub->d_evals,
                               rows * cols, st);
    }
    if (rc) {
      grid_gpu_matrix_destroy(m);
      return rc;
    }
    *out = m;
    return GRID_OK;
  }
  cudaError_t e = cudaMalloc(&m->d_evals, rows * cols * p->d * 4);
  if (e != cudaSuccess) {
    delete m;
    return cuda_status(e);
  }
  int rc;
  if (a_is_evals) {
    rc = cuda_status(cudaMemcpyAsync(m->d_evals, A, rows * cols * p->d * 4,
                                     cudaMemcpyDeviceToDevice, st));
  } else {
    rc = launch_ntt(p, MODE_FWD, A, nullptr, m->d_evals, rows * cols, st);
  }
  // a point-major copy for products on the TMA-fed tensor-core kernel
  EmmPmGeometry pg;
  if (!rc && ntt_tc_available(p) &&
      emm_pm_geometry(p, 1, (int)rows, (int)cols, (int)cols, EMM_DENSE, &pg)) {
    rc = cuda_status(cudaMalloc(&m->d_evals_pm, rows * cols * p->d * 4));
    if (!rc) rc = launch_to_point_major(m->d_evals, m->d_evals_pm, rows * cols, (int)p->d, st);
  }
  if (rc) {
    grid_gpu_matrix_destroy(m);
    return rc;
  }
  *out = m;
  return GRID_OK;
}

int grid_gpu_matrix_create(grid_gpu_plan* p, const uint32_t* A, size_t rows, size_t cols,
                           int a_is_evals, grid_gpu_matrix** out) {
  if (!p || !out || !A) return GRID_ERR_NULL_POINTER;
  *out = nullptr;
  if (!dims_ok(rows, cols, 1)) return GRID_ERR_INVALID_PARAMETERS;
  std::lock_guard<std::mutex> lk(p->mu);
  const size_t bytes = rows * cols * p->d * 4;
  int rc = ensure_scratch(p, 6, bytes);
  if (rc) return rc;
  rc = cuda_status(cudaMemcpyAsync(p->scratch[6].ptr, A, bytes, cudaMemcpyHostToDevice, p->stream));
  if (rc) return rc;
  rc = grid_gpu_matrix_create_dev(p, static_cast<uint32_t*>(p->scratch[6].ptr), rows, cols,
                                  a_is_evals, out, p->stream);
  const int fin = finish_host_call(p, p->stream);
  if (rc) return rc;
  if (fin && *out) {
    grid_gpu_matrix_destroy(*out);
    *out = nullptr;
  }
  return fin;
}

int grid_gpu_matrix_destroy(grid_gpu_matrix* m) {
  if (!m) return GRID_ERR_NULL_POINTER;
  for (grid_gpu_matrix* sub : m->crt)
    if (sub) grid_gpu_matrix_destroy(sub);
  if (m->owned && m->d_evals) cudaFree(m->d_evals);
  if (m->owned && m->d_evals_pm) cudaFree(m->d_evals_pm);
  delete m;
  return GRID_OK;
}

int grid_gpu_matrix_view(const grid_gpu_matrix* parent, size_t cols, grid_gpu_matrix** out) {
  if (!parent || !out) return GRID_ERR_NULL_POINTER;
  *out = nullptr;
  if (cols == 0 || cols > parent->cols) return GRID_ERR_DIMENSION_MISMATCH;
  grid_gpu_matrix* m = new (std::nothrow) grid_gpu_matrix();
  if (!m) return GRID_ERR_OUT_OF_MEMORY;
  m->plan = parent->plan;
  m->rows = parent->rows;
  m->cols = cols;
  m->ld = parent->ld;
  m->d_evals = parent->d_evals;
  m->d_evals_pm = parent->d_evals_pm;
  m->owned = false;
  for (int j = 0; j < 3; ++j)
    if (parent->crt[j]) {
      const int rc = grid_gpu_matrix_view(parent->crt[j], cols, &m->crt[j]);
      if (rc) {
        grid_gpu_matrix_destroy(m);
        return rc;
      }
    }
  *out = m;
  return GRID_OK;
}

int grid_gpu_matrix_shape(const grid_gpu_matrix* m, size_t* rows, size_t* cols) {
  if (!m || !rows || !cols) return GRID_ERR_NULL_POINTER;
  *rows = m->rows;
  *cols = m->cols;
  return GRID_OK;
}

int grid_gpu_matrix_device_evals(const grid_gpu_matrix* m, const uint32_t** evals) {
  if (!m || !evals) return GRID_ERR_NULL_POINTER;
  if (is_crt(m->plan)) return m->plan->ntt_status;  // no evaluation domain mod q
  *evals = m->d_evals;
  return GRID_OK;
}

/* ---- commitments ------------------------------------------------------- */

int grid_gpu_commit_workspace(const grid_gpu_matrix* A, size_t batch, size_t* bytes) {
  if (!A || !bytes) return GRID_ERR_NULL_POINTER;
  *bytes = commit_ws_bytes(A->plan, A->rows, A->cols, batch);
  return GRID_OK;
}

int grid_gpu_commit_dev(const grid_gpu_matrix* A, const uint32_t* s, size_t batch, uint32_t* t,
                        void* workspace, size_t workspace_bytes, void* stream) {
  if (!A || ((!s || !t) && batch)) return GRID_ERR_NULL_POINTER;
  if (batch == 0) return GRID_OK;
  if (!dims_ok(batch, A->rows, A->cols)) return GRID_ERR_INVALID_PARAMETERS;
  if (!aligned16(s) || !aligned16(t) || !aligned16(workspace)) return GRID_ERR_MISALIGNED;
  Carver cv(workspace, workspace_bytes);
  return commit_core(A, s, batch, t, cv, (cudaStream_t)stream);
}

int grid_gpu_commit(grid_gpu_matrix* A, const uint32_t* s, size_t batch, uint32_t* t) {
  if (!A || ((!s || !t) && batch)) return GRID_ERR_NULL_POINTER;
  if (batch == 0) return GRID_OK;
  if (!dims_ok(batch, A->rows, A->cols)) return GRID_ERR_INVALID_PARAMETERS;
  grid_gpu_plan* p = A->plan;
  std::lock_guard<std::mutex> lk(p->mu);
  const size_t s_bytes = batch * A->cols * p->d * 4, t_bytes = batch * A->rows * p->d * 4;
  const size_t ws = commit_ws_bytes(p, A->rows, A->cols, batch);
  int rc;
  if ((rc = ensure_scratch(p, 6, s_bytes)) || (rc = ensure_scratch(p, 7, t_bytes)) ||
      (rc = ensure_scratch(p, 8, ws)))
    return rc;
  cudaStream_t st = p->stream;
  rc = cuda_status(cudaMemcpyAsync(p->scratch[6].ptr, s, s_bytes, cudaMemcpyHostToDevice, st));
  if (!rc) {
    Carver cv(p->scratch[8].ptr, ws);
    rc = commit_core(A, static_cast<uint32_t*>(p->scratch[6].ptr), batch,
                     static_cast<uint32_t*>(p->scratch[7].ptr), cv, st);
  }
  if (!rc)
    rc = cuda_status(cudaMemcpyAsync(t, p->scratch[7].ptr, t_bytes, cudaMemcpyDeviceToHost, st));
  const int fin = finish_host_call(p, st);
  return rc ? rc : fin;
}

int grid_gpu_linear_commit_workspace(const grid_gpu_matrix* A_msg, const grid_gpu_matrix* A_open,
                                     size_t batch, size_t* bytes) {
  if (!A_msg || !A_open || !bytes) return GRID_ERR_NULL_POINTER;
  const grid_gpu_plan* p = A_msg->plan;
  *bytes = commit_ws_bytes(p, A_msg->rows, A_msg->cols, batch) +
           commit_ws_bytes(p, A_open->rows, A_open->cols, batch) +
           words_bytes(batch * A_open->rows * p->d);
  return GRID_OK;
}

int grid_gpu_linear_commit_dev(const grid_gpu_matrix* A_msg, const grid_gpu_matrix* A_open,
                               const uint32_t* m, const uint32_t* r, size_t batch, uint32_t* t,
                               void* workspace, size_t workspace_bytes, void* stream) {
  if (!A_msg || !A_open || ((!m || !r || !t) && batch)) return GRID_ERR_NULL_POINTER;
  if (A_msg->plan != A_open->plan) return GRID_ERR_INVALID_PARAMETERS;
  if (A_msg->rows != A_open->rows) return GRID_ERR_DIMENSION_MISMATCH;
  if (batch == 0) return GRID_OK;
  if (!dims_ok(batch, A_msg->rows, A_msg->cols) || !dims_ok(batch, A_open->rows, A_open->cols))
    return GRID_ERR_INVALID_PARAMETERS;
  if (!aligned16(m) || !aligned16(r) || !aligned16(t) || !aligned16(workspace))
    return GRID_ERR_MISALIGNED;
  const grid_gpu_plan* p = A_msg->plan;
  cudaStream_t st = (cudaStream_t)stream;
  Carver cv(workspace, workspace_bytes);
  uint32_t* t2 = cv.take<uint32_t>(batch * A_open->rows * p->d);
  if (!cv.ok) return GRID_ERR_INVALID_PARAMETERS;
  int rc = commit_core(A_msg, m, batch, t, cv, st);
  if (!rc) rc = commit_core(A_open, r, batch, t2, cv, st);
  // A_msg*m + A_open*r: INTT is linear, so adding the coefficient forms is exact.
  if (!rc) rc = launch_add(p, t, t2, batch * A_open->rows * p->d, st);
  return rc;
}

int grid_gpu_linear_commit(grid_gpu_matrix* A_msg, grid_gpu_matrix* A_open, const uint32_t* m,
                           const uint32_t* r, size_t batch, uint32_t* t) {
  if (!A_msg || !A_open || ((!m || !r || !t) && batch)) return GRID_ERR_NULL_POINTER;
  if (A_msg->plan != A_open->plan) return GRID_ERR_INVALID_PARAMETERS;
  if (A_msg->rows != A_open->rows) return GRID_ERR_DIMENSION_MISMATCH;
  if (batch == 0) return GRID_OK;
  grid_gpu_plan* p = A_msg->plan;
  std::lock_guard<std::mutex> lk(p->mu);
  const size_t rows = A_msg->rows, d = p->d;
  const size_t m_bytes = batch * A_msg->cols * d * 4, r_bytes = batch * A_open->cols * d * 4;
  const size_t t_bytes = batch * rows * d * 4;
  const size_t ws = commit_ws_bytes(p, rows, A_msg->cols, batch) +
                    commit_ws_bytes(p, rows, A_open->cols, batch);
  int rc;
  if ((rc = ensure_scratch(p, 6, m_bytes)) || (rc = ensure_scratch(p, 7, r_bytes)) ||
      (rc = ensure_scratch(p, 9, t_bytes)) || (rc = ensure_scratch(p, 10, t_bytes)) ||
      (rc = ensure_scratch(p, 8, ws)))
    return rc;
  cudaStream_t st = p->stream;
  uint32_t* dm = static_cast<uint32_t*>(p->scratch[6].ptr);
  uint32_t* dr = static_cast<uint32_t*>(p->scratch[7].ptr);
  uint32_t* t1 = static_cast<uint32_t*>(p->scratch[9].ptr);
  uint32_t* t2 = static_cast<uint32_t*>(p->scratch[10].ptr);
  rc = cuda_status(cudaMemcpyAsync(dm, m, m_bytes, cudaMemcpyHostToDevice, st));
  if (!rc) rc = cuda_status(cudaMemcpyAsync(dr, r, r_bytes, cudaMemcpyHostToDevice, st));
  if (!rc) {
    Carver cv(p->scratch[8].ptr, ws);
    rc = commit_core(A_msg, dm, batch, t1, cv, st);
    if (!rc) rc = commit_core(A_open, dr, batch, t2, cv, st);
  }
  // A_msg*m + A_open*r: INTT is linear, so adding the coefficient forms is exact.
  if (!rc) rc = launch_add(p, t1, t2, batch * rows * d, st);
  if (!rc) rc = cuda_status(cudaMemcpyAsync(t, t1, t_bytes, cudaMemcpyDeviceToHost, st));
  const int fin = finish_host_call(p, st);
  return rc ? rc : fin;
}

/* ---- BDLOP parts: u = A_mask * r, v = A_msg * m + A_open * r ---------- */

int grid_gpu_bdlop_workspace(const grid_gpu_matrix* A_mask, const grid_gpu_matrix* A_msg,
                             const grid_gpu_matrix* A_open, size_t batch, size_t* bytes) {
  if (!A_mask || !A_msg || !A_open || !bytes) return GRID_ERR_NULL_POINTER;
  const grid_gpu_plan* p = A_msg->plan;
  *bytes = commit_ws_bytes(p, A_mask->rows, A_mask->cols, batch) +
           commit_ws_bytes(p, A_msg->rows, A_msg->cols, batch) +
           commit_ws_bytes(p, A_open->rows, A_open->cols, batch) +
           words_bytes(batch * A_open->rows * p->d);
  return GRID_OK;
}

int grid_gpu_bdlop_commit_dev(const grid_gpu_matrix* A_mask, const grid_gpu_matrix* A_msg,
                              const grid_gpu_matrix* A_open, const uint32_t* m, const uint32_t* r,
                              size_t batch, uint32_t* u, uint32_t* v, void* workspace,
                              size_t workspace_bytes, void* stream) {
  if (!A_mask || !A_msg || !A_open || ((!m || !r || !u || !v) && batch))
    return GRID_ERR_NULL_POINTER;
  if (A_mask->plan != A_msg->plan || A_open->plan != A_msg->plan)
    return GRID_ERR_INVALID_PARAMETERS;
  // the mask and the opening part multiply the same randomness
  if (A_msg->rows != A_open->rows || A_mask->cols != A_open->cols)
    return GRID_ERR_DIMENSION_MISMATCH;
  if (batch == 0) return GRID_OK;
  if (!dims_ok(batch, A_msg->rows, A_msg->cols) || !dims_ok(batch, A_mask->rows, A_mask->cols))
    return GRID_ERR_INVALID_PARAMETERS;
  if (!aligned16(m) || !aligned16(r) || !aligned16(u) || !aligned16(v) || !aligned16(workspace))
    return GRID_ERR_MISALIGNED;
  const grid_gpu_plan* p = A_msg->plan;
  cudaStream_t st = (cudaStream_t)stream;
  Carver cv(workspace, workspace_bytes);
  uint32_t* t2 = cv.take<uint32_t>(batch * A_open->rows * p->d);
  if (!cv.ok) return GRID_ERR_INVALID_PARAMETERS;
  int rc = commit_core(A_mask, r, batch, u, cv, st);
  if (!rc) rc = commit_core(A_msg, m, batch, v, cv, st);
  if (!rc) rc = commit_core(A_open, r, batch, t2, cv, st);
  // A_msg*m + A_open*r: INTT is linear, so adding the coefficient forms is exact.
  if (!rc) rc = launch_add(p, v, t2, batch * A_open->rows * p->d, st);
  return rc;
}

int grid_gpu_bdlop_commit(grid_gpu_matrix* A_mask, grid_gpu_matrix* A_msg, grid_gpu_matrix* A_open,
                          const uint32_t* m, const uint32_t* r, size_t batch, uint32_t* u,
                          uint32_t* v) {
  if (!A_mask || !A_msg || !A_open || ((!m || !r || !u || !v) && batch))
    return GRID_ERR_NULL_POINTER;
  if (A_mask->plan != A_msg->plan || A_open->plan != A_msg->plan)
    return GRID_ERR_INVALID_PARAMETERS;
  if (A_msg->rows != A_open->rows || A_mask->cols != A_open->cols)
    return GRID_ERR_DIMENSION_MISMATCH;
  if (batch == 0) return GRID_OK;
  grid_gpu_plan* p = A_msg->plan;
  std::lock_guard<std::mutex> lk(p->mu);
  const size_t d = p->d;
  const size_t m_bytes = batch * A_msg->cols * d * 4, r_bytes = batch * A_open->cols * d * 4;
  const size_t u_bytes = batch * A_mask->rows * d * 4, v_bytes = batch * A_msg->rows * d * 4;
  size_t ws = 0;
  int rc = grid_gpu_bdlop_workspace(A_mask, A_msg, A_open, batch, &ws);
  if (rc || (rc = ensure_scratch(p, 6, m_bytes)) || (rc = ensure_scratch(p, 7, r_bytes)) ||
      (rc = ensure_scratch(p, 9, v_bytes)) || (rc = ensure_scratch(p, 10, u_bytes)) ||
      (rc = ensure_scratch(p, 8, ws)))
    return rc;
  cudaStream_t st = p->stream;
  rc = cuda_status(cudaMemcpyAsync(p->scratch[6].ptr, m, m_bytes, cudaMemcpyHostToDevice, st));
  if (!rc)
    rc = cuda_status(cudaMemcpyAsync(p->scratch[7].ptr, r, r_bytes, cudaMemcpyHostToDevice, st));
  if (!rc)
    rc = grid_gpu_bdlop_commit_dev(A_mask, A_msg, A_open,
                                   static_cast<uint32_t*>(p->scratch[6].ptr),
                                   static_cast<uint32_t*>(p->scratch[7].ptr), batch,
                                   static_cast<uint32_t*>(p->scratch[10].ptr),
                                   static_cast<uint32_t*>(p->scratch[9].ptr), p->scratch[8].ptr,
                                   ws, st);
  if (!rc)
    rc = cuda_status(cudaMemcpyAsync(u, p->scratch[10].ptr, u_bytes, cudaMemcpyDeviceToHost, st));
  if (!rc)
    rc = cuda_status(cudaMemcpyAsync(v, p->scratch[9].ptr, v_bytes, cudaMemcpyDeviceToHost, st));
  const int fin = finish_host_call(p, st);
  return rc ? rc : fin;
}

/* ---- Gram matrix (garbage g) ------------------------------------------- */

int grid_gpu_gram_workspace(const grid_gpu_plan* p, size_t r, size_t n, size_t* bytes) {
  if (!p || !bytes) return GRID_ERR_NULL_POINTER;
  if (!square_dims_ok(p, r, n)) return GRID_ERR_INVALID_PARAMETERS;
  *bytes = gram_ws_bytes(p, r, n);
  return GRID_OK;
}

int grid_gpu_gram_dev(const grid_gpu_plan* p, const uint32_t* S, size_t r, size_t n,
                      uint32_t* G, void* workspace, size_t workspace_bytes, void* stream) {
  if (!p || !S || !G) return GRID_ERR_NULL_POINTER;
  if (!square_dims_ok(p, r, n)) return GRID_ERR_INVALID_PARAMETERS;
  if (!aligned16(S) || !aligned16(G) || !aligned16(workspace)) return GRID_ERR_MISALIGNED;
  cudaStream_t st = (cudaStream_t)stream;
  if (is_crt(p) && !crt_bound_ok(p, n)) return GRID_ERR_INVALID_PARAMETERS;
  const grid_gpu_plan* e = is_crt(p) ? p->crt[0] : p;
  const size_t gw = r * (r + 1) / 2 * p->d;
  Carver cv(workspace, workspace_bytes);
  uint32_t* s_hat = cv.take<uint32_t>(r * n * p->d);
  const size_t ew = emm_workspace_words(e, (int)r, (int)r, (int)n, EMM_UPPER);
  uint32_t* work = ew ? cv.take<uint32_t>(ew) : nullptr;
  uint32_t* gj[3] = {};
  if (is_crt(p))
    for (auto& x : gj) x = cv.take<uint32_t>(gw);
  if (!cv.ok) return GRID_ERR_INVALID_PARAMETERS;
  int rc = GRID_OK;
  for (int j = 0; j < (is_crt(p) ? 3 : 1) && !rc; ++j) {
    const grid_gpu_plan* q = is_crt(p) ? p->crt[j] : p;
    uint32_t* out = is_crt(p) ? gj[j] : G;
    if (is_crt(p)) {
      rc = lift_one(p, j, S, r * n * p->d, s_hat, st);
      if (!rc) rc = launch_ntt(q, MODE_FWD, s_hat, nullptr, s_hat, r * n, st);
    } else if (pm_fits(q, r, r, n, n, EMM_UPPER)) {
      rc = launch_ntt_tc(q, MODE_FWD_PM, S, nullptr, s_hat, r * n, st);
      if (!rc)
        rc = launch_emm_pm(q, s_hat, s_hat, (int)r, (int)r, (int)n, (int)n, EMM_UPPER, out, work,
                           st);
      if (!rc) rc = launch_ntt(q, MODE_INV, out, nullptr, out, r * (r + 1) / 2, st);
      continue;
    } else {
      rc = launch_ntt(q, MODE_FWD, S, nullptr, s_hat, r * n, st);
    }
    if (!rc)
      rc = launch_emm(q, s_hat, s_hat, (int)r, (int)r, (int)n, (int)n, EMM_UPPER, out, work, st);
    if (!rc) rc = launch_ntt(q, MODE_INV, out, nullptr, out, r * (r + 1) / 2, st);
  }
  if (!rc && is_crt(p)) rc = crt_combine(p, gj[0], gj[1], gj[2], gw, G, st);
  return rc;
}

int grid_gpu_gram(grid_gpu_plan* p, const uint32_t* S, size_t r, size_t n, uint32_t* G) {
  if (!p || !S || !G) return GRID_ERR_NULL_POINTER;
  if (!square_dims_ok(p, r, n)) return GRID_ERR_INVALID_PARAMETERS;
  std::lock_guard<std::mutex> lk(p->mu);
  const size_t s_bytes = r * n * p->d * 4, g_bytes = r * (r + 1) / 2 * p->d * 4;
  const size_t ws = gram_ws_bytes(p, r, n);
  int rc;
  if ((rc = ensure_scratch(p, 6, s_bytes)) || (rc = ensure_scratch(p, 7, g_bytes)) ||
      (rc = ensure_scratch(p, 8, ws)))
    return rc;
  cudaStream_t st = p->stream;
  rc = cuda_status(cudaMemcpyAsync(p->scratch[6].ptr, S, s_bytes, cudaMemcpyHostToDevice, st));
  if (!rc)
    rc = grid_gpu_gram_dev(p, static_cast<uint32_t*>(p->scratch[6].ptr), r, n,
                           static_cast<uint32_t*>(p->scratch[7].ptr), p->scratch[8].ptr, ws, st);
  if (!rc)
    rc = cuda_status(cudaMemcpyAsync(G, p->scratch[7].ptr, g_bytes, cudaMemcpyDeviceToHost, st));
  const int fin = finish_host_call(p, st);
  return rc ? rc : fin;
}

/* ---- garbage h and the amortized witness -------------------------------- */

int grid_gpu_garbage_h_workspace(const grid_gpu_plan* p, size_t r, size_t n, size_t* bytes) {
  if (!p || !bytes) return GRID_ERR_NULL_POINTER;
  if (!square_dims_ok(p, r, n)) return GRID_ERR_INVALID_PARAMETERS;
  *bytes = garbage_h_ws_bytes(p, r, n);
  return GRID_OK;
}

int grid_gpu_garbage_h_dev(const grid_gpu_plan* p, const uint32_t* S, const uint32_t* Phi,
                           size_t r, size_t n, uint32_t* H, void* workspace,
                           size_t workspace_bytes, void* stream) {
  if (!p || !S || !Phi || !H) return GRID_ERR_NULL_POINTER;
  if (!square_dims_ok(p, r, n)) return GRID_ERR_INVALID_PARAMETERS;
  if (!aligned16(S) || !aligned16(Phi) || !aligned16(H) || !aligned16(workspace))
    return GRID_ERR_MISALIGNED;
  cudaStream_t st = (cudaStream_t)stream;
  Carver cv(workspace, workspace_bytes);
  uint32_t* s_hat = cv.take<uint32_t>(r * n * p->d);
  uint32_t* phi_hat = cv.take<uint32_t>(r * n * p->d);
  uint32_t* cross = cv.take<uint32_t>(r * r * p->d);
  const grid_gpu_plan* e = is_crt(p) ? p->crt[0] : p;
  const size_t ew = emm_workspace_words(e, (int)r, (int)r, (int)n, EMM_DENSE);
  uint32_t* work = ew ? cv.take<uint32_t>(ew) : nullptr;
  if (!is_crt(p)) {
    if (!cv.ok) return GRID_ERR_INVALID_PARAMETERS;
    // cross[i][j] = <phi_i, s_j>
    const bool pm = pm_fits(p, r, r, n, n, EMM_DENSE);
    const int fwd = pm ? MODE_FWD_PM : MODE_FWD;
    int rc = pm ? launch_ntt_tc(p, fwd, S, nullptr, s_hat, r * n, st)
                : launch_ntt(p, fwd, S, nullptr, s_hat, r * n, st);
    if (!rc)
      rc = pm ? launch_ntt_tc(p, fwd, Phi, nullptr, phi_hat, r * n, st)
              : launch_ntt(p, fwd, Phi, nullptr, phi_hat, r * n, st);
    if (!rc)
      rc = pm ? launch_emm_pm(p, phi_hat, s_hat, (int)r, (int)r, (int)n, (int)n, EMM_DENSE, cross,
                              work, st)
              : launch_emm(p, phi_hat, s_hat, (int)r, (int)r, (int)n, (int)n, EMM_DENSE, cross,
                           work, st);
    if (!rc) rc = launch_symmetrize_half(p, cross, (int)r, H, st);
    if (rc) return rc;
    return launch_ntt(p, MODE_INV, H, nullptr, H, r * (r + 1) / 2, st);
  }
  // ring plan without an NTT for q: the cross products per auxiliary prime,
  // back to coefficients, reconstructed mod q; then the (linear) symmetrisation
  if (!crt_bound_ok(p, n)) return GRID_ERR_INVALID_PARAMETERS;
  const size_t cw = r * r * p->d;
  uint32_t* cj[3] = {cv.take<uint32_t>(cw), cv.take<uint32_t>(cw), cv.take<uint32_t>(cw)};
  if (!cv.ok) return GRID_ERR_INVALID_PARAMETERS;
  int rc = GRID_OK;
  for (int j = 0; j < 3 && !rc; ++j) {
    const grid_gpu_plan* q = p->crt[j];
    rc = lift_one(p, j, S, r * n * p->d, s_hat, st);
    if (!rc) rc = lift_one(p, j, Phi, r * n * p->d, phi_hat, st);
    if (!rc) rc = launch_ntt(q, MODE_FWD, s_hat, nullptr, s_hat, r * n, st);
    if (!rc) rc = launch_ntt(q, MODE_FWD, phi_hat, nullptr, phi_hat, r * n, st);
    if (!rc)
      rc = launch_emm(q, phi_hat, s_hat, (int)r, (int)r, (int)n, (int)n, EMM_DENSE, cj[j], work,
                      st);
    if (!rc) rc = launch_ntt(q, MODE_INV, cj[j], nullptr, cj[j], r * r, st);
  }
  if (!rc) rc = crt_combine(p, cj[0], cj[1], cj[2], cw, cross, st);
  if (!rc) rc = launch_symmetrize_half(p, cross, (int)r, H, st);
  return rc;
}

int grid_gpu_garbage_h(grid_gpu_plan* p, const uint32_t* S, const uint32_t* Phi, size_t r,
                       size_t n, uint32_t* H) {
  if (!p || !S || !Phi || !H) return GRID_ERR_NULL_POINTER;
  if (!square_dims_ok(p, r, n)) return GRID_ERR_INVALID_PARAMETERS;
  std::lock_guard<std::mutex> lk(p->mu);
  const size_t s_bytes = r * n * p->d * 4, h_bytes = r * (r + 1) / 2 * p->d * 4;
  const size_t ws = garbage_h_ws_bytes(p, r, n);
  int rc;
  if ((rc = ensure_scratch(p, 6, s_bytes)) || (rc = ensure_scratch(p, 9, s_bytes)) ||
      (rc = ensure_scratch(p, 7, h_bytes)) || (rc = ensure_scratch(p, 8, ws)))
    return rc;
  cudaStream_t st = p->stream;
  rc = cuda_status(cudaMemcpyAsync(p->scratch[6].ptr, S, s_bytes, cudaMemcpyHostToDevice, st));
  if (!rc)
    rc = cuda_status(cudaMemcpyAsync(p->scratch[9].ptr, Phi, s_bytes, cudaMemcpyHostToDevice, st));
  if (!rc)
    rc = grid_gpu_garbage_h_dev(p, static_cast<uint32_t*>(p->scratch[6].ptr),
                                static_cast<uint32_t*>(p->scratch[9].ptr), r, n,
                                static_cast<uint32_t*>(p->scratch[7].ptr), p->scratch[8].ptr, ws,
                                st);
  if (!rc)
    rc = cuda_status(cudaMemcpyAsync(H, p->scratch[7].ptr, h_bytes, cudaMemcpyDeviceToHost, st));
  const int fin = finish_host_call(p, st);
  return rc ? rc : fin;
}

int grid_gpu_amortize_workspace(const grid_gpu_plan* p, size_t r, size_t n, size_t* bytes) {
  if (!p || !bytes) return GRID_ERR_NULL_POINTER;
  if (!square_dims_ok(p, r, n)) return GRID_ERR_INVALID_PARAMETERS;
  *bytes = amortize_ws_bytes(p, r, n);
  return GRID_OK;
}

int grid_gpu_amortize_dev(const grid_gpu_plan* p, const uint32_t* S, const uint32_t* c, size_t r,
                          size_t n, uint32_t* z, void* workspace, size_t workspace_bytes,
                          void* stream) {
  if (!p || !S || !c || !z) return GRID_ERR_NULL_POINTER;
  if (!square_dims_ok(p, r, n)) return GRID_ERR_INVALID_PARAMETERS;
  if (!aligned16(S) || !aligned16(c) || !aligned16(z) || !aligned16(workspace))
    return GRID_ERR_MISALIGNED;
  cudaStream_t st = (cudaStream_t)stream;
  Carver cv(workspace, workspace_bytes);
  uint32_t* s_hat = cv.take<uint32_t>(r * n * p->d);
  uint32_t* c_hat = cv.take<uint32_t>(r * p->d);
  if (!is_crt(p)) {
    if (!cv.ok) return GRID_ERR_INVALID_PARAMETERS;
    int rc = launch_ntt(p, MODE_FWD, S, nullptr, s_hat, r * n, st);
    if (!rc) rc = launch_ntt(p, MODE_FWD, c, nullptr, c_hat, r, st);
    if (!rc) rc = launch_amortize(p, c_hat, s_hat, (int)r, n, z, st);
    if (rc) return rc;
    return launch_ntt(p, MODE_INV, z, nullptr, z, n, st);
  }
  // ring plan without an NTT for q: z[k] = sum_i c_i s_i[k] sums r * d products
  if (!crt_bound_ok(p, r)) return GRID_ERR_INVALID_PARAMETERS;
  const size_t zw = n * p->d;
  uint32_t* zj[3] = {cv.take<uint32_t>(zw), cv.take<uint32_t>(zw), cv.take<uint32_t>(zw)};
  if (!cv.ok) return GRID_ERR_INVALID_PARAMETERS;
  int rc = GRID_OK;
  for (int j = 0; j < 3 && !rc; ++j) {
    const grid_gpu_plan* q = p->crt[j];
    rc = lift_one(p, j, S, r * n * p->d, s_hat, st);
    if (!rc) rc = lift_one(p, j, c, r * p->d, c_hat, st);
    if (!rc) rc = launch_ntt(q, MODE_FWD, s_hat, nullptr, s_hat, r * n, st);
    if (!rc) rc = launch_ntt(q, MODE_FWD, c_hat, nullptr, c_hat, r, st);
    if (!rc) rc = launch_amortize(q, c_hat, s_hat, (int)r, n, zj[j], st);
    if (!rc) rc = launch_ntt(q, MODE_INV, zj[j], nullptr, zj[j], n, st);
  }
  if (rc) return rc;
  return crt_combine(p, zj[0], zj[1], zj[2], zw, z, st);
}

int grid_gpu_amortize(grid_gpu_plan* p, const uint32_t* S, const uint32_t* c, size_t r, size_t n,
                      uint32_t* z) {
  if (!p || !S || !c || !z) return GRID_ERR_NULL_POINTER;
  if (!square_dims_ok(p, r, n)) return GRID_ERR_INVALID_PARAMETERS;
  std::lock_guard<std::mutex> lk(p->mu);
  const size_t s_bytes = r * n * p->d * 4, c_bytes = r * p->d * 4, z_bytes = n * p->d * 4;
  const size_t ws = amortize_ws_bytes(p, r, n);
  int rc;
  if ((rc = ensure_scratch(p, 6, s_bytes)) || (rc = ensure_scratch(p, 9, c_bytes)) ||
      (rc = ensure_scratch(p, 7, z_bytes)) || (rc = ensure_scratch(p, 8, ws)))
    return rc;
  cudaStream_t st = p->stream;
  rc = cuda_status(cudaMemcpyAsync(p->scratch[6].ptr, S, s_bytes, cudaMemcpyHostToDevice, st));
  if (!rc)
    rc = cuda_status(cudaMemcpyAsync(p->scratch[9].ptr, c, c_bytes, cudaMemcpyHostToDevice, st));
  if (!rc)
    rc = grid_gpu_amortize_dev(p, static_cast<uint32_t*>(p->scratch[6].ptr),
                               static_cast<uint32_t*>(p->scratch[9].ptr), r, n,
                               static_cast<uint32_t*>(p->scratch[7].ptr), p->scratch[8].ptr, ws,
                               st);
  if (!rc)
    rc = cuda_status(cudaMemcpyAsync(z, p->scratch[7].ptr, z_bytes, cudaMemcpyDeviceToHost, st));
  const int fin = finish_host_call(p, st);
  return rc ? rc : fin;
}

/* ---- JL projection ------------------------------------------------------ */

int grid_gpu_jl_workspace(size_t rows, size_t* bytes) {
  if (!bytes) return GRID_ERR_NULL_POINTER;
  *bytes = round_up(jl_scratch_bytes(rows, 0, 0), 256);
  return GRID_OK;
}

int grid_gpu_jl_project_dev(const grid_gpu_plan* p, const uint8_t* seed, size_t rows,
                            const uint32_t* parts, size_t num_parts, size_t cols, size_t d,
                            uint32_t* p_out, int8_t* flat_out, void* workspace,
                            size_t workspace_bytes, void* stream) {
  if (!p || !seed || !p_out || (!parts && cols && num_parts)) return GRID_ERR_NULL_POINTER;
  if (!aligned16(workspace)) return GRID_ERR_MISALIGNED;
  return launch_jl_project(p->f, seed, rows, parts, num_parts, cols, d, p_out, flat_out,
                           workspace, workspace_bytes, p->num_sms, p->d_err, (cudaStream_t)stream);
}

int grid_gpu_jl_project(grid_gpu_plan* p, const uint8_t* seed, size_t rows,
                        const uint32_t* parts, size_t num_parts, size_t cols, size_t d,
                        uint32_t* p_out, int8_t* flat_out) {
  if (!p || !seed || !p_out || (!parts && cols && num_parts)) return GRID_ERR_NULL_POINTER;
  if (rows == 0 || rows > 256 || d == 0 || cols % d) return GRID_ERR_INVALID_PARAMETERS;
  std::lock_guard<std::mutex> lk(p->mu);
  const size_t in_bytes = num_parts * cols * 4, flat_bytes = flat_out ? rows * num_parts * cols : 0;
  const size_t ws = round_up(jl_scratch_bytes(rows, 0, 0), 256);
  int rc;
  if ((rc = ensure_scratch(p, 6, in_bytes ? in_bytes : 16)) ||
      (rc = ensure_scratch(p, 7, rows * 4)) || (rc = ensure_scratch(p, 8, ws)) ||
      (flat_bytes && (rc = ensure_scratch(p, 11, flat_bytes))))
    return rc;
  cudaStream_t st = p->stream;
  if (in_bytes)
    rc = cuda_status(cudaMemcpyAsync(p->scratch[6].ptr, parts, in_bytes, cudaMemcpyHostToDevice, st));
  if (!rc)
    rc = launch_jl_project(p->f, seed, rows, static_cast<uint32_t*>(p->scratch[6].ptr), num_parts,
                           cols, d, static_cast<uint32_t*>(p->scratch[7].ptr),
                           flat_bytes ? static_cast<int8_t*>(p->scratch[11].ptr) : nullptr,
                           p->scratch[8].ptr, ws, p->num_sms, p->d_err, st);
  if (!rc)
    rc = cuda_status(cudaMemcpyAsync(p_out, p->scratch[7].ptr, rows * 4, cudaMemcpyDeviceToHost, st));
  if (!rc && flat_bytes)
    rc = cuda_status(cudaMemcpyAsync(flat_out, p->scratch[11].ptr, flat_bytes,
                                     cudaMemcpyDeviceToHost, st));
  const int fin = finish_host_call(p, st);
  return rc ? rc : fin;
}

/* ---- JL evaluations (aggregation side) --------------------------------- */

int grid_gpu_jl_evals_workspace(size_t* bytes) {
  if (!bytes) return GRID_ERR_NULL_POINTER;
  *bytes = round_up(jl_evals_scratch_bytes(), 256);
  return GRID_OK;
}

int grid_gpu_jl_evals_dev(const grid_gpu_plan* p, const uint8_t* seed, size_t rows,
                          const uint32_t* parts, size_t num_parts, size_t cols, size_t d,
                          uint32_t* evals, void* workspace, size_t workspace_bytes, void* stream) {
  if (!p || !seed || !evals || !parts) return GRID_ERR_NULL_POINTER;
  if (d != p->d) return GRID_ERR_INVALID_PARAMETERS;
  if (!aligned16(workspace)) return GRID_ERR_MISALIGNED;
  return launch_jl_evals(p->f, seed, rows, parts, num_parts, cols, d, evals, workspace,
                         workspace_bytes, p->num_sms, p->d_err, (cudaStream_t)stream);
}

int grid_gpu_jl_evals(grid_gpu_plan* p, const uint8_t* seed, size_t rows, const uint32_t* parts,
                      size_t num_parts, size_t cols, size_t d, uint32_t* evals) {
  if (!p || !seed || !evals || !parts) return GRID_ERR_NULL_POINTER;
  if (d != p->d || d == 0 || cols == 0 || cols % d || num_parts == 0)
    return GRID_ERR_INVALID_PARAMETERS;
  std::lock_guard<std::mutex> lk(p->mu);
  const size_t in_bytes = num_parts * cols * 4, out_bytes = rows * d * 4;
  const size_t ws = round_up(jl_evals_scratch_bytes(), 256);
  int rc;
  if ((rc = ensure_scratch(p, 6, in_bytes)) || (rc = ensure_scratch(p, 7, out_bytes)) ||
      (rc = ensure_scratch(p, 8, ws)))
    return rc;
  cudaStream_t st = p->stream;
  rc = cuda_status(cudaMemcpyAsync(p->scratch[6].ptr, parts, in_bytes, cudaMemcpyHostToDevice, st));
  if (!rc)
    rc = launch_jl_evals(p->f, seed, rows, static_cast<uint32_t*>(p->scratch[6].ptr), num_parts,
                         cols, d, static_cast<uint32_t*>(p->scratch[7].ptr), p->scratch[8].ptr, ws,
                         p->num_sms, p->d_err, st);
  if (!rc)
    rc = cuda_status(cudaMemcpyAsync(evals, p->scratch[7].ptr, out_bytes, cudaMemcpyDeviceToHost, st));
  const int fin = finish_host_call(p, st);
  return rc ? rc : fin;
}

/* ---- uniform ring elements (seeded commitment-key expansion) ----------- */

int grid_gpu_sample_uniform_polys_workspace(const grid_gpu_plan* p, size_t npolys,
                                            uint64_t accept_max, size_t* bytes) {
  if (!p || !bytes) return GRID_ERR_NULL_POINTER;
  *bytes = round_up(sample_uniform_workspace_bytes(p->f.q, (unsigned long long)npolys * p->d,
                                                   accept_max),
                    256);
  return GRID_OK;
}

int grid_gpu_sample_uniform_polys_dev(const grid_gpu_plan* p, const uint8_t* seed, size_t npolys,
                                      uint64_t accept_max, uint32_t* out, void* workspace,
                                      size_t workspace_bytes, void* stream) {
  if (!p || !seed || (!out && npolys)) return GRID_ERR_NULL_POINTER;
  if (!aligned16(workspace)) return GRID_ERR_MISALIGNED;
  return launch_sample_uniform(p, seed, (unsigned long long)npolys * p->d, accept_max, out,
                               workspace, workspace_bytes, (cudaStream_t)stream);
}

int grid_gpu_sample_uniform_polys(grid_gpu_plan* p, const uint8_t* seed, size_t npolys,
                                  uint64_t accept_max, uint32_t* out) {
  if (!p || !seed || (!out && npolys)) return GRID_ERR_NULL_POINTER;
  if (npolys == 0) return GRID_OK;
  std::lock_guard<std::mutex> lk(p->mu);
  const size_t out_bytes = npolys * p->d * 4;
  const size_t ws = round_up(
      sample_uniform_workspace_bytes(p->f.q, (unsigned long long)npolys * p->d, accept_max), 256);
  int rc;
  if ((rc = ensure_scratch(p, 7, out_bytes)) || (rc = ensure_scratch(p, 8, ws))) return rc;
  cudaStream_t st = p->stream;
  rc = launch_sample_uniform(p, seed, (unsigned long long)npolys * p->d, accept_max,
                             static_cast<uint32_t*>(p->scratch[7].ptr), p->scratch[8].ptr, ws, st);
  if (!rc)
    rc = cuda_status(cudaMemcpyAsync(out, p->scratch[7].ptr, out_bytes, cudaMemcpyDeviceToHost, st));
  const int fin = finish_host_call(p, st);
  return rc ? rc : fin;
}

/* ---- decompositions ---------------------------------------------------- */

int grid_gpu_decompose_balanced_dev(const grid_gpu_plan* p, const uint32_t* polys, size_t npolys,
                                    uint64_t base, size_t num_limbs, uint32_t* out, void* stream) {
  if (!p || ((!polys || !out) && npolys)) return GRID_ERR_NULL_POINTER;
  return launch_decompose_balanced(p, polys, npolys, base, num_limbs, out, (cudaStream_t)stream);
}

int grid_gpu_decompose_balanced(grid_gpu_plan* p, const uint32_t* polys, size_t npolys,
                                uint64_t base, size_t num_limbs, uint32_t* out) {
  if (!p || ((!polys || !out) && npolys)) return GRID_ERR_NULL_POINTER;
  if (base < 2 || num_limbs == 0 || num_limbs > 64) return GRID_ERR_INVALID_PARAMETERS;
  if (npolys == 0) return GRID_OK;
  std::lock_guard<std::mutex> lk(p->mu);
  const size_t in_bytes = npolys * p->d * 4, out_bytes = in_bytes * num_limbs;
  int rc;
  if ((rc = ensure_scratch(p, 6, in_bytes)) || (rc = ensure_scratch(p, 7, out_bytes))) return rc;
  cudaStream_t st = p->stream;
  rc = cuda_status(cudaMemcpyAsync(p->scratch[6].ptr, polys, in_bytes, cudaMemcpyHostToDevice, st));
  if (!rc)
    rc = launch_decompose_balanced(p, static_cast<uint32_t*>(p->scratch[6].ptr), npolys, base,
                                   num_limbs, static_cast<uint32_t*>(p->scratch[7].ptr), st);
  if (!rc)
    rc = cuda_status(cudaMemcpyAsync(out, p->scratch[7].ptr, out_bytes, cudaMemcpyDeviceToHost, st));
  const int fin = finish_host_call(p, st);
  return rc ? rc : fin;
}

int grid_gpu_gadget_digits(uint64_t q, uint64_t base, size_t* digits) {
  if (!digits) return GRID_ERR_NULL_POINTER;
  if (base < 2 || q < 3) return GRID_ERR_INVALID_PARAMETERS;
  *digits = gadget_digit_count(q, base);
  return GRID_OK;
}

int grid_gpu_gadget_decompose_dev(const grid_gpu_plan* p, const uint32_t* x, size_t len,
                                  uint64_t base, int digit_major, uint32_t* out, void* stream) {
  if (!p || ((!x || !out) && len)) return GRID_ERR_NULL_POINTER;
  if (base < 2) return GRID_ERR_INVALID_PARAMETERS;
  if (!digit_major && len % p->d) return GRID_ERR_LENGTH_MISMATCH;
  return launch_gadget_decompose(p, x, len, base, gadget_digit_count(p->q, base), digit_major,
                                 out, (cudaStream_t)stream);
}

int grid_gpu_gadget_decompose(grid_gpu_plan* p, const uint32_t* x, size_t len, uint64_t base,
                              int digit_major, uint32_t* out) {
  if (!p || ((!x || !out) && len)) return GRID_ERR_NULL_POINTER;
  if (base < 2) return GRID_ERR_INVALID_PARAMETERS;
  if (!digit_major && len % p->d) return GRID_ERR_LENGTH_MISMATCH;
  if (len == 0) return GRID_OK;
  std::lock_guard<std::mutex> lk(p->mu);
  const size_t k = gadget_digit_count(p->q, base);
  const size_t in_bytes = len * 4, out_bytes = in_bytes * k;
  int rc;
  if ((rc = ensure_scratch(p, 6, in_bytes)) || (rc = ensure_scratch(p, 7, out_bytes))) return rc;
  cudaStream_t st = p->stream;
  rc = cuda_status(cudaMemcpyAsync(p->scratch[6].ptr, x, in_bytes, cudaMemcpyHostToDevice, st));
  if (!rc)
    rc = launch_gadget_decompose(p, static_cast<uint32_t*>(p->scratch[6].ptr), len, base, k,
                                 digit_major, static_cast<uint32_t*>(p->scratch[7].ptr), st);
  if (!rc)
    rc = cuda_status(cudaMemcpyAsync(out, p->scratch[7].ptr, out_bytes, cudaMemcpyDeviceToHost, st));
  const int fin = finish_host_call(p, st);
  return rc ? rc : fin;
}

/* ---- fused LaBRADOR prover round ---------------------------------------- */

int grid_gpu_prover_round_workspace(const grid_gpu_matrix* A, size_t r, size_t jl_rows,
                                    size_t* bytes) {
  if (!A || !bytes) return GRID_ERR_NULL_POINTER;
  const grid_gpu_plan* p = A->plan;
  const size_t n = A->cols, kappa = A->rows, d = p->d;
  if (!dims_ok(r, n, kappa) || !square_dims_ok(p, r, n) || !words_fit(r, kappa, d))
    return GRID_ERR_INVALID_PARAMETERS;
  *bytes = round_ws_bytes(p, r, n, kappa, jl_rows);
  return GRID_OK;
}

int grid_gpu_prover_round_dev(const grid_gpu_matrix* A, const uint32_t* S, size_t r,
                              uint64_t b1, size_t t1, uint64_t b2, size_t t2,
                              const uint8_t* jl_seed, size_t jl_rows, uint32_t* t_limbs,
                              uint32_t* g, uint32_t* g_limbs, uint32_t* p_out, int8_t* jl_flat,
                              void* workspace, size_t workspace_bytes, void* stream) {
  if (!A || !S || !t_limbs || !g) return GRID_ERR_NULL_POINTER;
  const grid_gpu_plan* p = A->plan;
  const size_t n = A->cols, kappa = A->rows, d = p->d;
  if (!dims_ok(r, n, kappa) || !square_dims_ok(p, r, n) || !words_fit(r, kappa, d))
    return GRID_ERR_INVALID_PARAMETERS;
  if (!aligned16(S) || !aligned16(g) || !aligned16(workspace)) return GRID_ERR_MISALIGNED;
  if (is_crt(p) && !crt_bound_ok(p, n)) return GRID_ERR_INVALID_PARAMETERS;
  cudaStream_t st = (cudaStream_t)stream;
  const grid_gpu_plan* e = is_crt(p) ? p->crt[0] : p;
  Carver cv(workspace, workspace_bytes);
  uint32_t* s_hat = cv.take<uint32_t>(r * n * d);
  const size_t e1 = emm_workspace_words(e, (int)r, (int)kappa, (int)n, EMM_DENSE);
  const size_t e2 = emm_workspace_words(e, (int)r, (int)r, (int)n, EMM_UPPER);
  const size_t ew = e1 > e2 ? e1 : e2;
  uint32_t* work = ew ? cv.take<uint32_t>(ew) : nullptr;
  uint32_t* t = cv.take<uint32_t>(r * kappa * d);
  void* jl_ws = cv.take<char>(jl_scratch_bytes(jl_rows ? jl_rows : 1, 0, 0));
  // ring plan without an NTT for q: t and g per auxiliary prime
  const size_t tw = r * kappa * d, gw = r * (r + 1) / 2 * d;
  uint32_t *tj[3] = {}, *gj[3] = {};
  if (is_crt(p))
    for (int j = 0; j < 3; ++j) {
      tj[j] = cv.take<uint32_t>(tw);
      gj[j] = cv.take<uint32_t>(gw);
    }
  if (!cv.ok) return GRID_ERR_INVALID_PARAMETERS;
  // inner commitments and the Gram over the witness's evaluations (one
  // transform shared by both) on plan q into tt / gg
  auto contract = [&](const grid_gpu_plan* q, const grid_gpu_matrix* Aq, const uint32_t* src,
                      uint32_t* tt, uint32_t* gg, cudaStream_t cs) {
    if (src != s_hat && Aq->d_evals_pm && pm_fits(q, r, kappa, n, Aq->ld, EMM_DENSE) &&
        pm_fits(q, r, r, n, n, EMM_UPPER)) {
      // point-major evaluations: both products load their operands with TMA
      int rc = launch_ntt_tc(q, MODE_FWD_PM, src, nullptr, s_hat, r * n, cs);
      if (!rc)
        rc = launch_emm_pm(q, s_hat, Aq->d_evals_pm, (int)r, (int)kappa, (int)n, (int)Aq->ld,
                           EMM_DENSE, tt, work, cs);
      if (!rc) rc = launch_ntt(q, MODE_INV, tt, nullptr, tt, r * kappa, cs);
      if (!rc)
        rc = launch_emm_pm(q, s_hat, s_hat, (int)r, (int)r, (int)n, (int)n, EMM_UPPER, gg, work,
                           cs);
      if (!rc) rc = launch_ntt(q, MODE_INV, gg, nullptr, gg, r * (r + 1) / 2, cs);
      return rc;
    }
    int rc = launch_ntt(q, MODE_FWD, src, nullptr, s_hat, r * n, cs);
    if (!rc)
      rc = launch_emm(q, s_hat, Aq->d_evals, (int)r, (int)kappa, (int)n, (int)Aq->ld, EMM_DENSE,
                      tt, work, cs);
    if (!rc) rc = launch_ntt(q, MODE_INV, tt, nullptr, tt, r * kappa, cs);
    if (!rc)
      rc = launch_emm(q, s_hat, s_hat, (int)r, (int)r, (int)n, (int)n, EMM_UPPER, gg, work, cs);
    if (!rc) rc = launch_ntt(q, MODE_INV, gg, nullptr, gg, r * (r + 1) / 2, cs);
    return rc;
  };
  // The JL projection reads only S and shares nothing with the commitment and
  // Gram chain: fork both off the caller's stream (chain on the high-priority
  // stream, JL on the low-priority one, so the JL's CTAs fill the SMs the
  // chain leaves idle) and join them back before returning.
  const bool jl = jl_seed && p_out;
  cudaStream_t hi = p->fork_hi, lo = p->fork_lo;
  cudaEvent_t ev[3] = {};
  int rc = GRID_OK;
  for (int i = 0; i < 3 && !rc; ++i)
    rc = cuda_status(cudaEventCreateWithFlags(&ev[i], cudaEventDisableTiming));
  if (!rc) rc = cuda_status(cudaEventRecord(ev[0], st));
  if (!rc) rc = cuda_status(cudaStreamWaitEvent(hi, ev[0], 0));
  if (!rc && jl) rc = cuda_status(cudaStreamWaitEvent(lo, ev[0], 0));
  int rc_chain = rc, rc_jl = rc;
  if (!rc) {
    // 3. JL projection of the coefficient vectors (one part per witness vector)
    if (jl)
      rc_jl = launch_jl_project(p->f, jl_seed, jl_rows, S, r, n * d, d, p_out, jl_flat, jl_ws,
                                jl_scratch_bytes(jl_rows, 0, 0), p->num_sms, p->d_err, lo);
    // 1. inner commitments t_i = A s_i and 2. garbage g_ij = <s_i, s_j>, i <= j
    if (!is_crt(p)) {
      rc_chain = contract(p, A, S, t, g, hi);
    } else {
      for (int j = 0; j < 3 && !rc_chain; ++j) {
        rc_chain = lift_one(p, j, S, r * n * d, s_hat, hi);
        if (!rc_chain) rc_chain = contract(p->crt[j], A->crt[j], s_hat, tj[j], gj[j], hi);
      }
      if (!rc_chain) rc_chain = crt_combine(p, tj[0], tj[1], tj[2], tw, t, hi);
      if (!rc_chain) rc_chain = crt_combine(p, gj[0], gj[1], gj[2], gw, g, hi);
    }
    // balanced limbs of both (inner_commit_decomposed, decompose_polys)
    if (!rc_chain) rc_chain = launch_decompose_balanced(p, t, r * kappa, b1, t1, t_limbs, hi);
    if (!rc_chain && g_limbs)
      rc_chain = launch_decompose_balanced(p, g, r * (r + 1) / 2, b2, t2, g_limbs, hi);
    // join: the caller's stream waits for both forks (also after a failed launch)
    int rj = cuda_status(cudaEventRecord(ev[1], hi));
    if (!rj) rj = cuda_status(cudaStreamWaitEvent(st, ev[1], 0));
    if (!rj && jl) rj = cuda_status(cudaEventRecord(ev[2], lo));
    if (!rj && jl) rj = cuda_status(cudaStreamWaitEvent(st, ev[2], 0));
    rc = rc_chain ? rc_chain : rc_jl ? rc_jl : rj;
  }
  for (cudaEvent_t e : ev)
    if (e) cudaEventDestroy(e);
  return rc;
}

}  // extern "C"
