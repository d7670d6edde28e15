// Uneven batched commitments in one persistent, graph-capturable launch.
//
// Many Ajtai commitments t_i = A_{m_i}[:, :n_i] * s_i with different witness
// lengths n_i and different public matrices (each instance uses the first n_i
// columns of its matrix, e.g. one matrix per rank m) run as one sequence:
//   1. one NTT of every witness polynomial (packed s buffer -> s_hat),
//   2. a persistent grouped evaluation-domain matmul: instances are grouped by
//      matrix and sorted by length into tiles (32 to 128 instances, by the
//      matrix's rows); a work item is (tile,
//      8 evaluation points, K range); CTAs pull work items from an atomic
//      counter and add canonical partial sums into 64-bit accumulators,
//   3. a fold of the accumulators mod q and one INTT of every output.
// The reference runs each commitment separately (AjtaiCommitmentScheme::commit,
// commit/src/ajtai/mod.rs:429-441, through PreparedLinearOps,
// commit/src/linear.rs:717-770); the results are the same words.
//
// The K range per work item (k_split) is the tunable schedule parameter; the
// host autotuner (lattica_b200/batch.py) times candidates and stores the best.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <map>
#include <mutex>
#include <new>
#include <tuple>
#include <type_traits>
#include <vector>

#include "batch_tables.cuh"
#include "grid_async.cuh"
#include "grid_field.cuh"
#include "grid_internal.h"

namespace grid {
namespace {

constexpr int TN = 32, EG = 8, KC = 16;
constexpr int RS = KC * EG + 2;  // words per staged row (padded: rows 4 apart, 8 banks apart)
constexpr int kThreads = 256;

// Tile shapes: TMG groups of 4 instances by (32 / TMG) groups of 8 matrix
// rows, for 8 evaluation points; each thread keeps one evaluation point of a
// 4 x 8 sub-tile. A matrix of <= 8 rows takes 128-instance tiles, <= 16 rows
// 64-instance tiles, up to 32 rows 32-instance tiles, so no tile multiplies
// padding rows of a short matrix.
template <int TMG>
struct BTile {
  static constexpr int BM = 4 * TMG, BN = 8 * (32 / TMG);
  static constexpr int ROWS = BM + BN;
  static constexpr int STAGES = ROWS <= 80 ? 3 : 2;
  static constexpr size_t SMEM = (size_t)STAGES * ROWS * RS * 4;
};
constexpr int kMaxTileInstances = BTile<32>::BM;
constexpr size_t kBatchSmem = std::max({BTile<8>::SMEM, BTile<16>::SMEM, BTile<32>::SMEM});

__host__ __device__ constexpr int tile_tmg(uint32_t rows) { return rows <= 8 ? 32 : rows <= 16 ? 16 : 8; }


// One work item (a tile, evaluation points 8 eg .. + 7, K steps k0 .. k1) with
// tile shape TMG: operands stream through a cp.async ring (instances' witness
// evaluations, then the matrix rows, each row 16 K steps x 8 points in global
// order), 96-bit accumulators, canonical partial sums added into acc.
template <int TMG>
__device__ __forceinline__ void batch_item(const WorkDev& wk, const TileDev& tile,
                                           const MatDev& mat, const ItemDev* sitems,
                                           const uint32_t* __restrict__ s_hat,
                                           unsigned long long* __restrict__ acc, int d,
                                           const FieldParams& f, uint32_t* smem) {
  using Tl = BTile<TMG>;
  constexpr int BM = Tl::BM, BN = Tl::BN, STAGES = Tl::STAGES, SW = Tl::ROWS * RS;
  const int t = threadIdx.x;
  const int eg = t & 7, tm = (t >> 3) % TMG, tn = (t >> 3) / TMG;
  const int e0 = wk.eg * EG;
  const int nchunks = (int)((wk.k1 - wk.k0 + KC - 1) / KC);
  // this thread copies quarter t & 3 of step (t >> 2) & 15 of rows (t >> 6) + 4i
  const int cq = t & 3, ck = (t >> 2) & (KC - 1), cr = t >> 6;
  const int cdst = cr * RS + ck * EG + 2 * cq;

  auto issue = [&](int c) {
    uint32_t* st = smem + (c % STAGES) * SW + cdst;
    const uint32_t k = wk.k0 + (uint32_t)(c * KC + ck);
    const bool kval = k < wk.k1;
#pragma unroll
    for (int i = 0; i < BM / 4; ++i) {
      const int row = cr + 4 * i;
      const ItemDev& it = sitems[row];
      const bool valid = kval && (uint32_t)row < tile.count && k < it.n;
      const uint32_t* src = valid ? s_hat + (it.s_off + k) * d + e0 + 2 * cq : s_hat;
      cp_async8(st + 4 * i * RS, src, valid ? 8u : 0u);
    }
#pragma unroll
    for (int i = 0; i < BN / 4; ++i) {
      const int r = cr + 4 * i;
      const bool valid = kval && (uint32_t)r < mat.rows;
      const uint32_t* src =
          valid ? mat.evals + ((size_t)r * mat.ld + k) * d + e0 + 2 * cq : mat.evals;
      cp_async8(st + (BM + 4 * i) * RS, src, valid ? 8u : 0u);
    }
  };

  Acc96 a[4][8];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 8; ++j) acc96_zero(a[i][j]);
  const int xo = (tm * 4) * RS + eg;
  const int yo = (BM + tn * 8) * RS + eg;
#pragma unroll
  for (int c = 0; c < STAGES - 1; ++c) {
    if (c < nchunks) issue(c);
    cp_async_commit();
  }
  for (int c = 0; c < nchunks; ++c) {
    cp_async_wait<STAGES - 2>();
    __syncthreads();  // chunk c landed for every thread; stage (c - 1) % STAGES is free
    if (c + STAGES - 1 < nchunks) issue(c + STAGES - 1);
    cp_async_commit();
    const uint32_t* xs = smem + (c % STAGES) * SW + xo;
    const uint32_t* ys = smem + (c % STAGES) * SW + yo;
#pragma unroll
    for (int kk = 0; kk < KC; ++kk) {
      uint32_t xr[4], yr[8];
#pragma unroll
      for (int i = 0; i < 4; ++i) xr[i] = xs[kk * EG + i * RS];
#pragma unroll
      for (int j = 0; j < 8; ++j) yr[j] = ys[kk * EG + j * RS];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc96_mad(a[i][j], xr[i], yr[j]);
    }
  }
  cp_async_wait<0>();
  const int e = e0 + eg;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int m = tm * 4 + i;
    if ((uint32_t)m >= tile.count) continue;
    const unsigned long long t_off = sitems[m].t_off;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int row = tn * 8 + j;
      if ((uint32_t)row >= mat.rows) continue;
      atomicAdd(&acc[(t_off + row) * d + e], (unsigned long long)acc96_reduce(a[i][j], f));
    }
  }
}

// Persistent: CTAs pull work items from an atomic counter (longest K ranges
// first); one CTA per SM keeps the accumulators in registers.
__global__ void __launch_bounds__(kThreads, 1) batch_emm_kernel(
    const WorkDev* __restrict__ work, unsigned nwork, const TileDev* __restrict__ tiles,
    const ItemDev* __restrict__ items, const MatDev* __restrict__ mats,
    const uint32_t* __restrict__ s_hat, unsigned long long* __restrict__ acc,
    unsigned* __restrict__ counter, int d, FieldParams f) {
  extern __shared__ __align__(16) uint32_t batch_smem[];
  __shared__ ItemDev sitems[kMaxTileInstances];
  __shared__ unsigned widx;
  const int t = threadIdx.x;

  for (;;) {
    if (t == 0) widx = atomicAdd(counter, 1u);
    __syncthreads();
    const unsigned w = widx;
    if (w >= nwork) break;
    const WorkDev wk = work[w];
    const TileDev tile = tiles[wk.tile];
    const MatDev mat = mats[tile.matrix];
    for (int i = t; i < kMaxTileInstances; i += kThreads) {
      ItemDev it = {0, 0, 0, 0};
      if ((uint32_t)i < tile.count) it = items[tile.first + i];
      sitems[i] = it;
    }
    __syncthreads();
    switch (tile_tmg(mat.rows)) {
      case 32: batch_item<32>(wk, tile, mat, sitems, s_hat, acc, d, f, batch_smem); break;
      case 16: batch_item<16>(wk, tile, mat, sitems, s_hat, acc, d, f, batch_smem); break;
      default: batch_item<8>(wk, tile, mat, sitems, s_hat, acc, d, f, batch_smem); break;
    }
    __syncthreads();  // stages, sitems and widx are rewritten by the next work item
  }
}

__global__ void fold_kernel(const unsigned long long* __restrict__ acc, uint32_t* __restrict__ out,
                            size_t n, uint32_t q) {
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
    out[i] = (uint32_t)(acc[i] % q);
}

}  // namespace
}  // namespace grid

using namespace grid;

struct grid_gpu_batch {
  grid_gpu_plan* plan = nullptr;
  std::vector<grid_gpu_matrix*> mat_handles;
  std::vector<grid_gpu_batch_item> items;  // as given (tiles are rebuilt on a new config)
  std::vector<MatDev> mats;
  std::vector<ItemDev> sorted;    // items grouped by matrix, longest first
  std::vector<TileDev> tiles;
  uint64_t s_polys = 0, t_polys = 0;
  uint32_t k_split = 1024;
  uint32_t tile_instances = 0;    // 0: the engine's default
  int engine = GRID_GPU_ENGINE_AUTO;
  bool tc = false;                // the tensor-core kernel runs the grouped product
  bool pm = false;                // ... over point-major evaluations (grouped_pm.cu)
  unsigned class_begin[TC_CLASSES + 1] = {};
  // device tables
  MatDev* d_mats = nullptr;
  ItemDev* d_items = nullptr;
  TileDev* d_tiles = nullptr;
  WorkDev* d_work = nullptr;
  unsigned nwork = 0;
  // point-major engine: the witnesses' transform tile list, the padded rows
  uint4* d_xtiles = nullptr;
  unsigned long long nxtiles = 0;
  uint64_t s_region = 0;  // polys per point of the transformed witnesses
  // captured graphs, keyed by (s, t, workspace, stream)
  std::mutex mu;
  std::map<std::tuple<const void*, void*, void*, void*>, cudaGraphExec_t> graphs;
  int num_sms = 0;
};

namespace {

struct Tables {
  std::vector<MatDev> mats;
  std::vector<ItemDev> sorted;
  std::vector<TileDev> tiles;
  std::vector<WorkDev> work;
  uint64_t s_polys = 0, t_polys = 0;
  uint32_t k_split = 0;
  bool tc = false;
  bool pm = false;
  unsigned class_begin[TC_CLASSES + 1] = {};
  // Point-major layout: instance i's polys at a column of a multiple of 128
  // (ItemDev::s_off of the point-major tables), the transform's tile list.
  uint64_t pm_polys = 0;
  std::vector<uint4> xtiles;
};

// Evaluation groups of a tile: 8 points per CUDA-core work item; 4 or 2 per
// tensor-core work item (by the tile's Y rows); one per point-major item.
uint32_t tile_groups(const Tables& tb, const TileDev& tl, uint32_t d) {
  if (!tb.tc) return d / EG;
  if (tb.pm) return d;
  const uint32_t ny = tl.matrix == kUpperTile ? tl.count : tb.mats[tl.matrix].rows;
  return d / (uint32_t)tc_points(ny);
}

// Cut every tile into (K range, evaluation group) work items; longest K ranges
// first (within each tensor-core class, classes in order).
void make_work(Tables& tb, uint32_t d) {
  tb.work.clear();
  std::vector<int> cls;
  for (uint32_t ti = 0; ti < tb.tiles.size(); ++ti) {
    const TileDev& tl = tb.tiles[ti];
    const uint32_t groups = tile_groups(tb, tl, d);
    for (uint32_t k0 = 0; k0 < tl.kmax; k0 += tb.k_split) {
      const uint32_t k1 = std::min(tl.kmax, k0 + tb.k_split);
      for (uint32_t g = 0; g < groups; ++g) {
        tb.work.push_back(WorkDev{ti, k0, k1, g});
        cls.push_back(tb.tc ? tc_class(tl, tb.mats.data()) : 0);
      }
    }
  }
  std::vector<size_t> order(tb.work.size());
  for (size_t i = 0; i < order.size(); ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](size_t x, size_t y) {
    if (cls[x] != cls[y]) return cls[x] < cls[y];
    return (tb.work[x].k1 - tb.work[x].k0) > (tb.work[y].k1 - tb.work[y].k0);
  });
  std::vector<WorkDev> sorted(order.size());
  for (size_t i = 0; i < order.size(); ++i) sorted[i] = tb.work[order[i]];
  tb.work.swap(sorted);
  for (int c = 0; c <= TC_CLASSES; ++c) tb.class_begin[c] = 0;
  for (size_t i = 0; i < order.size(); ++i) tb.class_begin[cls[order[i]] + 1]++;
  for (int c = 0; c < TC_CLASSES; ++c) tb.class_begin[c + 1] += tb.class_begin[c];
}

// K range per work item when the caller leaves it to the library: about four
// work items per SM, so a small batch (a few instances, one tile) still
// spreads over the whole GPU instead of running its K loop on a few CTAs;
// large batches reach the 8192 cap, where fewer accumulator atomics win.
uint32_t auto_k_split(const Tables& tb, uint32_t d, int num_sms) {
  uint64_t steps = 0;  // KC-wide K steps over every tile and evaluation group
  for (const TileDev& tl : tb.tiles) steps += (uint64_t)((tl.kmax + KC - 1) / KC) * tile_groups(tb, tl, d);
  const uint64_t target = 4ull * (uint64_t)(num_sms > 0 ? num_sms : 148);
  uint64_t per = (steps + target - 1) / target;
  per = std::max<uint64_t>(tb.tc ? 2 : 1, std::min<uint64_t>(per, 8192 / KC));
  if (tb.tc) per = (per + 1) / 2 * 2;  // whole 32-word tensor-core chunks
  return (uint32_t)(per * KC);
}

bool engine_uses_tc(const grid_gpu_plan* plan, int engine) {
  if (engine == GRID_GPU_ENGINE_CUDA_CORE) return false;
  return plan->tc_emm && plan->d % 4 == 0;
}

// Group items by matrix, longest first, into tiles; then cut every tile into
// work items. Tensor-core tiles hold up to 128 instances (the MMA's M); the
// CUDA-core kernel's tiles 32, 64 or 128 (by the matrix's rows, tile_tmg).
// tile_instances (when nonzero) caps the instances per tile.
int build_tables(const grid_gpu_plan* plan, grid_gpu_matrix* const* mats, size_t nmats,
                 const grid_gpu_batch_item* items, size_t nitems, uint32_t k_split,
                 uint32_t tile_instances, int engine, Tables& tb) {
  if (!plan || (!mats && nmats) || (!items && nitems)) return GRID_ERR_NULL_POINTER;
  // the grouped kernels contract evaluations mod q: a ring plan without an NTT
  // for q commits through grid_gpu_commit_dev instead
  if (is_crt(plan)) return plan->ntt_status;
  if (nmats == 0 || nitems == 0 || nitems > (1u << 30)) return GRID_ERR_INVALID_PARAMETERS;
  if (k_split != 0 && (k_split < (uint32_t)KC || k_split % KC || k_split > kTcMaxK))
    return GRID_ERR_INVALID_PARAMETERS;
  // point-major work items cover whole 32-word chunks
  if (engine == GRID_GPU_ENGINE_POINT_MAJOR && k_split % 32) return GRID_ERR_INVALID_PARAMETERS;
  if (engine < GRID_GPU_ENGINE_AUTO || engine > GRID_GPU_ENGINE_POINT_MAJOR)
    return GRID_ERR_INVALID_PARAMETERS;
  if (tile_instances != 0 && (tile_instances % 4 || tile_instances > kTcMaxTileRows))
    return GRID_ERR_INVALID_PARAMETERS;
  for (size_t i = 0; i < nmats; ++i) {
    if (!mats[i]) return GRID_ERR_NULL_POINTER;
    if (mats[i]->plan != plan) return GRID_ERR_INVALID_PARAMETERS;
    if (mats[i]->rows > (size_t)TN) return GRID_ERR_INVALID_PARAMETERS;  // ranks up to 32
    tb.mats.push_back(MatDev{mats[i]->d_evals, mats[i]->d_evals_pm, (uint32_t)mats[i]->rows,
                             (uint32_t)mats[i]->ld});
  }
  std::vector<std::pair<uint32_t, uint32_t>> order;  // (matrix, index)
  order.reserve(nitems);
  for (size_t i = 0; i < nitems; ++i) {
    const grid_gpu_batch_item& it = items[i];
    if (it.matrix >= nmats || it.n == 0 || it.n > mats[it.matrix]->cols)
      return GRID_ERR_DIMENSION_MISMATCH;
    tb.s_polys = std::max<uint64_t>(tb.s_polys, it.s_offset + it.n);
    tb.t_polys = std::max<uint64_t>(tb.t_polys, it.t_offset + mats[it.matrix]->rows);
    tb.pm_polys += round_up(it.n, 128);  // the workspace does not depend on the engine
    order.emplace_back(it.matrix, (uint32_t)i);
  }
  // The point-major engine needs the point-major forward transform (d = 64,
  // tensor cores), every matrix's point-major evaluations, K ranges of whole
  // chunks, and transform tiles whose source rows and destination columns
  // stay below 2^31; AUTO takes it where those hold.
  bool pm_ok = plan->pm_emm && ntt_tc_available(plan) && k_split % 32 == 0 &&
               tb.s_polys <= (uint64_t)INT32_MAX - 128 && tb.pm_polys <= (uint64_t)INT32_MAX - 128;
  for (size_t i = 0; pm_ok && i < nmats; ++i) pm_ok = mats[i]->d_evals_pm != nullptr;
  if (engine == GRID_GPU_ENGINE_POINT_MAJOR && !pm_ok) return GRID_ERR_UNSUPPORTED_DEGREE;
  tb.pm = engine == GRID_GPU_ENGINE_POINT_MAJOR || (engine == GRID_GPU_ENGINE_AUTO && pm_ok);
  tb.tc = tb.pm || engine_uses_tc(plan, engine);
  if (engine == GRID_GPU_ENGINE_TENSOR && !tb.tc) return GRID_ERR_UNSUPPORTED_DEGREE;
  std::stable_sort(order.begin(), order.end(), [&](const auto& x, const auto& y) {
    if (x.first != y.first) return x.first < y.first;
    return items[x.second].n > items[y.second].n;
  });
  uint64_t pcol = 0;  // next point-major column
  for (size_t i = 0; i < order.size();) {
    const uint32_t m = order[i].first;
    size_t j = i;
    TileDev tl{(uint32_t)tb.sorted.size(), 0, m, 0};
    size_t cap = tb.tc ? (size_t)kTcMaxTileRows : 4 * (size_t)tile_tmg(tb.mats[m].rows);
    if (tile_instances) cap = std::min<size_t>(cap, tile_instances);
    while (j < order.size() && order[j].first == m && j - i < cap) {
      const grid_gpu_batch_item& it = items[order[j].second];
      uint64_t s_off = it.s_offset;
      if (tb.pm) {  // the instance's own 128-aligned columns; the rest of its last tile is 0
        for (uint32_t r = 0; r < it.n; r += 128)
          tb.xtiles.push_back(make_uint4((uint32_t)(it.s_offset + r), (uint32_t)(pcol + r),
                                         std::min<uint32_t>(128, it.n - r), 0));
        s_off = pcol;
        pcol += round_up(it.n, 128);
      }
      tb.sorted.push_back(ItemDev{s_off, it.t_offset, it.n, 0});
      tl.kmax = std::max(tl.kmax, it.n);
      ++j;
    }
    tl.count = (uint32_t)(j - i);
    tb.tiles.push_back(tl);
    i = j;
  }
  tb.k_split = k_split ? k_split : auto_k_split(tb, plan->d, plan->num_sms);
  make_work(tb, plan->d);
  return GRID_OK;
}

uint64_t witness_region(uint64_t s_polys, uint64_t pm_polys);

int upload(grid_gpu_batch* b) {
  for (auto& kv : b->graphs) cudaGraphExecDestroy(kv.second);
  b->graphs.clear();
  for (void* ptr : {(void*)b->d_mats, (void*)b->d_items, (void*)b->d_tiles, (void*)b->d_work,
                    (void*)b->d_xtiles})
    if (ptr) cudaFree(ptr);
  b->d_mats = nullptr;
  b->d_items = nullptr;
  b->d_tiles = nullptr;
  b->d_work = nullptr;
  b->d_xtiles = nullptr;
  Tables tb;
  int rc = build_tables(b->plan, b->mat_handles.data(), b->mat_handles.size(), b->items.data(),
                        b->items.size(), b->k_split, b->tile_instances, b->engine, tb);
  if (rc) return rc;
  b->mats = std::move(tb.mats);
  b->sorted = std::move(tb.sorted);
  b->tiles = std::move(tb.tiles);
  b->s_polys = tb.s_polys;
  b->t_polys = tb.t_polys;
  b->tc = tb.tc;
  b->pm = tb.pm;
  b->s_region = witness_region(tb.s_polys, tb.pm_polys);
  b->nxtiles = tb.xtiles.size();
  std::copy(tb.class_begin, tb.class_begin + TC_CLASSES + 1, b->class_begin);
  b->nwork = (unsigned)tb.work.size();
  auto send = [](auto** dst, const auto& v) {
    using T = typename std::remove_reference<decltype(v)>::type::value_type;
    cudaError_t e = cudaMalloc(dst, std::max<size_t>(1, v.size()) * sizeof(T));
    if (e == cudaSuccess && !v.empty())
      e = cudaMemcpy(*dst, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice);
    return e;
  };
  cudaError_t e = send(&b->d_mats, b->mats);
  if (e == cudaSuccess) e = send(&b->d_items, b->sorted);
  if (e == cudaSuccess) e = send(&b->d_tiles, b->tiles);
  if (e == cudaSuccess) e = send(&b->d_work, tb.work);
  if (e == cudaSuccess && b->pm) e = send(&b->d_xtiles, tb.xtiles);
  return cuda_status(e);
}

// The transformed witnesses, s_region polys per point (at least the packed
// witness buffer's and the point-major engine's padded layout, a multiple of
// 4), then the accumulators and one work counter per tensor-core class.
uint64_t witness_region(uint64_t s_polys, uint64_t pm_polys) {
  return std::max<uint64_t>((s_polys + 3) / 4 * 4, pm_polys);
}
size_t core_bytes(uint64_t s_region_polys, uint64_t t_polys, size_t d) {
  return round_up(s_region_polys * d * 4, 256) + round_up(t_polys * d * 8, 256) + 256;
}

size_t ws_bytes(const grid_gpu_batch* b) { return core_bytes(b->s_region, b->t_polys, b->plan->d); }

// Grouped product -> fold -> INTT over given transformed witnesses and tables:
// acc (t_polys x d u64) and the counters are cleared here. pm: s_hat is
// point-major with rows of ps polys (the point-major engine's tables).
int run_product(const grid_gpu_plan* p, bool tc, bool pm, const unsigned* class_begin,
                const MatDev* d_mats, const ItemDev* d_items, const TileDev* d_tiles,
                const WorkDev* d_work, unsigned nwork, const uint32_t* s_hat, uint64_t ps,
                unsigned long long* acc, unsigned* counters, uint64_t t_polys, uint32_t* t,
                cudaStream_t st) {
  const size_t d = p->d;
  cudaError_t e = cudaMemsetAsync(acc, 0, t_polys * d * 8, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(counters, 0, TC_CLASSES * sizeof(unsigned), st);
  if (e != cudaSuccess) return cuda_status(e);
  int rc = GRID_OK;
  if (pm) {
    for (int c = 0; c < TC_CLASSES && !rc; ++c) {
      const unsigned n = class_begin[c + 1] - class_begin[c];
      if (n)
        rc = launch_batch_pm(p, c, d_work + class_begin[c], n, d_tiles, d_items, d_mats, s_hat,
                             ps, acc, st);
    }
    if (rc) return rc;
  } else if (tc) {
    for (int c = 0; c < TC_CLASSES && !rc; ++c) {
      const unsigned n = class_begin[c + 1] - class_begin[c];
      if (n)
        rc = launch_batch_tc(p, c, d_work + class_begin[c], n, d_tiles, d_items, d_mats, s_hat,
                             acc, counters + c, st);
    }
    if (rc) return rc;
  } else if (nwork) {
    static int bps_cache[kMaxDevices] = {};
    int bps = 0;
    rc = prepare_kernel(batch_emm_kernel, kBatchSmem, kThreads, p->device, bps_cache, &bps);
    if (rc) return rc;
    const unsigned grid = std::min<unsigned>(nwork, (unsigned)(p->num_sms * bps));
    batch_emm_kernel<<<grid, kThreads, kBatchSmem, st>>>(d_work, nwork, d_tiles, d_items, d_mats,
                                                         s_hat, acc, counters, (int)d, p->f);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_status(e);
  }
  const size_t words = t_polys * d;
  unsigned blocks = (unsigned)std::min<size_t>((words + 255) / 256, (size_t)p->num_sms * 8);
  fold_kernel<<<blocks ? blocks : 1, 256, 0, st>>>(acc, t, words, p->f.q);
  if ((e = cudaGetLastError()) != cudaSuccess) return cuda_status(e);
  return launch_ntt(p, MODE_INV, t, nullptr, t, t_polys, st);
}

// NTT(s) -> grouped product -> fold -> INTT(t), with device tables given
// (layout of core_bytes).
int run_core(const grid_gpu_plan* p, bool tc, bool pm, const unsigned* class_begin,
             const MatDev* d_mats, const ItemDev* d_items, const TileDev* d_tiles,
             const WorkDev* d_work, unsigned nwork, uint64_t s_polys, uint64_t ps, uint64_t t_polys,
             const uint32_t* s, uint32_t* t, void* ws, cudaStream_t st,
             const uint4* xtiles = nullptr, unsigned long long nxtiles = 0) {
  const size_t d = p->d;
  char* base = static_cast<char*>(ws);
  uint32_t* s_hat = reinterpret_cast<uint32_t*>(base);
  unsigned long long* acc =
      reinterpret_cast<unsigned long long*>(base + round_up(ps * d * 4, 256));
  unsigned* counters =
      reinterpret_cast<unsigned*>(base + round_up(ps * d * 4, 256) + round_up(t_polys * d * 8, 256));
  // point-major: [point][ps], every instance at its own 128-aligned columns
  const int rc = pm ? launch_ntt_tc_pm_tiles(p, s, s_polys, s_hat, ps, xtiles, nxtiles, st)
                    : launch_ntt(p, MODE_FWD, s, nullptr, s_hat, s_polys, st);
  if (rc) return rc;
  return run_product(p, tc, pm, class_begin, d_mats, d_items, d_tiles, d_work, nwork, s_hat, ps,
                     acc, counters, t_polys, t, st);
}

int run_sequence(grid_gpu_batch* b, const uint32_t* s, uint32_t* t, void* ws, cudaStream_t st) {
  return run_core(b->plan, b->tc, b->pm, b->class_begin, b->d_mats, b->d_items, b->d_tiles,
                  b->d_work, b->nwork, b->s_polys, b->s_region, b->t_polys, s, t, ws, st,
                  b->d_xtiles, b->nxtiles);
}

size_t tables_bytes(const Tables& tb) {
  return round_up(tb.mats.size() * sizeof(MatDev), 256) +
         round_up(tb.sorted.size() * sizeof(ItemDev), 256) +
         round_up(tb.tiles.size() * sizeof(TileDev), 256) +
         round_up(tb.work.size() * sizeof(WorkDev), 256) +
         round_up(tb.xtiles.size() * sizeof(uint4), 256);
}

// Pack the tables (and the point-major transform's tile list) into one host
// image of the device layout at `dev` and send it with a single copy. The
// source is pageable: the copy returns once its bytes are staged, so the image
// may go away when the caller returns.
int send_tables(const Tables& tb, char* dev, const MatDev** dm, const ItemDev** di,
                const TileDev** dt, const WorkDev** dw, const uint4** dx, cudaStream_t st) {
  std::vector<char> image(tables_bytes(tb));
  size_t off = 0;
  auto put = [&](const void* src, size_t n) -> void* {
    if (n) std::memcpy(image.data() + off, src, n);
    void* dst = dev + off;
    off += round_up(n, 256);
    return dst;
  };
  *dm = static_cast<const MatDev*>(put(tb.mats.data(), tb.mats.size() * sizeof(MatDev)));
  *di = static_cast<const ItemDev*>(put(tb.sorted.data(), tb.sorted.size() * sizeof(ItemDev)));
  *dt = static_cast<const TileDev*>(put(tb.tiles.data(), tb.tiles.size() * sizeof(TileDev)));
  *dw = static_cast<const WorkDev*>(put(tb.work.data(), tb.work.size() * sizeof(WorkDev)));
  *dx = static_cast<const uint4*>(put(tb.xtiles.data(), tb.xtiles.size() * sizeof(uint4)));
  if (image.empty()) return GRID_OK;
  return cuda_status(cudaMemcpyAsync(dev, image.data(), image.size(), cudaMemcpyHostToDevice, st));
}

// ---- batched Gram matrices (the Gram of many witnesses of different r, n) ----

// Witness evaluations packed in item order; tiles = one instance (r rows).
int build_gram_tables(const grid_gpu_plan* plan, const grid_gpu_gram_item* items, size_t nitems,
                      uint32_t k_split, Tables& tb, uint64_t* g_polys) {
  if (!plan || (!items && nitems)) return GRID_ERR_NULL_POINTER;
  if (nitems == 0 || nitems > (1u << 24)) return GRID_ERR_INVALID_PARAMETERS;
  if (k_split != 0 && (k_split < (uint32_t)KC || k_split % KC || k_split > kTcMaxK))
    return GRID_ERR_INVALID_PARAMETERS;
  tb.tc = true;
  uint64_t shat = 0, g = 0;
  for (size_t i = 0; i < nitems; ++i) {
    const grid_gpu_gram_item& it = items[i];
    if (it.r == 0 || it.n == 0 || it.r > (uint32_t)kTcMaxYRows) return GRID_ERR_INVALID_PARAMETERS;
    TileDev tl{(uint32_t)tb.sorted.size(), it.r, kUpperTile, it.n};
    for (uint32_t j = 0; j < it.r; ++j)
      tb.sorted.push_back(ItemDev{shat + (uint64_t)j * it.n, g, it.n, 0});
    tb.tiles.push_back(tl);
    shat += (uint64_t)it.r * it.n;
    g += (uint64_t)it.r * (it.r + 1) / 2;
  }
  tb.s_polys = shat;
  tb.t_polys = g;
  *g_polys = g;
  tb.k_split = k_split ? k_split : auto_k_split(tb, plan->d, plan->num_sms);
  make_work(tb, plan->d);
  return GRID_OK;
}

bool gram_uses_tc(const grid_gpu_plan* plan) {
  return !is_crt(plan) && plan->tc_emm && plan->d % 4 == 0;
}

}  // namespace

extern "C" {

int grid_gpu_batch_create(grid_gpu_plan* plan, grid_gpu_matrix* const* mats, size_t nmats,
                          const grid_gpu_batch_item* items, size_t nitems, grid_gpu_batch** out) {
  if (!out) return GRID_ERR_NULL_POINTER;
  *out = nullptr;
  Tables probe;
  int rc = build_tables(plan, mats, nmats, items, nitems, 1024, 0, GRID_GPU_ENGINE_AUTO, probe);
  if (rc) return rc;
  grid_gpu_batch* b = new (std::nothrow) grid_gpu_batch();
  if (!b) return GRID_ERR_OUT_OF_MEMORY;
  b->plan = plan;
  b->num_sms = plan->num_sms;
  b->k_split = 1024;
  b->mat_handles.assign(mats, mats + nmats);
  b->items.assign(items, items + nitems);
  rc = upload(b);
  if (rc) {
    grid_gpu_batch_destroy(b);
    return rc;
  }
  *out = b;
  return GRID_OK;
}

int grid_gpu_batch_destroy(grid_gpu_batch* b) {
  if (!b) return GRID_ERR_NULL_POINTER;
  for (auto& kv : b->graphs) cudaGraphExecDestroy(kv.second);
  if (b->d_mats) cudaFree(b->d_mats);
  if (b->d_items) cudaFree(b->d_items);
  if (b->d_tiles) cudaFree(b->d_tiles);
  if (b->d_work) cudaFree(b->d_work);
  if (b->d_xtiles) cudaFree(b->d_xtiles);
  delete b;
  return GRID_OK;
}

int grid_gpu_batch_set_config(grid_gpu_batch* b, const grid_gpu_batch_config* cfg) {
  if (!b || !cfg) return GRID_ERR_NULL_POINTER;
  if (cfg->k_split < KC || cfg->k_split % KC || cfg->k_split > kTcMaxK)
    return GRID_ERR_INVALID_PARAMETERS;
  std::lock_guard<std::mutex> lk(b->mu);
  const uint32_t old_k = b->k_split, old_ti = b->tile_instances;
  const int old_engine = b->engine;
  b->k_split = cfg->k_split;
  b->tile_instances = cfg->tile_instances;
  b->engine = (int)cfg->engine;
  const int rc = upload(b);
  if (rc) {  // keep the previous (valid) configuration
    b->k_split = old_k;
    b->tile_instances = old_ti;
    b->engine = old_engine;
    upload(b);
  }
  return rc;
}

int grid_gpu_batch_get_config(const grid_gpu_batch* b, grid_gpu_batch_config* cfg) {
  if (!b || !cfg) return GRID_ERR_NULL_POINTER;
  cfg->k_split = b->k_split;
  cfg->work_items = b->nwork;
  cfg->tiles = (uint32_t)b->tiles.size();
  cfg->tile_instances = b->tile_instances;
  cfg->engine = (uint32_t)b->engine;
  cfg->tensor_cores = b->tc ? 1u : 0u;
  return GRID_OK;
}

int grid_gpu_batch_shape(const grid_gpu_batch* b, uint64_t* s_polys, uint64_t* t_polys) {
  if (!b || !s_polys || !t_polys) return GRID_ERR_NULL_POINTER;
  *s_polys = b->s_polys;
  *t_polys = b->t_polys;
  return GRID_OK;
}

int grid_gpu_batch_workspace(const grid_gpu_batch* b, size_t* bytes) {
  if (!b || !bytes) return GRID_ERR_NULL_POINTER;
  *bytes = ws_bytes(b);
  return GRID_OK;
}

int grid_gpu_batch_commit_dev(grid_gpu_batch* b, const uint32_t* s, uint32_t* t, void* workspace,
                              size_t workspace_bytes, void* stream) {
  if (!b || !s || !t || !workspace) return GRID_ERR_NULL_POINTER;
  if (workspace_bytes < ws_bytes(b)) return GRID_ERR_INVALID_PARAMETERS;
  if (((uintptr_t)s | (uintptr_t)t | (uintptr_t)workspace) & 15u) return GRID_ERR_MISALIGNED;
  std::lock_guard<std::mutex> lk(b->mu);
  return run_sequence(b, s, t, workspace, (cudaStream_t)stream);
}

int grid_gpu_batch_commit_graph(grid_gpu_batch* b, const uint32_t* s, uint32_t* t,
                                void* workspace, size_t workspace_bytes, void* stream) {
  if (!b || !s || !t || !workspace) return GRID_ERR_NULL_POINTER;
  if (workspace_bytes < ws_bytes(b)) return GRID_ERR_INVALID_PARAMETERS;
  if (((uintptr_t)s | (uintptr_t)t | (uintptr_t)workspace) & 15u) return GRID_ERR_MISALIGNED;
  cudaStream_t st = (cudaStream_t)stream;
  if (!st) return GRID_ERR_INVALID_PARAMETERS;  // capture needs a non-default stream
  std::lock_guard<std::mutex> lk(b->mu);
  const auto key = std::make_tuple((const void*)s, (void*)t, workspace, (void*)st);
  auto it = b->graphs.find(key);
  if (it == b->graphs.end()) {
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return cuda_status(e);
    const int rc = run_sequence(b, s, t, workspace, st);
    e = cudaStreamEndCapture(st, &g);
    if (rc) {
      if (g) cudaGraphDestroy(g);
      return rc;
    }
    if (e != cudaSuccess) return cuda_status(e);
    cudaGraphExec_t exec = nullptr;
    e = cudaGraphInstantiate(&exec, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return cuda_status(e);
    it = b->graphs.emplace(key, exec).first;
  }
  return cuda_status(cudaGraphLaunch(it->second, st));
}

int grid_gpu_batch_oneshot_workspace(grid_gpu_plan* plan, grid_gpu_matrix* const* mats,
                                     size_t nmats, const grid_gpu_batch_item* items,
                                     size_t nitems, uint32_t k_split, size_t* bytes) {
  if (!bytes) return GRID_ERR_NULL_POINTER;
  Tables tb;
  const int rc =
      build_tables(plan, mats, nmats, items, nitems, k_split, 0, GRID_GPU_ENGINE_AUTO, tb);
  if (rc) return rc;
  *bytes = core_bytes(witness_region(tb.s_polys, tb.pm_polys), tb.t_polys, plan->d) + tables_bytes(tb);
  return GRID_OK;
}

int grid_gpu_batch_commit_oneshot_dev(grid_gpu_plan* plan, grid_gpu_matrix* const* mats,
                                      size_t nmats, const grid_gpu_batch_item* items,
                                      size_t nitems, uint32_t k_split, const uint32_t* s,
                                      uint32_t* t, void* workspace, size_t workspace_bytes,
                                      void* stream) {
  if (!s || !t || !workspace) return GRID_ERR_NULL_POINTER;
  if (((uintptr_t)s | (uintptr_t)t | (uintptr_t)workspace) & 15u) return GRID_ERR_MISALIGNED;
  Tables tb;
  int rc = build_tables(plan, mats, nmats, items, nitems, k_split, 0, GRID_GPU_ENGINE_AUTO, tb);
  if (rc) return rc;
  const size_t core = core_bytes(witness_region(tb.s_polys, tb.pm_polys), tb.t_polys, plan->d);
  if (workspace_bytes < core + tables_bytes(tb)) return GRID_ERR_INVALID_PARAMETERS;
  cudaStream_t st = (cudaStream_t)stream;
  const MatDev* dm;
  const ItemDev* di;
  const TileDev* dt;
  const WorkDev* dw;
  const uint4* dx;
  rc = send_tables(tb, static_cast<char*>(workspace) + core, &dm, &di, &dt, &dw, &dx, st);
  if (rc) return rc;
  return run_core(plan, tb.tc, tb.pm, tb.class_begin, dm, di, dt, dw, (unsigned)tb.work.size(),
                  tb.s_polys, witness_region(tb.s_polys, tb.pm_polys), tb.t_polys, s, t, workspace,
                  st, dx, tb.xtiles.size());
}

int grid_gpu_batch_gram_workspace(const grid_gpu_plan* plan, const grid_gpu_gram_item* items,
                                  size_t nitems, uint32_t k_split, size_t* bytes) {
  if (!plan || !bytes) return GRID_ERR_NULL_POINTER;
  if (!gram_uses_tc(plan)) {  // one Gram call after another in a shared workspace
    if (!items && nitems) return GRID_ERR_NULL_POINTER;
    size_t need = 16;
    for (size_t i = 0; i < nitems; ++i) {
      size_t w = 0;
      const int rc = grid_gpu_gram_workspace(plan, items[i].r, items[i].n, &w);
      if (rc) return rc;
      need = std::max(need, w);
    }
    *bytes = need;
    return GRID_OK;
  }
  Tables tb;
  uint64_t g_polys = 0;
  const int rc = build_gram_tables(plan, items, nitems, k_split, tb, &g_polys);
  if (rc) return rc;
  *bytes = core_bytes(witness_region(tb.s_polys, tb.pm_polys), tb.t_polys, plan->d) + tables_bytes(tb);
  return GRID_OK;
}

int grid_gpu_batch_gram_dev(const grid_gpu_plan* plan, const uint32_t* S,
                            const grid_gpu_gram_item* items, size_t nitems, uint32_t k_split,
                            uint32_t* G, void* workspace, size_t workspace_bytes, void* stream) {
  if (!plan || !S || !G || !workspace || (!items && nitems)) return GRID_ERR_NULL_POINTER;
  if (((uintptr_t)S | (uintptr_t)G | (uintptr_t)workspace) & 15u) return GRID_ERR_MISALIGNED;
  cudaStream_t st = (cudaStream_t)stream;
  const size_t d = plan->d;
  if (!gram_uses_tc(plan)) {
    uint64_t g = 0;
    for (size_t i = 0; i < nitems; ++i) {
      const int rc = grid_gpu_gram_dev(plan, S + items[i].s_offset * d, items[i].r, items[i].n,
                                       G + g * d, workspace, workspace_bytes, stream);
      if (rc) return rc;
      g += (uint64_t)items[i].r * (items[i].r + 1) / 2;
    }
    return GRID_OK;
  }
  Tables tb;
  uint64_t g_polys = 0;
  int rc = build_gram_tables(plan, items, nitems, k_split, tb, &g_polys);
  if (rc) return rc;
  const size_t core = core_bytes(witness_region(tb.s_polys, tb.pm_polys), tb.t_polys, d);
  if (workspace_bytes < core + tables_bytes(tb)) return GRID_ERR_INVALID_PARAMETERS;
  char* base = static_cast<char*>(workspace);
  uint32_t* s_hat = reinterpret_cast<uint32_t*>(base);
  unsigned long long* acc =
      reinterpret_cast<unsigned long long*>(base + round_up(tb.s_polys * d * 4, 256));
  unsigned* counters = reinterpret_cast<unsigned*>(base + round_up(tb.s_polys * d * 4, 256) +
                                                   round_up(tb.t_polys * d * 8, 256));
  // every witness to the evaluation domain, packed in item order (one launch
  // when the witnesses already lie packed in that order)
  bool packed = true;
  uint64_t off = 0;
  for (size_t i = 0; i < nitems && packed; ++i) {
    packed = items[i].s_offset == off;
    off += (uint64_t)items[i].r * items[i].n;
  }
  if (packed) {
    rc = launch_ntt(plan, MODE_FWD, S, nullptr, s_hat, tb.s_polys, st);
  } else {
    off = 0;
    for (size_t i = 0; i < nitems && !rc; ++i) {
      const uint64_t np = (uint64_t)items[i].r * items[i].n;
      rc = launch_ntt(plan, MODE_FWD, S + items[i].s_offset * d, nullptr, s_hat + off * d, np, st);
      off += np;
    }
  }
  if (rc) return rc;
  const MatDev* dm;
  const ItemDev* di;
  const TileDev* dt;
  const WorkDev* dw;
  const uint4* dx;
  rc = send_tables(tb, base + core, &dm, &di, &dt, &dw, &dx, st);
  if (rc) return rc;
  return run_product(plan, true, false, tb.class_begin, dm, di, dt, dw, (unsigned)tb.work.size(),
                     s_hat, 0, acc, counters, g_polys, G, st);
}

}  // extern "C"
