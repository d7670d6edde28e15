// Work tables of the grouped (batched) contractions, shared by the CUDA-core
// kernel (batch.cu) and the tensor-core kernel (grouped_tc.cu).
//
// A tile groups up to 128 rows of X: instances of one matrix (commitments:
// row = one instance's witness s_i, its n_i evaluation polys at s_off, outputs
// at t_off + matrix row), or the r witness rows of one Gram instance (matrix =
// kUpperTile: X = Y, row i at s_off = the instance's offset + i n, every row's
// t_off = the instance's first output poly, outputs in garbage_index order). A
// work item is (tile, K range, evaluation group).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "grid_internal.h"

namespace grid {

constexpr uint32_t kUpperTile = 0xFFFFFFFFu;  // TileDev::matrix of a Gram tile

struct MatDev {
  const uint32_t* evals;
  const uint32_t* evals_pm;  // [point][row][ld] (point-major engine), or null
  uint32_t rows, ld;         // ld: row stride in polys
};
struct ItemDev {
  unsigned long long s_off, t_off;
  uint32_t n, pad;
};
struct TileDev {
  uint32_t first, count, matrix, kmax;
};
struct WorkDev {
  uint32_t tile, k0, k1, eg;
};

// Evaluation points per work item of the tensor-core kernel, by the Y rows of
// the tile (matrix rows, or the Gram's r): 4 for <= 16 rows, else 2.
__host__ __device__ constexpr int tc_points(uint32_t yrows) { return yrows <= 16 ? 4 : 2; }
constexpr int kTcMaxTileRows = 128;  // X rows per tile (the MMA's M)
constexpr int kTcMaxYRows = 64;      // Y rows (Gram r, matrix rows) per tile
constexpr uint32_t kTcMaxK = 8192;   // K words per work item: 4 * 8192 * 255^2 < 2^31

// Tile classes of the tensor-core kernel (one kernel instantiation each): dense
// tiles of <= 16 or <= 32 matrix rows, Gram tiles of r <= 16, 32 or 64.
enum TcClass : int { TC_D16 = 0, TC_D32, TC_U16, TC_U32, TC_U64, TC_CLASSES };
int tc_class(const TileDev& tile, const MatDev* host_mats);

// Persistent tensor-core kernel over one class's work list: every work item adds
// its canonical partial sums into the 64-bit accumulators acc[out poly][point].
int launch_batch_tc(const grid_gpu_plan* p, int cls, const WorkDev* work, unsigned nwork,
                    const TileDev* tiles, const ItemDev* items, const MatDev* mats,
                    const uint32_t* s_hat, unsigned long long* acc, unsigned* counter,
                    cudaStream_t s);

// grouped_pm.cu: the dense classes (TC_D16, TC_D32) over point-major
// evaluations s_pm [point][ps] (ps >= the packed witness polys, a multiple of 4),
// one evaluation point per work item (WorkDev::eg = the point).
int launch_batch_pm(const grid_gpu_plan* p, int cls, const WorkDev* work, unsigned nwork,
                    const TileDev* tiles, const ItemDev* items, const MatDev* mats,
                    const uint32_t* s_pm, uint64_t ps, unsigned long long* acc, cudaStream_t s);

}  // namespace grid
