// Vocabulary shared by the persistent (one cooperative launch per solve)
// Krylov kernels: launch shape, result record, per-block row loop, and the
// partial -> barrier -> total reduction step.
#pragma once

#include "common.cuh"

namespace sfr {

constexpr int kMaxK = 4;            // right-hand sides per launch
constexpr int kThreads = 512;       // threads per block of a persistent solve
constexpr int kMaxNV = 4 * kMaxK;   // values reduced together at most

struct SolveOut {
  int iters;
  int status;
  double xKx, norm_x, norm_r, norm_r_m, conv;
  double bnorm;        // ||b||_2
  int refinements;     // mixed: reliable updates (FP64 residual recomputations)
  int inner_iters;     // mixed: FP32 iterations
};

// Rows owned by this thread: warps of the block walk the block's slices, a
// lane takes one row of its slice.  Defines s_ (slice) and row_ (row < n).
#define SFR_FOR_OWN_ROWS(s0, s1)                                                \
  for (int s_ = (s0) + (threadIdx.x >> 5); s_ < (s1); s_ += (blockDim.x >> 5)) \
    for (int row_ = s_ * kWarp + (threadIdx.x & 31), once_ = 1; once_; once_ = 0) \
      if (row_ < n)

// Write NV block partials into the next slot, wait at the grid barrier, and
// total them (same order in every block).  False when the barrier failed.
template <int NV>
__device__ __forceinline__ bool reduce_step(double *part, const GridSync &gs, int &slot,
                                            double (&acc)[NV], double (&tot)[NV], double *sm) {
  const int G = gridDim.x;
  double *base = part + static_cast<size_t>(slot) * kMaxNV * G;
  block_partials<NV>(acc, base, G, sm);
  if (!grid_sync(gs)) return false;
  grid_totals<NV>(base, G, G, tot, sm);
  slot ^= 1;
  return true;
}

}  // namespace sfr
