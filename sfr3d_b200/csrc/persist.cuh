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
  double team_ms;      // batched launch: the team's time from launch to its result
};

// The GPU's nanosecond clock (comparable across SMs).
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Rows owned by this thread: warps of the block walk the block's slices, a
// lane takes one row of its slice.  Defines s_ (slice) and row_ (row < n).
#define SFR_FOR_OWN_ROWS(s0, s1)                                                \
  for (int s_ = (s0) + (threadIdx.x >> 5); s_ < (s1); s_ += (blockDim.x >> 5)) \
    for (int row_ = s_ * kWarp + (threadIdx.x & 31), once_ = 1; once_; once_ = 0) \
      if (row_ < n)

// A team is the set of blocks that solve one system together.  A launch for
// one system is a single team of every block; a batched launch gives each
// system its own team, with its own slice range, reductions over its own
// blocks and its own barrier, so the systems run independently.
struct TeamTable {
  const int4 *block;   // per block {first slice, end slice, first block, end block}
  const int2 *sys;     // per block {system, end row}
  unsigned int *bar;   // per system {barrier count, generation}
};

struct Team {
  int s0, s1;   // this block's slices
  int b0, b1;   // the team's blocks
  int sys;      // system index (0 for a single system)
  int row_end;  // rows of the system end here (global row numbering)
  GridSync gs;  // the team's barrier
  unsigned long long t0;  // this block's start (global_ns)
};

__device__ __forceinline__ Team make_team(const TeamTable &tt, const GridSync &global,
                                          int nslices, int n) {
  Team t;
  t.t0 = global_ns();
  t.gs = global;
  if (!tt.block) {
    block_slices(nslices, &t.s0, &t.s1);
    t.b0 = 0;
    t.b1 = gridDim.x;
    t.sys = 0;
    t.row_end = n;
  } else {
    const int4 e = tt.block[blockIdx.x];
    const int2 y = tt.sys[blockIdx.x];
    t.s0 = e.x;
    t.s1 = e.y;
    t.b0 = e.z;
    t.b1 = e.w;
    t.sys = y.x;
    t.row_end = y.y;
    t.gs.count = tt.bar + 2 * t.sys;
    t.gs.gen = tt.bar + 2 * t.sys + 1;
    t.gs.nblocks = static_cast<unsigned>(t.b1 - t.b0);
  }
  return t;
}

// NV block partials -> the team's barrier -> totals over the team's blocks
// in a fixed order.  False when the barrier failed.
template <int NV>
__device__ __forceinline__ bool reduce_team(double *part, const Team &t, int &slot,
                                            double (&acc)[NV], double (&tot)[NV], double *sm) {
  const int G = gridDim.x;
  double *base = part + static_cast<size_t>(slot) * kMaxNV * G;
  block_partials<NV>(acc, base, G, sm);
  if (!grid_sync(t.gs)) return false;
  grid_totals<NV>(base + t.b0, G, t.b1 - t.b0, tot, sm);
  slot ^= 1;
  return true;
}

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
