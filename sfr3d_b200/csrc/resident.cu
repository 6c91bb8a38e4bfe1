// Resident engine: mixed-precision Jacobi-PCG for large systems, with the
// FP32 inner iteration held on chip.
//
// B200 has a 126 MB L2 and up to 227 KB of shared memory per block.  The
// inner operator of a 128^3 pressure system, stored as SELL-32 with FP32
// couplings and 16-bit column offsets, is 75 MB and stays in L2 from one
// iteration to the next; the FP64 operator (150 MB) cannot.  One cooperative
// launch runs the whole solve with one block per SM.  Each block owns a
// contiguous range of SELL slices and keeps, for its rows, the inner
// residual, the FP32 solution increment, A p and (when it fits) the
// diagonal correction in shared memory (16 bytes a row).  The global traffic
// of an inner iteration is the operator (from L2), the gathers of p and the
// update of p; one exchange of partial sums separates its two phases, and a
// wait on the blocks whose p the next SpMV phase gathers ends it.
//
// Arithmetic.  PCG with the Jacobi preconditioner M = diag(1/ad) (Cg.c:47-209,
// PreCond.c:18-26) is CG on the symmetrically scaled system
//     (S A S) y = S b,   x = S y,   S = diag(1/sqrt(ad)),
// whose operator has a unit diagonal, so the inner iteration carries no
// preconditioner vector.  Its couplings are rounded to FP32 once; a per-row
// correction delta_i of the unit diagonal keeps the action of the rounded
// operator on S^-1 1 (the constant vector of the unscaled space, the
// near-null mode of a diffusion operator) equal to the FP64 one.  The 2-norm
// of a scaled residual is the reference's M-norm, ||S r||_2 = sqrt(r^T M r)
// (Cg.c:145).  Inner dot products accumulate in FP64.
//
// Reliable updates (Sleijpen & van der Vorst), as in mixed.cu: when the inner
// estimate has fallen by `delta` since the last refresh, or claims
// convergence, x += S xs in FP64, r = b - A x is recomputed with the FP64
// operator, the reference's criterion sqrt|(r, M r)| < tol sqrt|(b, M b)|
// (Cg.c:70-74, 145) is tested on it, and the inner residual restarts from
// fl32(S r) with the search direction kept.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>

#include "common.cuh"
#include "internal.h"
#include "persist.cuh"

namespace sfr {

namespace {

constexpr int kResNV = 2;          // values of the setup and refresh exchanges
constexpr int kResChunk = 6;       // slots of a row loaded before their gathers (a hex cell's faces)

// Block-to-block exchange without atomics.  Each block owns a 64-byte slot
// (eight 64-bit words) in each of three rotating buffers; epoch e uses buffer
// e % 3.  A block publishes its partial sums by storing every word of its slot
// with the two lowest bits of the FP64 pattern replaced by e & 3 (a change of
// at most 3 units in the last place, the same in every block); thread b of
// every block polls block b's words with relaxed loads until they carry the
// tag, and the block sums the partials in block order -- the same order in
// every block, so all blocks hold bit-identical totals.  Every word of buffer
// e % 3 was last written at epoch e - 3, whose tag differs from e's, and every
// block finished reading it before it published e - 2, so nothing needs
// emptying between uses.  The values travel
// inside the polled words: an exchange is one L2 round trip.
// kFence additionally makes every global write of every block before the
// call visible to every block after it (release fence before publishing,
// acquire fence after the poll); exchanges that only carry partial sums skip
// both.  Every wait is bounded: after spin_limit polls a block records
// SFR_TIMEOUT in *err; a block that sees *err set stops waiting.
struct alignas(64) ExSlot {
  unsigned long long v[8];
};

struct ExSync {
  ExSlot *slots;  // 3 * nblocks, zero at launch
  int *err;
  int nblocks;
  unsigned spin_limit;
};

__device__ __forceinline__ unsigned long long tagged(double v, unsigned tag) {
  return (static_cast<unsigned long long>(__double_as_longlong(v)) & ~3ull) | tag;
}

// Publishes NV block totals of acc and returns the totals over all blocks in
// tot (every thread).  `sm` holds 32 * (NV + 1) doubles; the block has at
// least nblocks threads.
template <int NV, bool kFence>
__device__ __forceinline__ bool exchange(const ExSync &f, unsigned &epoch, const double (&acc)[NV],
                                         double (&tot)[NV], double *sm) {
  static_assert(NV >= 1 && NV <= 8, "eight words a slot");
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    const double w = warp_sum(acc[v]);
    if (lane == 0) sm[v * 32 + warp] = w;
  }
  // with kFence, also orders the block's global writes before the release
  __syncthreads();
  ++epoch;
  const unsigned tag = epoch & 3u;
  ExSlot *cur = f.slots + static_cast<size_t>(epoch % 3u) * f.nblocks;
  if (warp == 0) {
    double t[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) t[v] = warp_sum(lane < nw ? sm[v * 32 + lane] : 0.0);
    if (lane == 0) {
      if (kFence) cuda::atomic_thread_fence(cuda::memory_order_release, cuda::thread_scope_device);
      // every word of the slot takes the new tag, also those this exchange
      // does not use: a word left untouched could carry a matching tag from
      // twelve epochs back when a later exchange polls it
#pragma unroll
      for (int v = 0; v < 8; ++v)
        cuda::atomic_ref<unsigned long long, cuda::thread_scope_device>(cur[blockIdx.x].v[v])
            .store(tagged(v < NV ? t[v < NV ? v : 0] : 0.0, tag), cuda::memory_order_relaxed);
    }
  }
  // thread b watches block b
  const bool watcher = static_cast<int>(threadIdx.x) < f.nblocks;
  double val[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) val[v] = 0.0;
  int seen = !watcher;
  int ok = 1;
  cuda::atomic_ref<int, cuda::thread_scope_device> err(*f.err);
  for (unsigned spins = 0;; ++spins) {
    if (!seen) {
      int all = 1;
#pragma unroll
      for (int v = 0; v < NV; ++v) {
        const unsigned long long u =
            cuda::atomic_ref<unsigned long long, cuda::thread_scope_device>(cur[threadIdx.x].v[v])
                .load(cuda::memory_order_relaxed);
        val[v] = __longlong_as_double(static_cast<long long>(u));
        all &= (u & 3ull) == tag;
      }
      seen = all;
    }
    if (__syncthreads_and(seen)) break;
    // every exit below is taken by the whole block together
    if ((spins & 63u) == 63u &&
        __syncthreads_or(threadIdx.x == 0 && err.load(cuda::memory_order_relaxed) != 0)) {
      ok = 0;
      break;
    }
    if (spins > f.spin_limit) {
      if (threadIdx.x == 0) {
        int expected = 0;
        err.compare_exchange_strong(expected, SFR_TIMEOUT, cuda::memory_order_relaxed);
      }
      ok = 0;
      break;
    }
  }
  if (kFence && watcher)
    cuda::atomic_thread_fence(cuda::memory_order_acquire, cuda::thread_scope_device);
  // totals in block order: lanes within a warp, then warps in order
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    const double w = warp_sum(val[v]);
    if (lane == 0) sm[v * 32 + warp] = w;
  }
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      const double w = warp_sum(lane < nw ? sm[v * 32 + lane] : 0.0);
      if (lane == 0) sm[NV * 32 + v] = w;
    }
  }
  __syncthreads();
#pragma unroll
  for (int v = 0; v < NV; ++v) tot[v] = sm[NV * 32 + v];
  return ok != 0;
}

// A barrier that also publishes the global writes before it.
__device__ __forceinline__ bool exchange_barrier(const ExSync &f, unsigned &epoch, double *sm) {
  const double z[1] = {0.0};
  double t[1];
  return exchange<1, true>(f, epoch, z, t, sm);
}

// The wait after an iteration's update of p (neighbour_wait, common.cuh):
// the next SpMV phase of a block gathers p only at the columns of its own
// rows, and the global exchange after each SpMV phase already keeps every
// block from rewriting p while another still reads it.
struct NbSync {
  unsigned *ticks;  // 16 words a block, zero at launch; word 0 counts updates
};

// The range [red_i[0], red_i[1]] of blocks owning the columns this block's
// rows gather from (block_slices's partition of nslices slices over
// gridDim.x blocks), in shared memory.
__device__ __forceinline__ void gather_blocks(const int *sm_sp, const int16_t *off, int s0,
                                              int s1, int nslices, int *red_i) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  int cmin = s0 * kWarp, cmax = s1 * kWarp - 1;
  for (int s = s0 + warp; s < s1; s += nw) {
    const int base = sm_sp[s - s0], end = sm_sp[s - s0 + 1];
    const int row = s * kWarp + lane;
    for (int e = base + lane; e < end; e += kWarp) {
      const int c = row + static_cast<int>(__ldcg(off + e));  // slot e is lane's
      cmin = min(cmin, c);
      cmax = max(cmax, c);
    }
  }
  if (threadIdx.x == 0) {
    red_i[0] = cmin;
    red_i[1] = cmax;
  }
  __syncthreads();
  atomicMin(red_i, cmin);
  atomicMax(red_i + 1, cmax);
  __syncthreads();
  const int lo = min(owner_block(red_i[0], nslices), static_cast<int>(blockIdx.x));
  const int hi = max(owner_block(red_i[1], nslices), static_cast<int>(blockIdx.x));
  __syncthreads();
  if (threadIdx.x == 0) {
    red_i[0] = lo;
    red_i[1] = hi;
  }
  __syncthreads();
}

struct ResArgs {
  int n, nslices;
  const int *sptr;
  // inner operator: FP32 scaled couplings and col - row offsets per slot,
  // per row the correction of the unit diagonal (nslices * 32 entries)
  const float *val;
  const int16_t *off;
  const float *delta;
  // FP64 operator (refreshes and the final residuals)
  const int *col64;
  const double *val64;
  const double *diag;
  const double *b;
  double *x;
  float *p;  // search direction, nslices * 32 entries (padding rows stay 0)
  ExSync ex;
  NbSync nb;  // ticks null: the update of p ends with a full barrier
  SolveOut *out;
  double tol, rdelta;
  unsigned maxit;
  int newx;
};

// (A x)[row] with the FP64 operator; the matrix streams (evict-first) so the
// FP32 operator keeps its place in L2.
__device__ __forceinline__ double row_fp64(const ResArgs &a, int s, int lane, int row) {
  const int base = __ldg(a.sptr + s);
  const int w = (__ldg(a.sptr + s + 1) - base) >> 5;
  double y = ld_vec(a.diag + row) * ld_vec(a.x + row);
  const int *c = a.col64 + base + lane;
  const double *v = a.val64 + base + lane;
#pragma unroll 2
  for (int e = 0; e < w; ++e) y = fma(ld_stream(v + e * kWarp), ld_vec(a.x + ld_stream(c + e * kWarp)), y);
  return y;
}

// (A_s p)[row] for one slice of the block (base and width from the block's
// slice pointers in shared memory), accumulated in FP64 from the unit
// diagonal: p_row (1 + delta_row) + sum_e val_e p_(row + off_e).  A chunk of
// slots -- offsets, couplings -- is loaded before its gathers, so a slice
// costs two dependent L2 round trips.
__device__ __forceinline__ double row_scaled(const ResArgs &a, int base, int w, int lane,
                                             int row, float p_row, float dl) {
  double y = fma(static_cast<double>(dl), static_cast<double>(p_row), static_cast<double>(p_row));
  const float *v = a.val + base + lane;
  const int16_t *o = a.off + base + lane;
  for (int e0 = 0; e0 < w; e0 += kResChunk) {
    int jj[kResChunk];
    float vv[kResChunk];
#pragma unroll
    for (int u = 0; u < kResChunk; ++u)
      if (e0 + u < w) {
        jj[u] = row + static_cast<int>(__ldcg(o + (e0 + u) * kWarp));
        vv[u] = __ldcg(v + (e0 + u) * kWarp);
      }
#pragma unroll
    for (int u = 0; u < kResChunk; ++u)
      if (e0 + u < w)
        y = fma(static_cast<double>(vv[u]), static_cast<double>(ld_vec(a.p + jj[u])), y);
  }
  return y;
}

// This block's rows, slice by slice: warp w takes slices s0 + w, s0 + w + NW,
// ...; defines s (slice), row and lr (row within the block's shared state).
#define SFR_RES_FOR(s, row, lr)                                             \
  for (int s = s0 + warp; s < s1; s += NW)                                  \
    for (int row = s * kWarp + lane, lr = row - r0, once_ = 1; once_; once_ = 0)

// Refresh: r = b - A x in FP64 for this block's rows, r_s = fl32(S r) into
// shared memory (and p = r_s on the first call), xs = 0.
// tot[0] = (r, M r) = sum r^2 / ad, tot[1] = (r_s, r_s).  The first call
// publishes p (and x) to every block.
template <int kT>
__device__ __forceinline__ bool refresh(const ResArgs &a, int s0, int s1, int r0, float *sm_r,
                                        float *sm_xs, bool first, unsigned &epoch, double *red,
                                        double (&tot)[kResNV]) {
  constexpr int NW = kT / kWarp;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double acc[kResNV] = {0.0, 0.0};
  SFR_RES_FOR(s, row, lr) {
    float rs = 0.0f;
    if (row < a.n) {
      const double d = ld_vec(a.diag + row);
      const double r = ld_vec(a.b + row) - row_fp64(a, s, lane, row);
      rs = __double2float_rn(r / sqrt(d));
      acc[0] += r * (r / d);
      acc[1] += static_cast<double>(rs) * static_cast<double>(rs);
    }
    sm_r[lr] = rs;
    sm_xs[lr] = 0.0f;
    if (first) st_vec(a.p + row, rs);
  }
  return first ? exchange<kResNV, true>(a.ex, epoch, acc, tot, red)
               : exchange<kResNV, false>(a.ex, epoch, acc, tot, red);
}

// x += S (xs + a_pend p) in FP64 for this block's rows; xs = 0.  a_pend is
// the step of the current direction not yet added to xs.
template <int kT>
__device__ __forceinline__ void fold(const ResArgs &a, int s0, int s1, int r0, float *sm_xs,
                                     float a_pend) {
  constexpr int NW = kT / kWarp;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  SFR_RES_FOR(s, row, lr) {
    if (row < a.n) {
      const float xs = fmaf(a_pend, ld_vec(a.p + row), sm_xs[lr]);
      st_vec(a.x + row, ld_vec(a.x + row) + static_cast<double>(xs) / sqrt(ld_vec(a.diag + row)));
    }
    sm_xs[lr] = 0.0f;
  }
}

// Iteration j (one exchange of partial sums, one wait on the neighbours):
//   q = A_s p ; (p, q), (r, q), (q, q), (r, r)                 [exchange]
//   alpha = (r, r) / (p, q)
//   (r', r') = (r, r) - 2 alpha (r, q) + alpha^2 (q, q)   for r' = r - alpha q
//   (refresh when due)
//   r = r - alpha q ; xs += alpha p ; p = r + beta p            [wait]
// The norm of the next residual follows from dot products the SpMV phase
// already forms, so the residual update needs no exchange of its own; it is
// accumulated in FP64 and only decides beta and when to refresh.  The next
// SpMV phase recomputes (r, r) from the stored residual, so the recurrence's
// alpha always uses the norm of the r it holds.
template <int kT, bool kDeltaShared>
__global__ void __launch_bounds__(kT, 1) pcg_resident_kernel(ResArgs a) {
  constexpr int NW = kT / kWarp;
  extern __shared__ float sm_dyn[];
  __shared__ double red[32 * 5];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int s0, s1;
  block_slices(a.nslices, &s0, &s1);
  const int r0 = s0 * kWarp;
  const int rows = (s1 - s0) * kWarp;
  float *sm_r = sm_dyn;          // inner residual (scaled)
  float *sm_xs = sm_r + rows;    // FP32 solution increment (scaled)
  float *sm_q = sm_xs + rows;    // A_s p
  float *sm_d = sm_q + rows;     // diagonal correction (kDeltaShared)
  int *sm_sp = reinterpret_cast<int *>(sm_q + (kDeltaShared ? 2 : 1) * rows);  // slice pointers
  unsigned epoch = 0;
  for (int i = threadIdx.x; i <= s1 - s0; i += kT) sm_sp[i] = __ldg(a.sptr + s0 + i);
  if (kDeltaShared)
    for (int lr = threadIdx.x; lr < rows; lr += kT) sm_d[lr] = __ldcg(a.delta + r0 + lr);
  __syncthreads();
  // the blocks whose p this block's SpMV phases gather
  __shared__ int nb_range[2];
  nb_range[0] = 0;
  nb_range[1] = kT;  // no neighbour waits unless the range is computed
  if (a.nb.ticks) gather_blocks(sm_sp, a.off, s0, s1, a.nslices, nb_range);

  // setup: x0, (b, M b), (b, b)
  double bm = 0.0, bnorm = 0.0;
  {
    double acc[kResNV] = {0.0, 0.0}, tot[kResNV];
    for (int lr = threadIdx.x; lr < rows; lr += kT) {
      const int row = r0 + lr;
      if (row < a.n) {
        if (a.newx) st_vec(a.x + row, 0.0);
        const double bk = ld_vec(a.b + row);
        acc[0] += bk * (bk / ld_vec(a.diag + row));
        acc[1] += bk * bk;
      }
    }
    if (!exchange<kResNV, true>(a.ex, epoch, acc, tot, red)) return;
    bm = tot[0];
    bnorm = sqrt(tot[1]);
  }
  const double conv = a.tol * sqrt(fabs(bm));
  double d = 0.0, rmax;  // d: (r, r) of the residual the last direction was built from
  bool act = true;
  int status = SFR_OK, refine = 0;
  unsigned iters = 0;
  {
    double tot[kResNV];
    if (!refresh<kT>(a, s0, s1, r0, sm_r, sm_xs, true, epoch, red, tot)) return;
    rmax = sqrt(fabs(tot[0]));
    if (rmax < conv) act = false;
  }
  float a_pend = 0.0f;  // alpha of the current direction, not yet in xs
  unsigned j = 0;
  for (; j < a.maxit && act; ++j) {
    // q = A_s p and the four dot products
    double alpha, di;
    {
      double acc[4] = {0.0, 0.0, 0.0, 0.0}, tot[4];
      auto dots = [&](int lr, float qi, float pr) {
        const float ri = sm_r[lr];
        sm_q[lr] = qi;
        acc[0] += static_cast<double>(qi) * static_cast<double>(pr);
        acc[1] += static_cast<double>(qi) * static_cast<double>(ri);
        acc[2] += static_cast<double>(qi) * static_cast<double>(qi);
        acc[3] += static_cast<double>(ri) * static_cast<double>(ri);
      };
      SFR_RES_FOR(s, row, lr) {
        const int base = sm_sp[s - s0];
        const int w = (sm_sp[s - s0 + 1] - base) >> 5;
        const float pr = ld_vec(a.p + row);
        const float dl = kDeltaShared ? sm_d[lr] : __ldcg(a.delta + row);
        dots(lr, __double2float_rn(row_scaled(a, base, w, lane, row, pr, dl)), pr);
      }
      if (!exchange<4, false>(a.ex, epoch, acc, tot, red)) return;
      d = tot[3];
      alpha = d / tot[0];
      di = d - 2.0 * alpha * tot[1] + alpha * alpha * tot[2];
      if (!isfinite(alpha) || !isfinite(di)) {
        act = false;
        status = SFR_BREAKDOWN;
        iters = j + 1;
        break;
      }
      a_pend = static_cast<float>(alpha);
    }
    const double est = sqrt(fabs(di));
    double beta;
    bool step = true;  // r -= alpha q still to do
    if (est < a.rdelta * rmax || est < conv) {
      // reliable update: x += S (xs + alpha p), r = fl32(S (b - A x))
      fold<kT>(a, s0, s1, r0, sm_xs, a_pend);
      a_pend = 0.0f;
      step = false;
      if (!exchange_barrier(a.ex, epoch, red)) return;
      double tot[kResNV];
      if (!refresh<kT>(a, s0, s1, r0, sm_r, sm_xs, false, epoch, red, tot)) return;
      ++refine;
      const double tr = sqrt(fabs(tot[0]));
      if (tr < conv) {
        act = false;
        iters = j + 1;
        break;
      }
      beta = tot[1] / d;
      rmax = tr;
    } else {
      beta = di / d;
    }
    // r -= alpha q ; xs += alpha p ; p = r + beta p
    {
      const float bf = static_cast<float>(beta);
      SFR_RES_FOR(s, row, lr) {
        const float pr = ld_vec(a.p + row);
        const float ri = step ? fmaf(-a_pend, sm_q[lr], sm_r[lr]) : sm_r[lr];
        sm_r[lr] = ri;
        sm_xs[lr] = fmaf(a_pend, pr, sm_xs[lr]);
        st_vec(a.p + row, fmaf(bf, pr, ri));
      }
      a_pend = 0.0f;
      // one update of p an iteration: iteration j publishes its (j + 1)-th
      if (nb_range[1] - nb_range[0] < kT) {
        if (!neighbour_wait(a.nb.ticks, a.ex.err, a.ex.spin_limit, j + 1, nb_range[0],
                            nb_range[1]))
          return;
      } else if (!exchange_barrier(a.ex, epoch, red)) {
        return;
      }
    }
  }
  if (act) {  // iteration cap
    status = SFR_MAXIT;
    iters = j + 1;
  }
  if (status != SFR_OK) {  // fold the last increment (a converged solve has folded it)
    fold<kT>(a, s0, s1, r0, sm_xs, a_pend);
    if (!exchange_barrier(a.ex, epoch, red)) return;
  }
  // xKx, ||x||, ||b - Ax||_M, ||b - Ax|| (Cg.c:155-176)
  double acc[4] = {0.0, 0.0, 0.0, 0.0}, tot[4];
  SFR_RES_FOR(s, row, lr) {
    (void)lr;
    if (row < a.n) {
      const double y = row_fp64(a, s, lane, row);
      const double xk = ld_vec(a.x + row);
      const double rk = ld_vec(a.b + row) - y;
      acc[0] += xk * y;
      acc[1] += xk * xk;
      acc[2] += rk * (rk / ld_vec(a.diag + row));
      acc[3] += rk * rk;
    }
  }
  if (!exchange<4, false>(a.ex, epoch, acc, tot, red)) return;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    SolveOut o;
    o.iters = static_cast<int>(iters);
    o.status = status;
    o.xKx = tot[0];
    o.norm_x = sqrt(tot[1]);
    o.norm_r_m = sqrt(fabs(tot[2]));
    o.norm_r = sqrt(tot[3]);
    o.conv = conv;
    o.bnorm = bnorm;
    o.refinements = refine;
    o.inner_iters = static_cast<int>(iters);
    o.team_ms = 0.0;
    *a.out = o;
  }
}

#undef SFR_RES_FOR

// Scaled FP32 operator from the FP64 SELL values and the diagonal:
//   val_e = fl32(a_e / sqrt(ad_row ad_col)),
//   delta_row = -sum_e (val_e - a_e / sqrt(ad_row ad_col)) sqrt(ad_col / ad_row).
// *bad is set when a diagonal entry is not positive and finite.
__global__ void scaled_operator_kernel(const int *sptr, const int *col, const double *val,
                                       const double *diag, int n, int nslices, float *sval,
                                       float *delta, int *bad) {
  const int stride = gridDim.x * blockDim.x;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nslices * kWarp; t += stride) {
    const int s = t >> 5, lane = t & 31, row = t;
    const int base = sptr[s];
    const int w = (sptr[s + 1] - base) >> 5;
    if (row >= n) {
      for (int k = 0; k < w; ++k) sval[base + k * kWarp + lane] = 0.0f;
      delta[row] = 0.0f;
      continue;
    }
    const double di = diag[row];
    if (!(di > 0.0) || !isfinite(di)) {
      atomicExch(bad, 1);
      continue;
    }
    const double si = 1.0 / sqrt(di);
    double acc = 0.0;
    for (int k = 0; k < w; ++k) {
      const int e = base + k * kWarp + lane;
      const int c = col[e];
      const double dc = diag[c];
      const double sc = dc > 0.0 ? sqrt(dc) : 0.0;
      const double exact = sc > 0.0 ? val[e] * si / sc : 0.0;
      const float f = __double2float_rn(exact);
      sval[e] = f;
      acc += (static_cast<double>(f) - exact) * sc;
    }
    delta[row] = __double2float_rn(-acc * si);
  }
}

int ensure_scaled_operator(sfr_system *s, cudaStream_t st) {
  const int64_t nslots = s->A.nslots;
  if (!s->d_rval) {
    const size_t ns = static_cast<size_t>(std::max<int64_t>(nslots, 1));
    if (cudaMalloc(&s->d_rval, sizeof(float) * ns) != cudaSuccess) return SFR_CUDA_ERROR;
    const size_t rows = static_cast<size_t>(std::max(s->A.nslices, 1)) * kWarp;
    if (cudaMalloc(&s->d_rdelta, sizeof(float) * rows) != cudaSuccess) return SFR_CUDA_ERROR;
    if (cudaMalloc(&s->d_rbad, sizeof(int)) != cudaSuccess) return SFR_CUDA_ERROR;
    s->bytes += static_cast<int64_t>(sizeof(float) * ns +
                                     sizeof(float) * rows + sizeof(int));
  }
  if (s->resident_epoch == s->values_epoch) return SFR_OK;
  if (cudaMemsetAsync(s->d_rbad, 0, sizeof(int), st) != cudaSuccess) return SFR_CUDA_ERROR;
  const int grid = static_cast<int>(
      std::min<int64_t>((static_cast<int64_t>(s->A.nslices) * kWarp + 255) / 256, 8192));
  scaled_operator_kernel<<<std::max(grid, 1), 256, 0, st>>>(
      s->A.sptr, s->A.col, s->A.val, s->d_diag, s->n, s->A.nslices, s->d_rval, s->d_rdelta,
      s->d_rbad);
  if (cudaGetLastError() != cudaSuccess) return SFR_CUDA_ERROR;
  int bad = 0;
  if (cudaMemcpyAsync(&bad, s->d_rbad, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return SFR_CUDA_ERROR;
  s->resident_epoch = s->values_epoch;
  s->resident_ok = bad == 0;
  return SFR_OK;
}

// Launch shape: one block of 1024 threads per SM.  Shared state: 12 bytes per
// row (inner residual, FP32 solution increment, A p), 16 when the diagonal
// correction fits there too, and the block's slice pointers.
constexpr int kResThreads = 1024;

int max_smem_optin(int device) {
  int v = 0;
  if (cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, device) != cudaSuccess)
    return 0;
  return v;
}

// Dynamic shared memory of a block with `per_row` bytes of state a row, or 0
// when a block's rows do not fit.
size_t block_smem(int nslices, int grid, int device, int per_row) {
  const int per_block = (nslices + grid - 1) / grid;
  const size_t bytes = static_cast<size_t>(per_block) * kWarp * per_row +
                       sizeof(int) * (static_cast<size_t>(per_block) + 2);
  // the kernel's static shared memory (reductions, 1,280 bytes) comes on top
  if (bytes + 1536 > static_cast<size_t>(max_smem_optin(device))) return 0;
  return std::max<size_t>(bytes, 16);
}

// Self-test of the exchange's bounded wait: the grid exchanges one partial
// sum, except its last `absent` blocks, which leave before publishing, so
// the others' polls of their words run out and record SFR_TIMEOUT.
__global__ void k_res_wait_selftest(int absent, ExSync f) {
  __shared__ double red[32 * 2];
  if (static_cast<int>(blockIdx.x) >= static_cast<int>(gridDim.x) - absent) return;
  unsigned epoch = 0;
  const double acc[1] = {1.0};
  double tot[1];
  (void)exchange<1, false>(f, epoch, acc, tot, red);
}

}  // namespace

int wait_selftest_resident(int32_t absent, uint32_t spin_limit, cudaStream_t st) {
  constexpr int kGrid = 4;
  if (absent < 0 || absent >= kGrid) return SFR_BAD_INPUT;
  const size_t slots = sizeof(ExSlot) * 3 * kGrid;
  char *buf = nullptr;
  if (cudaMalloc(&buf, slots + 64) != cudaSuccess) return SFR_CUDA_ERROR;
  ExSync f;
  f.slots = reinterpret_cast<ExSlot *>(buf);
  f.err = reinterpret_cast<int *>(buf + slots);
  f.nblocks = kGrid;
  f.spin_limit = spin_limit;
  void *params[] = {&absent, &f};
  int err = 0;
  cudaError_t ce = cudaMemsetAsync(buf, 0, slots + 64, st);
  if (ce == cudaSuccess)
    ce = cudaLaunchCooperativeKernel(reinterpret_cast<void *>(k_res_wait_selftest), dim3(kGrid),
                                     dim3(128), params, 0, st);
  if (ce == cudaSuccess) ce = cudaMemcpyAsync(&err, f.err, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
  cudaFree(buf);
  if (ce != cudaSuccess) {
    set_last_error(cudaGetErrorString(ce));
    return SFR_CUDA_ERROR;
  }
  return err;
}

bool resident_fits(sfr_system *s) {
  if (!s->A.off) return false;  // bandwidth above 32767: no 16-bit column offsets
  return block_smem(s->A.nslices, std::max(1, num_sms(s->device)), s->device, 12) != 0;
}

int solve_resident(sfr_system *s, const double *d_b, double *d_x, double tol, uint32_t maxit,
                   int32_t newx, cudaStream_t st, sfr_solve_info *info) {
  if (maxit == 0) return SFR_BAD_INPUT;
  if (!resident_fits(s)) return SFR_UNSUPPORTED;
  int rc = ensure_scaled_operator(s, st);
  if (rc != SFR_OK) return rc;
  if (!s->resident_ok) return SFR_UNSUPPORTED;  // Jacobi scaling needs ad > 0
  // a block per SM, fewer for small systems (a slice per warp at least):
  // the cost of an exchange grows with the blocks taking part
  const int warps = kResThreads / kWarp;
  const int grid = std::max(1, std::min(num_sms(s->device), (s->A.nslices + warps - 1) / warps));
  // the diagonal correction in shared memory when it fits (the FP32 operator
  // then keeps more of L2 to itself), else read with the couplings
  size_t smem = block_smem(s->A.nslices, grid, s->device, 16);
  const bool dshared = smem != 0;
  if (!dshared) smem = block_smem(s->A.nslices, grid, s->device, 12);
  if (!smem) return SFR_UNSUPPORTED;
  void (*kern)(ResArgs) = dshared ? pcg_resident_kernel<kResThreads, true>
                                  : pcg_resident_kernel<kResThreads, false>;
  if (cudaFuncSetAttribute(reinterpret_cast<const void *>(kern),
                           cudaFuncAttributeMaxDynamicSharedMemorySize,
                           static_cast<int>(smem)) != cudaSuccess)
    return SFR_CUDA_ERROR;
  int occ = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, kResThreads, smem) !=
          cudaSuccess ||
      occ < 1)
    return SFR_UNSUPPORTED;

  auto align = [](size_t v) { return (v + 255) & ~static_cast<size_t>(255); };
  const size_t p_bytes = align(sizeof(float) * static_cast<size_t>(s->A.nslices) * kWarp);
  const size_t part_bytes = align(sizeof(ExSlot) * 3 * static_cast<size_t>(grid));
  const size_t ctl_bytes = 256;
  const size_t out_bytes = align(sizeof(SolveOut));
  const size_t tick_bytes = align(64 * static_cast<size_t>(grid));
  rc = ensure_workspace(s, p_bytes + part_bytes + ctl_bytes + out_bytes + tick_bytes);
  if (rc != SFR_OK) return rc;
  char *base = static_cast<char *>(s->ws.base);

  ResArgs a;
  std::memset(&a, 0, sizeof(a));
  a.n = s->n;
  a.nslices = s->A.nslices;
  a.sptr = s->A.sptr;
  a.val = s->d_rval;
  a.off = s->A.off;
  a.delta = s->d_rdelta;
  a.col64 = s->A.col;
  a.val64 = s->A.val;
  a.diag = s->d_diag;
  a.b = d_b;
  a.x = d_x;
  a.p = reinterpret_cast<float *>(base);
  base += p_bytes;
  a.ex.slots = reinterpret_cast<ExSlot *>(base);
  unsigned *ctl = reinterpret_cast<unsigned *>(base + part_bytes);
  a.ex.err = reinterpret_cast<int *>(ctl);
  a.ex.nblocks = grid;
  a.ex.spin_limit = 1u << 22;
  a.out = reinterpret_cast<SolveOut *>(base + part_bytes + ctl_bytes);
  a.nb.ticks = reinterpret_cast<unsigned *>(base + part_bytes + ctl_bytes + out_bytes);
  a.tol = tol;
  a.rdelta = reliable_delta_resident();
  a.maxit = maxit;
  a.newx = newx;

  // padding rows of p must read as 0; epochs restart at 0 in every launch,
  // with every exchange word untagged
  if (cudaMemsetAsync(a.p, 0, p_bytes, st) != cudaSuccess) return SFR_CUDA_ERROR;
  if (cudaMemsetAsync(a.ex.slots, 0, part_bytes + ctl_bytes, st) != cudaSuccess ||
      cudaMemsetAsync(a.nb.ticks, 0, tick_bytes, st) != cudaSuccess)
    return SFR_CUDA_ERROR;
  cudaEvent_t e0, e1;
  if (cudaEventCreate(&e0) != cudaSuccess) return SFR_CUDA_ERROR;
  if (cudaEventCreate(&e1) != cudaSuccess) {
    cudaEventDestroy(e0);
    return SFR_CUDA_ERROR;
  }
  void *params[] = {&a};
  cudaEventRecord(e0, st);
  const cudaError_t le = cudaLaunchCooperativeKernel(reinterpret_cast<void *>(kern), dim3(grid),
                                                     dim3(kResThreads), params, smem, st);
  cudaEventRecord(e1, st);
  SolveOut out{};
  int err = 0;
  cudaError_t ce = le;
  if (ce == cudaSuccess)
    ce = cudaMemcpyAsync(&out, a.out, sizeof(SolveOut), cudaMemcpyDeviceToHost, st);
  if (ce == cudaSuccess)
    ce = cudaMemcpyAsync(&err, a.ex.err, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
  float ms = 0.f;
  if (ce == cudaSuccess) cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (ce != cudaSuccess) {
    set_last_error(cudaGetErrorString(ce));
    return SFR_CUDA_ERROR;
  }
  if (err != 0) return err;
  if (info) {
    std::memset(info, 0, sizeof(*info));
    info->iters = out.iters;
    info->status = out.status;
    info->xKx = out.xKx;
    info->norm_x = out.norm_x;
    info->norm_r = out.norm_r;
    info->norm_r_m = out.norm_r_m;
    info->conv = out.conv;
    info->seconds = ms * 1e-3;
    info->refinements = out.refinements;
    info->inner_iters = out.inner_iters;
    info->relres = out.bnorm > 0 ? out.norm_r / out.bnorm : 0.0;
  }
  return out.status;
}

}  // namespace sfr
