// Persistent Krylov solvers (Jacobi-PCG, Jacobi-BiCGSTAB) for sm_100a.
//
// One cooperative launch runs a whole solve: every block owns a contiguous
// range of SELL slices, each phase (SpMV, vector update) sweeps the block's
// rows, and the global dot products that separate the phases go through
// per-block partials and a bounded grid barrier.  Every block sums the
// partials in the same fixed order, so the Krylov scalars are bit-identical
// across blocks and across runs, and the stopping decision is taken by all
// blocks at the same iteration without any host round trip.
//
// FP64 arithmetic follows the reference exactly (one rounding per multiply
// and per add, no FMA): SpMV rows and vector updates are bit-identical to
// HccaBlas.c / Cg.c / Bicgstab.c; only the dot products sum in a different
// (fixed) order.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>

#include "common.cuh"
#include "internal.h"
#include "persist.cuh"

namespace sfr {

struct KrylovArgs {
  SellView<double> A;
  int n;
  const double *diag[kMaxK];
  const double *b[kMaxK];
  double *x[kMaxK];
  double *m[kMaxK];
  double *r[kMaxK];
  double *z[kMaxK];
  double *q[kMaxK];   // PCG: A p ; BiCGSTAB: v
  double *p0[kMaxK];
  double *p1[kMaxK];  // PCG second p buffer ; BiCGSTAB: t
  double *r0[kMaxK];  // BiCGSTAB shadow residual
  double *part;       // 2 slots x kMaxNV x gridDim
  GridSync gs;
  TeamTable team;     // block -> system map of a batched launch (null: one system)
  SolveOut *out;
  double tol;
  unsigned maxit;
  int newx;
};

// Reduce NV values of a FP64 solve: partials, barrier, totals.
template <int NV>
__device__ __forceinline__ bool reduce_all(const KrylovArgs &a, const Team &t, int &slot,
                                           double (&acc)[NV], double (&tot)[NV], double *sm) {
  return reduce_team<NV>(a.part, t, slot, acc, tot, sm);
}

// y_k[row] for K right-hand sides from a gather functor g(k, col).
template <int K, typename Gather>
__device__ __forceinline__ void row_spmv_k(const SellView<double> &A, const double *const *diag,
                                           int s, int lane, const bool (&act)[K], Gather g,
                                           double (&y)[K]) {
  const int row = s * kWarp + lane;
  const int base = __ldg(A.sptr + s);
  const int w = (__ldg(A.sptr + s + 1) - base) >> 5;
#pragma unroll
  for (int k = 0; k < K; ++k)
    if (act[k]) y[k] = xmul(ld_stream(diag[k] + row), g(k, row));
  const int *c = A.col + base + lane;
  const double *v = A.val + base + lane;
#pragma unroll 2
  for (int e = 0; e < w; ++e) {
    const int j = ld_stream(c + e * kWarp);
    const double av = ld_stream(v + e * kWarp);
#pragma unroll
    for (int k = 0; k < K; ++k)
      if (act[k]) y[k] = xadd(y[k], xmul(av, g(k, j)));
  }
}

// ---------------------------------------------------------------------------
// PCG, Cg.c:47-209 (pcg): one launch for K independent right-hand sides.
// ---------------------------------------------------------------------------
template <int K>
__global__ void __launch_bounds__(kThreads) pcg_fp64_kernel(KrylovArgs a) {
  __shared__ double sm[kMaxNV * 32];
  const Team team = make_team(a.team, a.gs, a.A.nslices, a.n);
  const int n = team.row_end;
  const int lane = threadIdx.x & 31;
  const int s0 = team.s0, s1 = team.s1;
  int slot = 0;
  bool act[K];
  double d[K], conv[K], alpha[K], beta[K];
  int iters[K], status[K];
#pragma unroll
  for (int k = 0; k < K; ++k) {
    act[k] = true;
    beta[k] = 0.0;
    iters[k] = 0;
    status[k] = SFR_OK;
  }

  // setup: m = 1/ad (PreCond.c:18-26), x0, z = M b, d = (b, z)  (Cg.c:66-81)
  {
    double acc[K], tot[K];
#pragma unroll
    for (int k = 0; k < K; ++k) acc[k] = 0.0;
    SFR_FOR_OWN_ROWS(s0, s1) {
#pragma unroll
      for (int k = 0; k < K; ++k) {
        const double mk = 1.0 / ld_vec(a.diag[k] + row_);
        st_vec(a.m[k] + row_, mk);
        if (a.newx) st_vec(a.x[k] + row_, 0.0);
        const double bk = ld_vec(a.b[k] + row_);
        acc[k] += bk * xmul(bk, mk);
      }
    }
    if (!reduce_all<K>(a, team, slot, acc, tot, sm)) return;
#pragma unroll
    for (int k = 0; k < K; ++k) conv[k] = a.tol * sqrt(fabs(tot[k]));
  }
  // r = b - A x ; z = M r ; p = z ; d = (r, z)   (Cg.c:84-102)
  {
    double acc[K], tot[K];
#pragma unroll
    for (int k = 0; k < K; ++k) acc[k] = 0.0;
    SFR_FOR_OWN_ROWS(s0, s1) {
      double y[K];
      row_spmv_k<K>(a.A, a.diag, s_, lane, act,
                    [&](int k, int c) { return ld_vec(a.x[k] + c); }, y);
#pragma unroll
      for (int k = 0; k < K; ++k) {
        const double rk = xsub(ld_vec(a.b[k] + row_), y[k]);
        const double zk = xmul(rk, ld_vec(a.m[k] + row_));
        st_vec(a.r[k] + row_, rk);
        st_vec(a.z[k] + row_, zk);
        st_vec(a.p0[k] + row_, zk);
        acc[k] += rk * zk;
      }
    }
    if (!reduce_all<K>(a, team, slot, acc, tot, sm)) return;
#pragma unroll
    for (int k = 0; k < K; ++k) d[k] = tot[k];
  }

  unsigned j = 0;
  for (; j < a.maxit; ++j) {
    // phase A: p_j = z + beta p_{j-1} (fused, Cg.c:139-141), q = A p_j,
    // (q, p_j)  (Cg.c:105-109)
    double *const *pcur = (j & 1) ? a.p1 : a.p0;
    double *const *pprev = (j & 1) ? a.p0 : a.p1;
    const bool first = j == 0;
    {
      double acc[K], tot[K];
#pragma unroll
      for (int k = 0; k < K; ++k) acc[k] = 0.0;
      auto pval = [&](int k, int c) -> double {
        if (first) return ld_vec(a.p0[k] + c);
        return xadd(ld_vec(a.z[k] + c), xmul(beta[k], ld_vec(pprev[k] + c)));
      };
      SFR_FOR_OWN_ROWS(s0, s1) {
        double y[K];
        row_spmv_k<K>(a.A, a.diag, s_, lane, act, pval, y);
#pragma unroll
        for (int k = 0; k < K; ++k) {
          if (!act[k]) continue;
          const double pk = pval(k, row_);
          if (!first) st_vec(pcur[k] + row_, pk);
          st_vec(a.q[k] + row_, y[k]);
          acc[k] += y[k] * pk;
        }
      }
      if (!reduce_all<K>(a, team, slot, acc, tot, sm)) return;
#pragma unroll
      for (int k = 0; k < K; ++k) {
        if (!act[k]) continue;
        alpha[k] = d[k] / tot[k];
        if (!isfinite(alpha[k])) {
          act[k] = false;
          status[k] = SFR_BREAKDOWN;
          iters[k] = j + 1;
        }
      }
    }
    // phase B: x += alpha p ; r -= alpha q ; z = M r ; (r, z)  (Cg.c:112-136)
    {
      double acc[K], tot[K];
#pragma unroll
      for (int k = 0; k < K; ++k) acc[k] = 0.0;
      SFR_FOR_OWN_ROWS(s0, s1) {
#pragma unroll
        for (int k = 0; k < K; ++k) {
          if (!act[k]) continue;
          const double pk = ld_vec(pcur[k] + row_);
          const double xk = xadd(ld_vec(a.x[k] + row_), xmul(alpha[k], pk));
          const double rk = xsub(ld_vec(a.r[k] + row_), xmul(alpha[k], ld_vec(a.q[k] + row_)));
          const double zk = xmul(rk, ld_vec(a.m[k] + row_));
          st_vec(a.x[k] + row_, xk);
          st_vec(a.r[k] + row_, rk);
          st_vec(a.z[k] + row_, zk);
          acc[k] += rk * zk;
        }
      }
      if (!reduce_all<K>(a, team, slot, acc, tot, sm)) return;
      bool any = false;
#pragma unroll
      for (int k = 0; k < K; ++k) {
        if (!act[k]) continue;
        const double di = tot[k];
        beta[k] = di / d[k];
        d[k] = di;
        if (sqrt(fabs(d[k])) < conv[k]) {
          act[k] = false;
          iters[k] = j + 1;
        } else if (!isfinite(beta[k])) {
          act[k] = false;
          status[k] = SFR_BREAKDOWN;
          iters[k] = j + 1;
        }
        any = any || act[k];
      }
      if (!any) break;
    }
  }
#pragma unroll
  for (int k = 0; k < K; ++k)
    if (act[k]) {
      status[k] = SFR_MAXIT;
      iters[k] = j + 1;
    }

  // post-processing (Cg.c:155-176): xKx, ||x||, ||b - Ax||_M, ||b - Ax||
  {
    bool all[K];
#pragma unroll
    for (int k = 0; k < K; ++k) all[k] = true;
    double acc[4 * K], tot[4 * K];
#pragma unroll
    for (int v = 0; v < 4 * K; ++v) acc[v] = 0.0;
    SFR_FOR_OWN_ROWS(s0, s1) {
      double y[K];
      row_spmv_k<K>(a.A, a.diag, s_, lane, all,
                    [&](int k, int c) { return ld_vec(a.x[k] + c); }, y);
#pragma unroll
      for (int k = 0; k < K; ++k) {
        const double xk = ld_vec(a.x[k] + row_);
        const double rk = xsub(ld_vec(a.b[k] + row_), y[k]);
        const double zk = xmul(rk, ld_vec(a.m[k] + row_));
        acc[4 * k + 0] += xk * y[k];
        acc[4 * k + 1] += xk * xk;
        acc[4 * k + 2] += rk * zk;
        acc[4 * k + 3] += rk * rk;
      }
    }
    if (!reduce_all<4 * K>(a, team, slot, acc, tot, sm)) return;
    if (blockIdx.x == team.b0 && threadIdx.x == 0) {
#pragma unroll
      for (int k = 0; k < K; ++k) {
        SolveOut o;
        o.iters = iters[k];
        o.status = status[k];
        o.xKx = tot[4 * k + 0];
        o.norm_x = sqrt(tot[4 * k + 1]);
        o.norm_r_m = sqrt(fabs(tot[4 * k + 2]));
        o.norm_r = sqrt(tot[4 * k + 3]);
        o.conv = conv[k];
        o.bnorm = 0.0;
        o.refinements = 0;
        o.inner_iters = iters[k];
        o.team_ms = (global_ns() - team.t0) * 1e-6;
        a.out[team.sys * K + k] = o;
      }
    }
  }
}

// ---------------------------------------------------------------------------
// BiCGSTAB, Bicgstab.c:50-245 (pbicgstab), right-preconditioned.
// q holds v = A M^-1 p, p1 holds t = A M^-1 s.
// ---------------------------------------------------------------------------
template <int K>
__global__ void __launch_bounds__(kThreads) bicgstab_fp64_kernel(KrylovArgs a) {
  __shared__ double sm[kMaxNV * 32];
  const Team team = make_team(a.team, a.gs, a.A.nslices, a.n);
  const int n = team.row_end;
  const int lane = threadIdx.x & 31;
  const int s0 = team.s0, s1 = team.s1;
  int slot = 0;
  bool act[K];
  double conv[K], alpha[K], w[K], rr0[K], beta[K];
  int iters[K], status[K];
#pragma unroll
  for (int k = 0; k < K; ++k) {
    act[k] = true;
    iters[k] = 0;
    status[k] = SFR_OK;
  }
  // conv = tol ||b|| (Bicgstab.c:72-80)
  {
    double acc[K], tot[K];
#pragma unroll
    for (int k = 0; k < K; ++k) acc[k] = 0.0;
    SFR_FOR_OWN_ROWS(s0, s1) {
#pragma unroll
      for (int k = 0; k < K; ++k) {
        st_vec(a.m[k] + row_, 1.0 / ld_vec(a.diag[k] + row_));
        if (a.newx) st_vec(a.x[k] + row_, 0.0);
        const double bk = ld_vec(a.b[k] + row_);
        acc[k] += bk * bk;
      }
    }
    if (!reduce_all<K>(a, team, slot, acc, tot, sm)) return;
#pragma unroll
    for (int k = 0; k < K; ++k) conv[k] = a.tol * sqrt(tot[k]);
  }
  // r0 = b - A x ; p = r = r0 ; z = M p  (Bicgstab.c:83-99)
  {
    SFR_FOR_OWN_ROWS(s0, s1) {
      double y[K];
      row_spmv_k<K>(a.A, a.diag, s_, lane, act,
                    [&](int k, int c) { return ld_vec(a.x[k] + c); }, y);
#pragma unroll
      for (int k = 0; k < K; ++k) {
        const double rk = xsub(ld_vec(a.b[k] + row_), y[k]);
        st_vec(a.r0[k] + row_, rk);
        st_vec(a.p0[k] + row_, rk);
        st_vec(a.r[k] + row_, rk);
        st_vec(a.z[k] + row_, xmul(rk, ld_vec(a.m[k] + row_)));
      }
    }
    if (!grid_sync(team.gs)) return;
  }
  unsigned j = 0;
  bool any = true;
  for (; j < a.maxit && any; ++j) {
    // v = A z ; rr0 = (r, r0) ; alpha = rr0 / (v, r0)  (Bicgstab.c:105-113)
    {
      double acc[2 * K], tot[2 * K];
#pragma unroll
      for (int v = 0; v < 2 * K; ++v) acc[v] = 0.0;
      SFR_FOR_OWN_ROWS(s0, s1) {
        double y[K];
        row_spmv_k<K>(a.A, a.diag, s_, lane, act,
                      [&](int k, int c) { return ld_vec(a.z[k] + c); }, y);
#pragma unroll
        for (int k = 0; k < K; ++k) {
          if (!act[k]) continue;
          st_vec(a.q[k] + row_, y[k]);
          const double r0k = ld_vec(a.r0[k] + row_);
          acc[2 * k] += ld_vec(a.r[k] + row_) * r0k;
          acc[2 * k + 1] += y[k] * r0k;
        }
      }
      if (!reduce_all<2 * K>(a, team, slot, acc, tot, sm)) return;
#pragma unroll
      for (int k = 0; k < K; ++k) {
        if (!act[k]) continue;
        rr0[k] = tot[2 * k];
        alpha[k] = rr0[k] / tot[2 * k + 1];
        if (!isfinite(alpha[k])) {
          act[k] = false;
          status[k] = SFR_BREAKDOWN;
          iters[k] = j + 1;
        }
      }
    }
    // x += alpha z ; s = r -= alpha v ; z = M s ; (s, s)  (Bicgstab.c:116-133)
    {
      double acc[K], tot[K];
#pragma unroll
      for (int k = 0; k < K; ++k) acc[k] = 0.0;
      SFR_FOR_OWN_ROWS(s0, s1) {
#pragma unroll
        for (int k = 0; k < K; ++k) {
          if (!act[k]) continue;
          const double xk = xadd(ld_vec(a.x[k] + row_), xmul(alpha[k], ld_vec(a.z[k] + row_)));
          const double rk = xsub(ld_vec(a.r[k] + row_), xmul(alpha[k], ld_vec(a.q[k] + row_)));
          st_vec(a.x[k] + row_, xk);
          st_vec(a.r[k] + row_, rk);
          st_vec(a.z[k] + row_, xmul(rk, ld_vec(a.m[k] + row_)));
          acc[k] += rk * rk;
        }
      }
      if (!reduce_all<K>(a, team, slot, acc, tot, sm)) return;
#pragma unroll
      for (int k = 0; k < K; ++k) {
        if (!act[k]) continue;
        if (sqrt(tot[k]) < conv[k]) {
          act[k] = false;
          iters[k] = j + 1;
        }
      }
    }
    // t = A z ; w = (t, s) / (t, t)  (Bicgstab.c:136-142)
    {
      double acc[2 * K], tot[2 * K];
#pragma unroll
      for (int v = 0; v < 2 * K; ++v) acc[v] = 0.0;
      SFR_FOR_OWN_ROWS(s0, s1) {
        double y[K];
        row_spmv_k<K>(a.A, a.diag, s_, lane, act,
                      [&](int k, int c) { return ld_vec(a.z[k] + c); }, y);
#pragma unroll
        for (int k = 0; k < K; ++k) {
          if (!act[k]) continue;
          st_vec(a.p1[k] + row_, y[k]);
          acc[2 * k] += y[k] * ld_vec(a.r[k] + row_);
          acc[2 * k + 1] += y[k] * y[k];
        }
      }
      if (!reduce_all<2 * K>(a, team, slot, acc, tot, sm)) return;
#pragma unroll
      for (int k = 0; k < K; ++k) {
        if (!act[k]) continue;
        w[k] = tot[2 * k] / tot[2 * k + 1];
        if (!isfinite(w[k])) {
          act[k] = false;
          status[k] = SFR_BREAKDOWN;
          iters[k] = j + 1;
        }
      }
    }
    // x += w z ; r -= w t ; (r, r), (r, r0)  (Bicgstab.c:145-165)
    {
      double acc[2 * K], tot[2 * K];
#pragma unroll
      for (int v = 0; v < 2 * K; ++v) acc[v] = 0.0;
      SFR_FOR_OWN_ROWS(s0, s1) {
#pragma unroll
        for (int k = 0; k < K; ++k) {
          if (!act[k]) continue;
          const double xk = xadd(ld_vec(a.x[k] + row_), xmul(w[k], ld_vec(a.z[k] + row_)));
          const double rk = xsub(ld_vec(a.r[k] + row_), xmul(w[k], ld_vec(a.p1[k] + row_)));
          st_vec(a.x[k] + row_, xk);
          st_vec(a.r[k] + row_, rk);
          acc[2 * k] += rk * rk;
          acc[2 * k + 1] += rk * ld_vec(a.r0[k] + row_);
        }
      }
      if (!reduce_all<2 * K>(a, team, slot, acc, tot, sm)) return;
      any = false;
#pragma unroll
      for (int k = 0; k < K; ++k) {
        if (!act[k]) continue;
        if (sqrt(tot[2 * k]) < conv[k]) {
          act[k] = false;
          iters[k] = j + 1;
          continue;
        }
        beta[k] = (tot[2 * k + 1] / rr0[k]) * (alpha[k] / w[k]);
        if (!isfinite(beta[k])) {
          act[k] = false;
          status[k] = SFR_BREAKDOWN;
          iters[k] = j + 1;
          continue;
        }
        any = true;
      }
    }
    if (!any) break;
    // p = r + beta (p - w v) ; z = M p  (Bicgstab.c:168-176)
    {
      SFR_FOR_OWN_ROWS(s0, s1) {
#pragma unroll
        for (int k = 0; k < K; ++k) {
          if (!act[k]) continue;
          const double pk = xadd(ld_vec(a.r[k] + row_),
                                 xmul(beta[k], xsub(ld_vec(a.p0[k] + row_),
                                                    xmul(w[k], ld_vec(a.q[k] + row_)))));
          st_vec(a.p0[k] + row_, pk);
          st_vec(a.z[k] + row_, xmul(pk, ld_vec(a.m[k] + row_)));
        }
      }
      if (!grid_sync(team.gs)) return;
    }
  }
#pragma unroll
  for (int k = 0; k < K; ++k)
    if (act[k]) {
      status[k] = SFR_MAXIT;
      iters[k] = j + 1;
    }
  // post-processing (Bicgstab.c:188-204)
  {
    bool all[K];
#pragma unroll
    for (int k = 0; k < K; ++k) all[k] = true;
    double acc[3 * K], tot[3 * K];
#pragma unroll
    for (int v = 0; v < 3 * K; ++v) acc[v] = 0.0;
    SFR_FOR_OWN_ROWS(s0, s1) {
      double y[K];
      row_spmv_k<K>(a.A, a.diag, s_, lane, all,
                    [&](int k, int c) { return ld_vec(a.x[k] + c); }, y);
#pragma unroll
      for (int k = 0; k < K; ++k) {
        const double xk = ld_vec(a.x[k] + row_);
        const double rk = xsub(ld_vec(a.b[k] + row_), y[k]);
        acc[3 * k + 0] += xk * y[k];
        acc[3 * k + 1] += xk * xk;
        acc[3 * k + 2] += rk * rk;
      }
    }
    if (!reduce_all<3 * K>(a, team, slot, acc, tot, sm)) return;
    if (blockIdx.x == team.b0 && threadIdx.x == 0) {
#pragma unroll
      for (int k = 0; k < K; ++k) {
        SolveOut o;
        o.iters = iters[k];
        o.status = status[k];
        o.xKx = tot[3 * k + 0];
        o.norm_x = sqrt(tot[3 * k + 1]);
        o.norm_r = sqrt(tot[3 * k + 2]);
        o.norm_r_m = 0.0;
        o.conv = conv[k];
        o.bnorm = 0.0;
        o.refinements = 0;
        o.inner_iters = iters[k];
        o.team_ms = (global_ns() - team.t0) * 1e-6;
        a.out[team.sys * K + k] = o;
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Standalone kernels: SpMV, SpMV fused with (y, x), dot.  The reductions end
// in the last block to finish (fixed order over the block partials).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) spmv_kernel(SellView<double> A, const double *x,
                                                   double *y) {
  const int n = A.n;
  const int lane = threadIdx.x & 31;
  int s0, s1;
  block_slices(A.nslices, &s0, &s1);
  const double *diag[1] = {A.diag};
  const int act[1] = {1};
  SFR_FOR_OWN_ROWS(s0, s1) {
    double yv[1];
    row_product<1, true, double>(A.sptr, A.col, A.val, diag, s_, lane, act,
                                 [&](int, int c) { return x[c]; }, yv);
    y[row_] = yv[0];
  }
}

__device__ __forceinline__ void last_block_total(double local, double *part, unsigned *counter,
                                                 double *out) {
  __shared__ double sm[32];
  __shared__ bool last;
  double acc[1] = {local};
  block_partials<1>(acc, part, gridDim.x, sm);
  if (threadIdx.x == 0) {
    __threadfence();
    const unsigned prev = atomicAdd(counter, 1u);
    last = prev == gridDim.x - 1;
  }
  __syncthreads();
  if (last) {
    __threadfence();
    double tot[1];
    grid_totals<1>(part, gridDim.x, gridDim.x, tot, sm);
    if (threadIdx.x == 0) {
      *out = tot[0];
      *counter = 0u;
    }
  }
}

__global__ void __launch_bounds__(256) spmv_dot_kernel(SellView<double> A, const double *x,
                                                       double *y, double *part,
                                                       unsigned *counter, double *out) {
  const int lane = threadIdx.x & 31;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  double acc = 0.0;
  for (int s = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; s < A.nslices; s += nw) {
    const int row = s * kWarp + lane;
    if (row < A.n) {
      const double t = row_spmv_exact(A, s, lane, x);
      y[row] = t;
      acc += t * x[row];
    }
  }
  last_block_total(acc, part, counter, out);
}

__global__ void __launch_bounds__(256) dot_kernel(const double *a, const double *b, int n,
                                                  double *part, unsigned *counter, double *out) {
  double acc = 0.0;
  // 64-bit index: i + stride must not overflow for n close to INT32_MAX
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += stride)
    acc += a[i] * b[i];
  last_block_total(acc, part, counter, out);
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
int num_sms(int device) {
  int v = 0;
  if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) return 0;
  return v;
}

// standalone kernels: 4 blocks of 256 threads per SM (the device's own SM
// count); the scratch holds partials for GPUs of up to 256 SMs
constexpr int kStatBlocksPerSm = 4;
constexpr int kStatGrid = kStatBlocksPerSm * 256;

int stat_grid(int device, int64_t n) {
  const int64_t cap = static_cast<int64_t>(kStatBlocksPerSm) * std::max(1, num_sms(device));
  const int64_t want = (std::max<int64_t>(n, 0) + 255) / 256;
  return static_cast<int>(std::max<int64_t>(1, std::min({cap, want, int64_t{kStatGrid}})));
}

namespace {

// automatic engine choice: the graph engine from this many rows up
constexpr int kGraphEngineRows = 100000;

struct Scratch {  // per-device scratch for the standalone reductions
  double *part = nullptr;
  unsigned *counter = nullptr;
  double *out = nullptr;
};
Scratch g_scratch[64];

int scratch_for(int device, Scratch **s) {
  if (device < 0 || device >= 64) return SFR_BAD_INPUT;
  Scratch &sc = g_scratch[device];
  if (!sc.part) {
    void *p = nullptr;
    if (cudaMalloc(&p, sizeof(double) * (kStatGrid + 1) + sizeof(unsigned) * 2) != cudaSuccess)
      return SFR_CUDA_ERROR;
    if (cudaMemset(p, 0, sizeof(double) * (kStatGrid + 1) + sizeof(unsigned) * 2) != cudaSuccess)
      return SFR_CUDA_ERROR;
    sc.part = static_cast<double *>(p);
    sc.out = sc.part + kStatGrid;
    sc.counter = reinterpret_cast<unsigned *>(sc.out + 1);
  }
  *s = &sc;
  return SFR_OK;
}

int grid_for_slices(int nslices, int device) {
  const int want = (nslices + 7) / 8;  // 8 warps per 256-thread block
  return std::max(1, std::min(want, stat_grid(device, INT64_MAX)));
}

template <typename F>
int occupancy_grid(F kernel, int threads, int device, int *blocks_per_sm) {
  int occ = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kernel, threads, 0) != cudaSuccess)
    return 0;
  *blocks_per_sm = occ;
  return occ * num_sms(device);
}

}  // namespace

int spmv_device(sfr_system *s, const DevSell &A, const double *d_diag, const double *d_x,
                double *d_y, double *d_dot, cudaStream_t st) {
  SellView<double> v{A.n, A.nslices, A.sptr, A.col, A.val, d_diag};
  const int grid = grid_for_slices(A.nslices, s->device);
  if (!d_dot) {
    // the graph engine's launch shape: 8 warps per block, block-contiguous
    // slice ranges; graph_spw slices per warp, or (0) one wave of resident
    // blocks
    int g2 = 0;
    if (s->graph_spw > 0) {
      g2 = std::max(1, (A.nslices + 8 * s->graph_spw - 1) / (8 * s->graph_spw));
    } else {
      static int occ[64] = {};
      const int d = s->device & 63;
      if (!occ[d] && (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ[d], spmv_kernel, 256, 0) !=
                          cudaSuccess ||
                      occ[d] < 1))
        occ[d] = 1;
      g2 = std::max(1, std::min((A.nslices + 7) / 8, occ[d] * num_sms(s->device)));
    }
    spmv_kernel<<<g2, 256, 0, st>>>(v, d_x, d_y);
  } else {
    Scratch *sc = nullptr;
    int rc = scratch_for(s->device, &sc);
    if (rc != SFR_OK) return rc;
    spmv_dot_kernel<<<grid, 256, 0, st>>>(v, d_x, d_y, sc->part, sc->counter, d_dot);
  }
  return cudaGetLastError() == cudaSuccess ? SFR_OK : SFR_CUDA_ERROR;
}

int dot_device(const double *d_a, const double *d_b, int32_t n, double *d_dot, cudaStream_t st) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return SFR_CUDA_ERROR;
  Scratch *sc = nullptr;
  int rc = scratch_for(dev, &sc);
  if (rc != SFR_OK) return rc;
  const int grid = stat_grid(dev, n);
  dot_kernel<<<grid, 256, 0, st>>>(d_a, d_b, n, sc->part, sc->counter, d_dot);
  return cudaGetLastError() == cudaSuccess ? SFR_OK : SFR_CUDA_ERROR;
}

int dot_host(const double *d_a, const double *d_b, int32_t n, double *h_out, cudaStream_t st) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return SFR_CUDA_ERROR;
  Scratch *sc = nullptr;
  int rc = scratch_for(dev, &sc);
  if (rc != SFR_OK) return rc;
  rc = dot_device(d_a, d_b, n, sc->out, st);
  if (rc != SFR_OK) return rc;
  if (cudaMemcpyAsync(h_out, sc->out, sizeof(double), cudaMemcpyDeviceToHost, st) != cudaSuccess)
    return SFR_CUDA_ERROR;
  return cudaStreamSynchronize(st) == cudaSuccess ? SFR_OK : SFR_CUDA_ERROR;
}

namespace {

// Workspace layout for a K-RHS solve: vectors, partials, control words.
struct Layout {
  size_t vec_off, part_off, ctl_off, out_off, total;
};

constexpr int kVecs = 8;  // m r z q p0 p1 r0 (+1 spare)

Layout layout_for(int n, int k, int grid) {
  Layout L{};
  size_t off = 0;
  auto align = [](size_t v) { return (v + 255) & ~static_cast<size_t>(255); };
  L.vec_off = off;
  off = align(off + sizeof(double) * static_cast<size_t>(n) * kVecs * k);
  L.part_off = off;
  off = align(off + sizeof(double) * 2 * kMaxNV * static_cast<size_t>(grid));
  L.ctl_off = off;
  off = align(off + 64);
  L.out_off = off;
  off = align(off + sizeof(SolveOut) * kMaxK);
  L.total = off;
  return L;
}

template <int K>
int launch_krylov(sfr_system *s, int32_t solver, const double *d_diag_k, const double *d_b,
                  double *d_x, double tol, uint32_t maxit, int32_t newx, cudaStream_t st,
                  SolveOut *host_out, float *ms) {
  const int n = s->n;
  void (*kern)(KrylovArgs) = solver == SFR_PCG ? pcg_fp64_kernel<K> : bicgstab_fp64_kernel<K>;
  int bps = 0;
  const int max_grid = occupancy_grid(kern, kThreads, s->device, &bps);
  if (max_grid <= 0) return SFR_CUDA_ERROR;
  const int warps = kThreads / kWarp;
  const int grid = std::max(1, std::min(max_grid, (s->A.nslices + warps - 1) / warps));
  const Layout L = layout_for(n, K, grid);
  int rc = ensure_workspace(s, L.total);
  if (rc != SFR_OK) return rc;
  char *base = static_cast<char *>(s->ws.base);
  double *vec = reinterpret_cast<double *>(base + L.vec_off);
  auto V = [&](int which, int k) { return vec + (static_cast<size_t>(which) * K + k) * n; };

  KrylovArgs a;
  std::memset(&a, 0, sizeof(a));
  a.A = SellView<double>{s->A.n, s->A.nslices, s->A.sptr, s->A.col, s->A.val, s->d_diag};
  a.n = n;
  for (int k = 0; k < K; ++k) {
    a.diag[k] = d_diag_k ? d_diag_k + static_cast<size_t>(k) * n : s->d_diag;
    a.b[k] = d_b + static_cast<size_t>(k) * n;
    a.x[k] = d_x + static_cast<size_t>(k) * n;
    a.m[k] = V(0, k);
    a.r[k] = V(1, k);
    a.z[k] = V(2, k);
    a.q[k] = V(3, k);
    a.p0[k] = V(4, k);
    a.p1[k] = V(5, k);
    a.r0[k] = V(6, k);
  }
  a.part = reinterpret_cast<double *>(base + L.part_off);
  unsigned *ctl = reinterpret_cast<unsigned *>(base + L.ctl_off);
  a.gs.count = ctl;
  a.gs.gen = ctl + 1;
  a.gs.err = reinterpret_cast<int *>(ctl + 2);
  a.gs.nblocks = grid;
  a.gs.spin_limit = 1u << 22;  // about a second or more of polling
  a.out = reinterpret_cast<SolveOut *>(base + L.out_off);
  a.tol = tol;
  a.maxit = maxit;
  a.newx = newx;

  if (cudaMemsetAsync(ctl, 0, 64, st) != cudaSuccess) return SFR_CUDA_ERROR;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, st);
  void *params[] = {&a};
  cudaError_t err = cudaLaunchCooperativeKernel(reinterpret_cast<void *>(kern), dim3(grid),
                                                dim3(kThreads), params, 0, st);
  cudaEventRecord(e1, st);
  int ctl_host[3] = {0, 0, 0};
  if (err == cudaSuccess) err = cudaMemcpyAsync(host_out, a.out, sizeof(SolveOut) * K,
                                                cudaMemcpyDeviceToHost, st);
  if (err == cudaSuccess) err = cudaMemcpyAsync(ctl_host, ctl, sizeof(ctl_host),
                                                cudaMemcpyDeviceToHost, st);
  if (err == cudaSuccess) err = cudaStreamSynchronize(st);
  if (err == cudaSuccess) cudaEventElapsedTime(ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (err != cudaSuccess) return SFR_CUDA_ERROR;
  if (ctl_host[2] != 0) return ctl_host[2];
  return SFR_OK;
}

}  // namespace

// ---- batched (team) launches: K = 1, no host synchronisation, so the
// launch can be captured in a CUDA graph.
size_t team_ws_bytes_fp64(int n, int grid) {
  auto align = [](size_t v) { return (v + 255) & ~static_cast<size_t>(255); };
  return align(sizeof(double) * static_cast<size_t>(n) * kVecs) +
         align(sizeof(double) * 2 * kMaxNV * static_cast<size_t>(grid));
}

int team_max_grid_fp64(int32_t solver, int device) {
  void (*kern)(KrylovArgs) = solver == SFR_PCG ? pcg_fp64_kernel<1> : bicgstab_fp64_kernel<1>;
  int bps = 0;
  return occupancy_grid(kern, kThreads, device, &bps);
}

int enqueue_team_fp64(sfr_system *s, int32_t solver, const double *d_b, double *d_x, double tol,
                      uint32_t maxit, int32_t newx, const TeamTable &team, int grid, void *ws,
                      SolveOut *d_out, unsigned *ctl, cudaStream_t st) {
  const int n = s->n;
  auto align = [](size_t v) { return (v + 255) & ~static_cast<size_t>(255); };
  double *vec = static_cast<double *>(ws);
  auto V = [&](int which) { return vec + static_cast<size_t>(which) * n; };
  KrylovArgs a;
  std::memset(&a, 0, sizeof(a));
  a.A = SellView<double>{s->A.n, s->A.nslices, s->A.sptr, s->A.col, s->A.val, s->d_diag};
  a.n = n;
  a.diag[0] = s->d_diag;
  a.b[0] = d_b;
  a.x[0] = d_x;
  a.m[0] = V(0);
  a.r[0] = V(1);
  a.z[0] = V(2);
  a.q[0] = V(3);
  a.p0[0] = V(4);
  a.p1[0] = V(5);
  a.r0[0] = V(6);
  a.part = reinterpret_cast<double *>(static_cast<char *>(ws) +
                                      align(sizeof(double) * static_cast<size_t>(n) * kVecs));
  a.gs.count = ctl;
  a.gs.gen = ctl + 1;
  a.gs.err = reinterpret_cast<int *>(ctl + 2);
  a.gs.nblocks = grid;
  a.gs.spin_limit = 1u << 22;
  a.team = team;
  a.out = d_out;
  a.tol = tol;
  a.maxit = maxit;
  a.newx = newx;
  if (cudaMemsetAsync(ctl, 0, 64, st) != cudaSuccess) return SFR_CUDA_ERROR;
  void (*kern)(KrylovArgs) = solver == SFR_PCG ? pcg_fp64_kernel<1> : bicgstab_fp64_kernel<1>;
  void *params[] = {&a};
  return cudaLaunchCooperativeKernel(reinterpret_cast<void *>(kern), dim3(grid), dim3(kThreads),
                                     params, 0, st) == cudaSuccess
             ? SFR_OK
             : SFR_CUDA_ERROR;
}

int auto_engine(sfr_system *s, int32_t solver, int32_t k, int32_t precision, bool own_diag) {
  const bool resident_case = precision == SFR_MIXED && solver == SFR_PCG && k == 1 && own_diag;
  if (resident_case && s->n >= kGraphEngineRows && resident_fits(s)) return 4;
  return s->n >= kGraphEngineRows ? 2 : 1;
}

int solve_device(sfr_system *s, int32_t solver, int32_t k, const double *d_diag_k,
                 const double *d_b, double *d_x, double tol, uint32_t maxit, int32_t newx,
                 int32_t precision, cudaStream_t st, sfr_solve_info *info) {
  if (k < 1 || k > kMaxK) return SFR_BAD_INPUT;
  if (solver == SFR_PBICGSTABL2 || solver == SFR_GMRES || solver == SFR_MINRES) {
    // one right-hand side, FP64, on every engine setting
    if (k != 1 || precision != SFR_FP64) return SFR_UNSUPPORTED;
    return solve_ext(s, solver, d_diag_k, d_b, d_x, tol, maxit, newx, st, info);
  }
  if (solver != SFR_PCG && solver != SFR_PBICGSTAB) return SFR_UNSUPPORTED;
  int engine = s->engine;
  int threads = s->graph_threads, spw = s->graph_spw, pf = s->graph_pf, fused = s->graph_fused;
  const bool resident_case = precision == SFR_MIXED && solver == SFR_PCG && k == 1 && !d_diag_k;
  bool tuned = false;
  if (engine == 0) {
    if (const Tuned *t = find_tuned(s, solver, k, precision, d_diag_k == nullptr)) {
      engine = t->engine;
      threads = t->threads;
      spw = t->spw;
      pf = t->pf;
      fused = t->fused;
      tuned = true;
    }
  }
  if (engine == 4 || (engine == 0 && resident_case && s->n >= kGraphEngineRows && resident_fits(s))) {
    if (!resident_case) return SFR_UNSUPPORTED;
    const int rc = solve_resident(s, d_b, d_x, tol, maxit, newx, st, info);
    // automatic choice: a diagonal that is not positive has no Jacobi scaling
    if (rc != SFR_UNSUPPORTED || (engine == 4 && !tuned)) return rc;
  }
  if (engine == 0 || engine == 4) engine = s->n >= kGraphEngineRows ? 2 : 1;
  if (engine == 2 || engine == 3)
    return solve_stream(s, solver, k, d_diag_k, d_b, d_x, tol, maxit, newx, precision,
                        reliable_delta(solver), threads, spw, pf, fused, engine == 3, st, info);
  if (precision == SFR_MIXED)
    return solve_mixed(s, solver, k, d_diag_k, d_b, d_x, tol, maxit, newx, st, info);
  if (precision != SFR_FP64) return SFR_UNSUPPORTED;
  SolveOut out[kMaxK];
  float ms = 0.f;
  int rc;
  switch (k) {
    case 1: rc = launch_krylov<1>(s, solver, d_diag_k, d_b, d_x, tol, maxit, newx, st, out, &ms); break;
    case 2: rc = launch_krylov<2>(s, solver, d_diag_k, d_b, d_x, tol, maxit, newx, st, out, &ms); break;
    case 3: rc = launch_krylov<3>(s, solver, d_diag_k, d_b, d_x, tol, maxit, newx, st, out, &ms); break;
    default: rc = launch_krylov<4>(s, solver, d_diag_k, d_b, d_x, tol, maxit, newx, st, out, &ms); break;
  }
  if (rc != SFR_OK) return rc;
  int worst = SFR_OK;
  for (int i = 0; i < k; ++i) {
    if (info) {
      sfr_solve_info &f = info[i];
      std::memset(&f, 0, sizeof(f));
      f.iters = out[i].iters;
      f.status = out[i].status;
      f.xKx = out[i].xKx;
      f.norm_x = out[i].norm_x;
      f.norm_r = out[i].norm_r;
      f.norm_r_m = out[i].norm_r_m;
      f.conv = out[i].conv;
      f.seconds = ms * 1e-3;
      f.refinements = 0;
      f.inner_iters = out[i].iters;
      f.relres = std::nan("");
    }
    if (out[i].status != SFR_OK && worst == SFR_OK) worst = out[i].status;
  }
  return worst;
}

}  // namespace sfr
