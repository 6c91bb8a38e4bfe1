// Mixed precision: FP32 matrix values and inner Krylov vectors inside an
// FP64 refinement loop, in one persistent launch per solve.
//
// The inner recurrence (PCG or BiCGSTAB on the FP32 copy of A, FP32 vectors,
// dot products accumulated in FP64) keeps running across refinements; this is
// iterative refinement with "reliable updates" (Sleijpen & van der Vorst,
// 1996): whenever the inner residual estimate has dropped by `delta` since the
// last refinement, or claims convergence, the FP32 correction is added to the
// FP64 solution, the true residual r = b - A x is recomputed with the FP64
// matrix, and the inner residual is replaced by it.  The solution, the true
// residual and the refinement-level dot products are FP64; convergence is
// decided only on the FP64 true residual, with the reference's criterion:
// sqrt|(r, M^-1 r)| < tol sqrt|(b, M^-1 b)| for PCG (Cg.c:70-74, 145) and
// ||r|| < tol ||b|| for BiCGSTAB (Bicgstab.c:72-80, 130, 155).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>

#include "common.cuh"
#include "internal.h"
#include "persist.cuh"

namespace sfr {

namespace {

struct MixedArgs {
  SellView<double> A64;  // FP64 values (diagonals come per right-hand side)
  SellView<float> A32;   // FP32 copy
  int n;
  const double *diag64[kMaxK];
  const double *b[kMaxK];
  double *x[kMaxK];
  double *dc[kMaxK];  // diagonal of the FP32 operator: ad + row compensation (FP64)
  const double *comp; // -sum_row (fl32(a_ij) - a_ij)
  float *m32[kMaxK];  // FP32 Jacobi 1/diag
  float *r[kMaxK];    // inner residual
  float *z[kMaxK];    // PCG: M r ; BiCGSTAB: M p
  float *p0[kMaxK];   // search direction (PCG double-buffers it)
  float *p1[kMaxK];
  float *q[kMaxK];    // PCG: A p ; BiCGSTAB: v = A z
  float *xs[kMaxK];   // FP32 correction since the last reliable update
  float *r0[kMaxK];   // BiCGSTAB shadow residual
  float *t[kMaxK];    // BiCGSTAB t = A z
  double *part;
  GridSync gs;
  TeamTable team;  // block -> system map of a batched launch (null: one system)
  SolveOut *out;
  double tol;
  double delta;
  unsigned maxit;
  int newx;
};

// y_k = (A32 v_k)[row]: FP32 couplings and FP32 vectors, accumulated in FP64
// around the compensated FP64 diagonal (so the FP32 operator keeps the FP64
// row sums), rounded to FP32 once.
template <int K, typename Gather>
__device__ __forceinline__ void row_spmv32(const MixedArgs &a, int s, int lane, const bool (&act)[K],
                                           Gather g, float (&y)[K]) {
  int ia[K];
#pragma unroll
  for (int k = 0; k < K; ++k) ia[k] = act[k];
  double yd[K];
  const double *const *dc = a.dc;
  row_product_t<K, double, false, float, double>(a.A32.sptr, a.A32.col, a.A32.val, dc, s, lane,
                                                 ia, g, yd);
#pragma unroll
  for (int k = 0; k < K; ++k)
    if (act[k]) y[k] = __double2float_rn(yd[k]);
}

// (A64 x_k)[row] in FP64 (FMA allowed: this is the refinement residual).
__device__ __forceinline__ double row_spmv64(const MixedArgs &a, int k, int s, int lane) {
  const int row = s * kWarp + lane;
  const int base = __ldg(a.A64.sptr + s);
  const int w = (__ldg(a.A64.sptr + s + 1) - base) >> 5;
  const double *x = a.x[k];
  double y = ld_vec(a.diag64[k] + row) * ld_vec(x + row);
  const int *c = a.A64.col + base + lane;
  const double *v = a.A64.val + base + lane;
#pragma unroll 2
  for (int e = 0; e < w; ++e) y = fma(ld_stream(v + e * kWarp), ld_vec(x + ld_stream(c + e * kWarp)), y);
  return y;
}

// Reliable update of the selected right-hand sides:
//   x += xs (FP64), barrier, r_true = b - A64 x, r = fl32(r_true),
//   z = M r, xs = 0.  (BiCGSTAB after a full step overwrites z = M p next.)
// tot[2k]   = (r_true, M^-1 r_true) (PCG) or (r_true, r_true) (BiCGSTAB)
// tot[2k+1] = (r, z) (PCG) or (r, r0) (BiCGSTAB), in FP64 from the FP32 r.
// With `first`, x is not updated and the PCG direction / BiCGSTAB shadow
// residual and direction are initialised from r.
template <int K, bool kPcg>
__device__ bool reliable_update(const MixedArgs &a, const Team &t, const bool (&sel)[K],
                                bool first, int &slot, double *sm, double (&tot)[2 * K]) {
  const int n = t.row_end;
  const int s0 = t.s0, s1 = t.s1;
  const int lane = threadIdx.x & 31;
  if (!first) {
    SFR_FOR_OWN_ROWS(s0, s1) {
#pragma unroll
      for (int k = 0; k < K; ++k) {
        if (!sel[k]) continue;
        const double xk = ld_vec(a.x[k] + row_) + static_cast<double>(ld_vec(a.xs[k] + row_));
        st_vec(a.x[k] + row_, xk);
      }
    }
    if (!grid_sync(t.gs)) return false;
  }
  double acc[2 * K];
#pragma unroll
  for (int v = 0; v < 2 * K; ++v) acc[v] = 0.0;
  SFR_FOR_OWN_ROWS(s0, s1) {
#pragma unroll
    for (int k = 0; k < K; ++k) {
      if (!sel[k]) continue;
      const double rt = ld_vec(a.b[k] + row_) - row_spmv64(a, k, s_, lane);
      const float rs = __double2float_rn(rt);
      st_vec(a.r[k] + row_, rs);
      st_vec(a.xs[k] + row_, 0.0f);
      const float zs = ld_vec(a.m32[k] + row_) * rs;
      st_vec(a.z[k] + row_, zs);
      if (kPcg) {
        if (first) st_vec(a.p0[k] + row_, zs);
        acc[2 * k] += rt * (rt / ld_vec(a.diag64[k] + row_));
        acc[2 * k + 1] += static_cast<double>(rs) * static_cast<double>(zs);
      } else {
        if (first) {
          st_vec(a.r0[k] + row_, rs);
          st_vec(a.p0[k] + row_, rs);
        }
        acc[2 * k] += rt * rt;
        acc[2 * k + 1] += static_cast<double>(rs) * static_cast<double>(ld_vec(a.r0[k] + row_));
      }
    }
  }
  // BiCGSTAB: r0 was written above only on the first call; the (r, r0) read
  // uses the value this thread just stored, so no barrier is needed before it.
  return reduce_team<2 * K>(a.part, t, slot, acc, tot, sm);
}

template <int K, bool kPcg>
__device__ void finish(const MixedArgs &a, const Team &t, const int (&iters)[K],
                       const int (&status)[K], const int (&refine)[K], const double (&conv)[K],
                       const double (&bnorm)[K], int &slot, double *sm) {
  const int n = t.row_end;
  const int s0 = t.s0, s1 = t.s1;
  const int lane = threadIdx.x & 31;
  double acc[4 * K], tot[4 * K];
#pragma unroll
  for (int v = 0; v < 4 * K; ++v) acc[v] = 0.0;
  SFR_FOR_OWN_ROWS(s0, s1) {
#pragma unroll
    for (int k = 0; k < K; ++k) {
      const double y = row_spmv64(a, k, s_, lane);
      const double xk = ld_vec(a.x[k] + row_);
      const double rk = ld_vec(a.b[k] + row_) - y;
      acc[4 * k + 0] += xk * y;
      acc[4 * k + 1] += xk * xk;
      acc[4 * k + 2] += rk * (rk / ld_vec(a.diag64[k] + row_));
      acc[4 * k + 3] += rk * rk;
    }
  }
  if (!reduce_team<4 * K>(a.part, t, slot, acc, tot, sm)) return;
  if (blockIdx.x == t.b0 && threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < K; ++k) {
      SolveOut o;
      o.iters = iters[k];
      o.status = status[k];
      o.xKx = tot[4 * k + 0];
      o.norm_x = sqrt(tot[4 * k + 1]);
      o.norm_r_m = kPcg ? sqrt(fabs(tot[4 * k + 2])) : 0.0;
      o.norm_r = sqrt(tot[4 * k + 3]);
      o.conv = conv[k];
      o.bnorm = bnorm[k];
      o.refinements = refine[k];
      o.inner_iters = iters[k];
      o.team_ms = (global_ns() - t.t0) * 1e-6;
      a.out[t.sys * K + k] = o;
    }
  }
}

// Setup shared by both solvers: FP32 diagonal and Jacobi, x0, and the two
// norms of b ((b, M^-1 b) and (b, b)).
template <int K>
__device__ bool setup(const MixedArgs &a, const Team &t, int &slot, double *sm,
                      double (&bm)[K], double (&bb)[K]) {
  const int n = t.row_end;
  const int s0 = t.s0, s1 = t.s1;
  double acc[2 * K], tot[2 * K];
#pragma unroll
  for (int v = 0; v < 2 * K; ++v) acc[v] = 0.0;
  SFR_FOR_OWN_ROWS(s0, s1) {
#pragma unroll
    for (int k = 0; k < K; ++k) {
      const double dk = ld_vec(a.diag64[k] + row_);
      st_vec(a.dc[k] + row_, dk + ld_vec(a.comp + row_));
      st_vec(a.m32[k] + row_, __double2float_rn(1.0 / dk));
      if (a.newx) st_vec(a.x[k] + row_, 0.0);
      const double bk = ld_vec(a.b[k] + row_);
      acc[2 * k] += bk * (bk / dk);
      acc[2 * k + 1] += bk * bk;
    }
  }
  if (!reduce_team<2 * K>(a.part, t, slot, acc, tot, sm)) return false;
#pragma unroll
  for (int k = 0; k < K; ++k) {
    bm[k] = tot[2 * k];
    bb[k] = tot[2 * k + 1];
  }
  return true;
}

// ---------------------------------------------------------------------------
// Mixed PCG.
// ---------------------------------------------------------------------------
template <int K>
__global__ void __launch_bounds__(kThreads, K == 1 ? 2 : 1) pcg_mixed_kernel(MixedArgs a) {
  __shared__ double sm[kMaxNV * 32];
  const Team team = make_team(a.team, a.gs, a.A32.nslices, a.n);
  const int n = team.row_end;
  const int lane = threadIdx.x & 31;
  const int s0 = team.s0, s1 = team.s1;
  int slot = 0;
  bool act[K];
  double d[K], conv[K], bnorm[K], alpha[K], beta[K], rmax[K];
  int iters[K], status[K], refine[K];
  {
    double bm[K], bb[K];
    if (!setup<K>(a, team, slot, sm, bm, bb)) return;
#pragma unroll
    for (int k = 0; k < K; ++k) {
      conv[k] = a.tol * sqrt(fabs(bm[k]));
      bnorm[k] = sqrt(bb[k]);
      act[k] = true;
      beta[k] = 0.0;
      iters[k] = 0;
      status[k] = SFR_OK;
      refine[k] = 0;
    }
  }
  {
    double tot[2 * K];
    if (!reliable_update<K, true>(a, team, act, true, slot, sm, tot)) return;
#pragma unroll
    for (int k = 0; k < K; ++k) {
      rmax[k] = sqrt(fabs(tot[2 * k]));
      d[k] = tot[2 * k + 1];
      if (rmax[k] < conv[k]) act[k] = false;
    }
  }
  bool any = false;
#pragma unroll
  for (int k = 0; k < K; ++k) any = any || act[k];
  unsigned j = 0;
  for (; j < a.maxit && any; ++j) {
    float *const *pcur = (j & 1) ? a.p1 : a.p0;
    float *const *pprev = (j & 1) ? a.p0 : a.p1;
    const bool first = j == 0;
    float bf[K];
#pragma unroll
    for (int k = 0; k < K; ++k) bf[k] = static_cast<float>(beta[k]);
    // q = A32 p_j with p_j = z + beta p_{j-1} formed at every gather
    {
      double acc[K], tot[K];
#pragma unroll
      for (int k = 0; k < K; ++k) acc[k] = 0.0;
      auto pval = [&](int k, int c) -> float {
        if (first) return ld_vec(a.p0[k] + c);
        return fmaf(bf[k], ld_vec(pprev[k] + c), ld_vec(a.z[k] + c));
      };
      SFR_FOR_OWN_ROWS(s0, s1) {
        float y[K];
        row_spmv32<K>(a, s_, lane, act, pval, y);
#pragma unroll
        for (int k = 0; k < K; ++k) {
          if (!act[k]) continue;
          const float pk = pval(k, row_);
          if (!first) st_vec(pcur[k] + row_, pk);
          st_vec(a.q[k] + row_, y[k]);
          acc[k] += static_cast<double>(y[k]) * static_cast<double>(pk);
        }
      }
      if (!reduce_team<K>(a.part, team, slot, acc, tot, sm)) return;
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
    // xs += alpha p ; r -= alpha q ; z = M r ; (r, z)
    bool upd[K];
    bool any_upd = false;
    {
      double acc[K], tot[K];
      float af[K];
#pragma unroll
      for (int k = 0; k < K; ++k) {
        acc[k] = 0.0;
        af[k] = static_cast<float>(alpha[k]);
      }
      SFR_FOR_OWN_ROWS(s0, s1) {
#pragma unroll
        for (int k = 0; k < K; ++k) {
          if (!act[k]) continue;
          const float pk = ld_vec(pcur[k] + row_);
          st_vec(a.xs[k] + row_, fmaf(af[k], pk, ld_vec(a.xs[k] + row_)));
          const float rk = fmaf(-af[k], ld_vec(a.q[k] + row_), ld_vec(a.r[k] + row_));
          const float zk = ld_vec(a.m32[k] + row_) * rk;
          st_vec(a.r[k] + row_, rk);
          st_vec(a.z[k] + row_, zk);
          acc[k] += static_cast<double>(rk) * static_cast<double>(zk);
        }
      }
      if (!reduce_team<K>(a.part, team, slot, acc, tot, sm)) return;
#pragma unroll
      for (int k = 0; k < K; ++k) {
        upd[k] = false;
        if (!act[k]) continue;
        const double est = sqrt(fabs(tot[k]));
        if (!isfinite(tot[k])) {
          act[k] = false;
          status[k] = SFR_BREAKDOWN;
          iters[k] = j + 1;
          continue;
        }
        if (est < a.delta * rmax[k] || est < conv[k]) {
          upd[k] = true;
          any_upd = true;
        } else {
          beta[k] = tot[k] / d[k];
          d[k] = tot[k];
        }
      }
    }
    if (any_upd) {
      double tot[2 * K];
      if (!reliable_update<K, true>(a, team, upd, false, slot, sm, tot)) return;
#pragma unroll
      for (int k = 0; k < K; ++k) {
        if (!upd[k]) continue;
        ++refine[k];
        const double tr = sqrt(fabs(tot[2 * k]));
        if (tr < conv[k]) {
          act[k] = false;
          iters[k] = j + 1;
        } else {
          beta[k] = tot[2 * k + 1] / d[k];
          d[k] = tot[2 * k + 1];
          rmax[k] = tr;
        }
      }
    }
    any = false;
#pragma unroll
    for (int k = 0; k < K; ++k) any = any || act[k];
  }
  // iteration cap: fold the last correction into x
  bool left[K];
  bool any_left = false;
#pragma unroll
  for (int k = 0; k < K; ++k) {
    left[k] = act[k];
    if (act[k]) {
      status[k] = SFR_MAXIT;
      iters[k] = j + 1;
      any_left = true;
    }
  }
  if (any_left) {
    SFR_FOR_OWN_ROWS(s0, s1) {
#pragma unroll
      for (int k = 0; k < K; ++k)
        if (left[k])
          st_vec(a.x[k] + row_, ld_vec(a.x[k] + row_) + static_cast<double>(ld_vec(a.xs[k] + row_)));
    }
    if (!grid_sync(team.gs)) return;
  }
  finish<K, true>(a, team, iters, status, refine, conv, bnorm, slot, sm);
}

// ---------------------------------------------------------------------------
// Mixed BiCGSTAB (right-preconditioned, Bicgstab.c:50-245).
// ---------------------------------------------------------------------------
template <int K>
__global__ void __launch_bounds__(kThreads, K == 1 ? 2 : 1) bicgstab_mixed_kernel(MixedArgs a) {
  __shared__ double sm[kMaxNV * 32];
  const Team team = make_team(a.team, a.gs, a.A32.nslices, a.n);
  const int n = team.row_end;
  const int lane = threadIdx.x & 31;
  const int s0 = team.s0, s1 = team.s1;
  int slot = 0;
  bool act[K];
  double conv[K], bnorm[K], alpha[K], w[K], rr0[K], beta[K], rmax[K];
  int iters[K], status[K], refine[K];
  {
    double bm[K], bb[K];
    if (!setup<K>(a, team, slot, sm, bm, bb)) return;
#pragma unroll
    for (int k = 0; k < K; ++k) {
      bnorm[k] = sqrt(bb[k]);
      conv[k] = a.tol * bnorm[k];
      act[k] = true;
      iters[k] = 0;
      status[k] = SFR_OK;
      refine[k] = 0;
    }
  }
  {
    double tot[2 * K];
    if (!reliable_update<K, false>(a, team, act, true, slot, sm, tot)) return;
#pragma unroll
    for (int k = 0; k < K; ++k) {
      rmax[k] = sqrt(tot[2 * k]);
      if (rmax[k] < conv[k]) act[k] = false;
    }
  }
  bool any = false;
#pragma unroll
  for (int k = 0; k < K; ++k) any = any || act[k];
  unsigned j = 0;
  for (; j < a.maxit && any; ++j) {
    // v = A32 z ; rr0 = (r, r0) ; alpha = rr0 / (v, r0)
    {
      double acc[2 * K], tot[2 * K];
#pragma unroll
      for (int v = 0; v < 2 * K; ++v) acc[v] = 0.0;
      SFR_FOR_OWN_ROWS(s0, s1) {
        float y[K];
        row_spmv32<K>(a, s_, lane, act, [&](int k, int c) { return ld_vec(a.z[k] + c); }, y);
#pragma unroll
        for (int k = 0; k < K; ++k) {
          if (!act[k]) continue;
          st_vec(a.q[k] + row_, y[k]);
          const double r0k = ld_vec(a.r0[k] + row_);
          acc[2 * k] += static_cast<double>(ld_vec(a.r[k] + row_)) * r0k;
          acc[2 * k + 1] += static_cast<double>(y[k]) * r0k;
        }
      }
      if (!reduce_team<2 * K>(a.part, team, slot, acc, tot, sm)) return;
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
    // xs += alpha z ; s = r -= alpha v ; z = M s ; (s, s)
    bool upd[K];
    bool any_upd = false;
    {
      double acc[K], tot[K];
#pragma unroll
      for (int k = 0; k < K; ++k) acc[k] = 0.0;
      SFR_FOR_OWN_ROWS(s0, s1) {
#pragma unroll
        for (int k = 0; k < K; ++k) {
          if (!act[k]) continue;
          const float af = static_cast<float>(alpha[k]);
          st_vec(a.xs[k] + row_, fmaf(af, ld_vec(a.z[k] + row_), ld_vec(a.xs[k] + row_)));
          const float rk = fmaf(-af, ld_vec(a.q[k] + row_), ld_vec(a.r[k] + row_));
          st_vec(a.r[k] + row_, rk);
          st_vec(a.z[k] + row_, ld_vec(a.m32[k] + row_) * rk);
          acc[k] += static_cast<double>(rk) * static_cast<double>(rk);
        }
      }
      if (!reduce_team<K>(a.part, team, slot, acc, tot, sm)) return;
#pragma unroll
      for (int k = 0; k < K; ++k) {
        upd[k] = act[k] && sqrt(tot[k]) < conv[k];
        any_upd = any_upd || upd[k];
      }
    }
    if (any_upd) {  // half-step convergence claimed: check the true residual
      double tot[2 * K];
      if (!reliable_update<K, false>(a, team, upd, false, slot, sm, tot)) return;
#pragma unroll
      for (int k = 0; k < K; ++k) {
        if (!upd[k]) continue;
        ++refine[k];
        const double tr = sqrt(tot[2 * k]);
        if (tr < conv[k]) {
          act[k] = false;
          iters[k] = j + 1;
        } else {
          rmax[k] = tr;
        }
      }
    }
    // t = A32 z ; w = (t, s) / (t, t)
    {
      double acc[2 * K], tot[2 * K];
#pragma unroll
      for (int v = 0; v < 2 * K; ++v) acc[v] = 0.0;
      SFR_FOR_OWN_ROWS(s0, s1) {
        float y[K];
        row_spmv32<K>(a, s_, lane, act, [&](int k, int c) { return ld_vec(a.z[k] + c); }, y);
#pragma unroll
        for (int k = 0; k < K; ++k) {
          if (!act[k]) continue;
          st_vec(a.t[k] + row_, y[k]);
          acc[2 * k] += static_cast<double>(y[k]) * static_cast<double>(ld_vec(a.r[k] + row_));
          acc[2 * k + 1] += static_cast<double>(y[k]) * static_cast<double>(y[k]);
        }
      }
      if (!reduce_team<2 * K>(a.part, team, slot, acc, tot, sm)) return;
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
    // xs += w z ; r -= w t ; (r, r), (r, r0)
    {
      double acc[2 * K], tot[2 * K];
#pragma unroll
      for (int v = 0; v < 2 * K; ++v) acc[v] = 0.0;
      SFR_FOR_OWN_ROWS(s0, s1) {
#pragma unroll
        for (int k = 0; k < K; ++k) {
          if (!act[k]) continue;
          const float wf = static_cast<float>(w[k]);
          st_vec(a.xs[k] + row_, fmaf(wf, ld_vec(a.z[k] + row_), ld_vec(a.xs[k] + row_)));
          const float rk = fmaf(-wf, ld_vec(a.t[k] + row_), ld_vec(a.r[k] + row_));
          st_vec(a.r[k] + row_, rk);
          acc[2 * k] += static_cast<double>(rk) * static_cast<double>(rk);
          acc[2 * k + 1] += static_cast<double>(rk) * static_cast<double>(ld_vec(a.r0[k] + row_));
        }
      }
      if (!reduce_team<2 * K>(a.part, team, slot, acc, tot, sm)) return;
      any_upd = false;
#pragma unroll
      for (int k = 0; k < K; ++k) {
        upd[k] = false;
        if (!act[k]) continue;
        const double est = sqrt(tot[2 * k]);
        beta[k] = (tot[2 * k + 1] / rr0[k]) * (alpha[k] / w[k]);
        if (est < conv[k] || est < a.delta * rmax[k]) {
          upd[k] = true;
          any_upd = true;
        }
      }
    }
    if (any_upd) {
      double tot[2 * K];
      if (!reliable_update<K, false>(a, team, upd, false, slot, sm, tot)) return;
#pragma unroll
      for (int k = 0; k < K; ++k) {
        if (!upd[k]) continue;
        ++refine[k];
        const double tr = sqrt(tot[2 * k]);
        if (tr < conv[k]) {
          act[k] = false;
          iters[k] = j + 1;
        } else {
          rmax[k] = tr;
          beta[k] = (tot[2 * k + 1] / rr0[k]) * (alpha[k] / w[k]);
        }
      }
    }
#pragma unroll
    for (int k = 0; k < K; ++k)
      if (act[k] && !isfinite(beta[k])) {
        act[k] = false;
        status[k] = SFR_BREAKDOWN;
        iters[k] = j + 1;
      }
    any = false;
#pragma unroll
    for (int k = 0; k < K; ++k) any = any || act[k];
    if (!any) break;
    // p = r + beta (p - w v) ; z = M p
    SFR_FOR_OWN_ROWS(s0, s1) {
#pragma unroll
      for (int k = 0; k < K; ++k) {
        if (!act[k]) continue;
        const float bfk = static_cast<float>(beta[k]);
        const float wf = static_cast<float>(w[k]);
        const float pk = fmaf(bfk, fmaf(-wf, ld_vec(a.q[k] + row_), ld_vec(a.p0[k] + row_)),
                              ld_vec(a.r[k] + row_));
        st_vec(a.p0[k] + row_, pk);
        st_vec(a.z[k] + row_, ld_vec(a.m32[k] + row_) * pk);
      }
    }
    if (!grid_sync(team.gs)) return;
  }
  bool left[K];
  bool any_left = false;
#pragma unroll
  for (int k = 0; k < K; ++k) {
    left[k] = act[k];
    if (act[k]) {
      status[k] = SFR_MAXIT;
      iters[k] = j + 1;
      any_left = true;
    }
  }
  if (any_left) {
    SFR_FOR_OWN_ROWS(s0, s1) {
#pragma unroll
      for (int k = 0; k < K; ++k)
        if (left[k])
          st_vec(a.x[k] + row_, ld_vec(a.x[k] + row_) + static_cast<double>(ld_vec(a.xs[k] + row_)));
    }
    if (!grid_sync(team.gs)) return;
  }
  finish<K, false>(a, team, iters, status, refine, conv, bnorm, slot, sm);
}

// --------------------------------------------------------------- host ---
constexpr int kFloatVecs = 10;  // (unused) m32 r z p0 p1 q xs r0 t

// Refresh factor per solver.  PCG on the ill-conditioned pressure systems
// needs frequent refreshes (a smaller factor lets the FP32 recurrence drift
// and multiplies the iterations); BiCGSTAB on the diagonally dominant
// momentum systems converges in a few iterations, where each refresh (an
// FP64 SpMV) is a large share of the work.
double g_delta_pcg = 0.1;
double g_delta_bicg = 1e-4;
// The resident engine's PCG restarts its recurrence less often: its FP32
// recurrence on the scaled operator holds the true residual closely, and
// each restart costs conjugacy (128^3 Poisson: 1825 inner iterations at
// 0.02 against 2068 at 0.1).
double g_delta_pcg_resident = 0.02;

template <int K>
int launch_mixed(sfr_system *s, int32_t solver, const double *d_diag_k, const double *d_b,
                 double *d_x, double tol, uint32_t maxit, int32_t newx, cudaStream_t st,
                 SolveOut *host_out, float *ms) {
  const int n = s->n;
  void (*kern)(MixedArgs) = solver == SFR_PCG ? pcg_mixed_kernel<K> : bicgstab_mixed_kernel<K>;
  int occ = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, kThreads, 0) != cudaSuccess ||
      occ <= 0)
    return SFR_CUDA_ERROR;
  const int max_grid = occ * num_sms(s->device);
  const int warps = kThreads / kWarp;
  const int grid = std::max(1, std::min(max_grid, (s->A.nslices + warps - 1) / warps));
  auto align = [](size_t v) { return (v + 255) & ~static_cast<size_t>(255); };
  const size_t dc_bytes = align(sizeof(double) * static_cast<size_t>(n) * K);
  const size_t vec_bytes = dc_bytes + align(sizeof(float) * static_cast<size_t>(n) * kFloatVecs * K);
  const size_t part_bytes = align(sizeof(double) * 2 * kMaxNV * static_cast<size_t>(grid));
  const size_t ctl_bytes = 256;
  const size_t out_bytes = align(sizeof(SolveOut) * kMaxK);
  int rc = ensure_workspace(s, vec_bytes + part_bytes + ctl_bytes + out_bytes);
  if (rc != SFR_OK) return rc;
  char *base = static_cast<char *>(s->ws.base);
  double *dcv = reinterpret_cast<double *>(base);
  float *vec = reinterpret_cast<float *>(base + dc_bytes);
  auto V = [&](int which, int k) { return vec + (static_cast<size_t>(which) * K + k) * n; };

  MixedArgs a;
  std::memset(&a, 0, sizeof(a));
  a.A64 = SellView<double>{s->A.n, s->A.nslices, s->A.sptr, s->A.col, s->A.val, nullptr};
  a.A32 = SellView<float>{s->A.n, s->A.nslices, s->A.sptr, s->A.col, s->A.val32, nullptr};
  a.n = n;
  a.comp = s->d_comp;
  for (int k = 0; k < K; ++k) {
    a.diag64[k] = d_diag_k ? d_diag_k + static_cast<size_t>(k) * n : s->d_diag;
    a.b[k] = d_b + static_cast<size_t>(k) * n;
    a.x[k] = d_x + static_cast<size_t>(k) * n;
    a.dc[k] = dcv + static_cast<size_t>(k) * n;
    a.m32[k] = V(1, k);
    a.r[k] = V(2, k);
    a.z[k] = V(3, k);
    a.p0[k] = V(4, k);
    a.p1[k] = V(5, k);
    a.q[k] = V(6, k);
    a.xs[k] = V(7, k);
    a.r0[k] = V(8, k);
    a.t[k] = V(9, k);
  }
  a.part = reinterpret_cast<double *>(base + vec_bytes);
  unsigned *ctl = reinterpret_cast<unsigned *>(base + vec_bytes + part_bytes);
  a.gs.count = ctl;
  a.gs.gen = ctl + 1;
  a.gs.err = reinterpret_cast<int *>(ctl + 2);
  a.gs.nblocks = grid;
  a.gs.spin_limit = 1u << 22;
  a.out = reinterpret_cast<SolveOut *>(base + vec_bytes + part_bytes + ctl_bytes);
  a.tol = tol;
  a.delta = reliable_delta(solver);
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
  if (err == cudaSuccess)
    err = cudaMemcpyAsync(host_out, a.out, sizeof(SolveOut) * K, cudaMemcpyDeviceToHost, st);
  if (err == cudaSuccess)
    err = cudaMemcpyAsync(ctl_host, ctl, sizeof(ctl_host), cudaMemcpyDeviceToHost, st);
  if (err == cudaSuccess) err = cudaStreamSynchronize(st);
  if (err == cudaSuccess) cudaEventElapsedTime(ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (err != cudaSuccess) return SFR_CUDA_ERROR;
  if (ctl_host[2] != 0) return ctl_host[2];
  return SFR_OK;
}

}  // namespace

// ---- batched (team) launch, K = 1, capturable (no host synchronisation).
size_t team_ws_bytes_mixed(int n, int grid) {
  auto align = [](size_t v) { return (v + 255) & ~static_cast<size_t>(255); };
  return align(sizeof(double) * static_cast<size_t>(n)) +
         align(sizeof(float) * static_cast<size_t>(n) * kFloatVecs) +
         align(sizeof(double) * 2 * kMaxNV * static_cast<size_t>(grid));
}

int team_max_grid_mixed(int32_t solver, int device) {
  void (*kern)(MixedArgs) = solver == SFR_PCG ? pcg_mixed_kernel<1> : bicgstab_mixed_kernel<1>;
  int occ = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, kThreads, 0) != cudaSuccess)
    return 0;
  return occ * num_sms(device);
}

int enqueue_team_mixed(sfr_system *s, int32_t solver, const double *d_b, double *d_x, double tol,
                       uint32_t maxit, int32_t newx, const TeamTable &team, int grid, void *ws,
                       SolveOut *d_out, unsigned *ctl, cudaStream_t st) {
  const int n = s->n;
  auto align = [](size_t v) { return (v + 255) & ~static_cast<size_t>(255); };
  const size_t dc_bytes = align(sizeof(double) * static_cast<size_t>(n));
  double *dcv = static_cast<double *>(ws);
  float *vec = reinterpret_cast<float *>(static_cast<char *>(ws) + dc_bytes);
  auto V = [&](int which) { return vec + static_cast<size_t>(which) * n; };
  MixedArgs a;
  std::memset(&a, 0, sizeof(a));
  a.A64 = SellView<double>{s->A.n, s->A.nslices, s->A.sptr, s->A.col, s->A.val, nullptr};
  a.A32 = SellView<float>{s->A.n, s->A.nslices, s->A.sptr, s->A.col, s->A.val32, nullptr};
  a.n = n;
  a.diag64[0] = s->d_diag;
  a.comp = s->d_comp;
  a.b[0] = d_b;
  a.x[0] = d_x;
  a.dc[0] = dcv;
  a.m32[0] = V(1);
  a.r[0] = V(2);
  a.z[0] = V(3);
  a.p0[0] = V(4);
  a.p1[0] = V(5);
  a.q[0] = V(6);
  a.xs[0] = V(7);
  a.r0[0] = V(8);
  a.t[0] = V(9);
  a.part = reinterpret_cast<double *>(static_cast<char *>(ws) + dc_bytes +
                                      align(sizeof(float) * static_cast<size_t>(n) * kFloatVecs));
  a.gs.count = ctl;
  a.gs.gen = ctl + 1;
  a.gs.err = reinterpret_cast<int *>(ctl + 2);
  a.gs.nblocks = grid;
  a.gs.spin_limit = 1u << 22;
  a.team = team;
  a.out = d_out;
  a.tol = tol;
  a.delta = reliable_delta(solver);
  a.maxit = maxit;
  a.newx = newx;
  if (cudaMemsetAsync(ctl, 0, 64, st) != cudaSuccess) return SFR_CUDA_ERROR;
  void (*kern)(MixedArgs) = solver == SFR_PCG ? pcg_mixed_kernel<1> : bicgstab_mixed_kernel<1>;
  void *params[] = {&a};
  return cudaLaunchCooperativeKernel(reinterpret_cast<void *>(kern), dim3(grid), dim3(kThreads),
                                     params, 0, st) == cudaSuccess
             ? SFR_OK
             : SFR_CUDA_ERROR;
}

int solve_mixed(sfr_system *s, int32_t solver, int32_t k, const double *d_diag_k,
                const double *d_b, double *d_x, double tol, uint32_t maxit, int32_t newx,
                cudaStream_t st, sfr_solve_info *info) {
  if (k < 1 || k > kMaxK) return SFR_BAD_INPUT;
  SolveOut out[kMaxK];
  float ms = 0.f;
  int rc;
  switch (k) {
    case 1: rc = launch_mixed<1>(s, solver, d_diag_k, d_b, d_x, tol, maxit, newx, st, out, &ms); break;
    case 2: rc = launch_mixed<2>(s, solver, d_diag_k, d_b, d_x, tol, maxit, newx, st, out, &ms); break;
    case 3: rc = launch_mixed<3>(s, solver, d_diag_k, d_b, d_x, tol, maxit, newx, st, out, &ms); break;
    default: rc = launch_mixed<4>(s, solver, d_diag_k, d_b, d_x, tol, maxit, newx, st, out, &ms); break;
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
      f.refinements = out[i].refinements;
      f.inner_iters = out[i].inner_iters;
      f.relres = out[i].bnorm > 0 ? out[i].norm_r / out[i].bnorm : 0.0;
    }
    if (out[i].status != SFR_OK && worst == SFR_OK) worst = out[i].status;
  }
  return worst;
}

double reliable_delta(int32_t solver) {
  return solver == SFR_PCG ? g_delta_pcg : g_delta_bicg;
}

double reliable_delta_resident() { return g_delta_pcg_resident; }

}  // namespace sfr

extern "C" void sfr_set_reliable_delta(double delta) {
  if (delta > 0.0 && delta < 1.0)
    sfr::g_delta_pcg = sfr::g_delta_bicg = sfr::g_delta_pcg_resident = delta;
}

extern "C" int sfr_set_solver_reliable_delta(int32_t solver, double delta) {
  if (!(delta > 0.0 && delta < 1.0)) return SFR_BAD_INPUT;
  if (solver == SFR_PCG)
    sfr::g_delta_pcg = sfr::g_delta_pcg_resident = delta;
  else if (solver == SFR_PBICGSTAB)
    sfr::g_delta_bicg = delta;
  else
    return SFR_BAD_INPUT;
  return SFR_OK;
}
