// MINRES (Iters.c:309-558, pminres) with its scalar recurrence on the device:
// the whole solve is one CUDA graph whose iteration loop is a conditional
// WHILE node, like the graph engine's PCG (stream_solve.cu), so no dot
// product travels to the host.
//
// One iteration is two kernels, or, with the handle's fused-iteration
// option (sfr_gpu_set_fused) and a co-resident launch shape, one cooperative
// kernel (k_mr_fused; at 128^3 it measured slower, 126 against 97 us an
// iteration for three kernels: 55 registers and 57 KB of shared memory a
// block leave four blocks an SM for the SpMV phase).  The steps:
//   a. p = A z0 and (z0, p); the last block forms alpha = (z0, p) / beta^2
//      and the three-term coefficients t1 = 1/beta, t2 = -alpha/beta,
//      t3 = -beta/beta_old;
//   b. p = t1 p + t2 v + t3 v0, z = M p and (z, p); the last block runs the
//      rest of the reference's scalar step -- beta, delta, ro2, ro3, symOrtho
//      (Iters.c:1171-1211, with its branch tests as written: |b| is compared
//      with a, not |a|), u1..u4, |r| = |s| |r| -- decides convergence,
//      breakdown (a non-finite u) or maxIt, and clears the WHILE condition;
//   c. w = u1 z0 + u2 w0 + u3 w00, x += u4 w (skipped after a breakdown, as
//      the reference breaks before its update), done by the next
//      iteration's kernel a for its own rows before its product, and after
//      the loop by a tail kernel.
// The reference rotates its vectors (v0 <- v <- p, z0 <- z, w00 <- w0 <- w)
// by pointer swaps, with periods 3 and 2; the graph body unrolls six
// iterations, each with its own fixed roles, and the kernels of iterations
// after the stop return at once.
//
// Every scalar is computed with the reference's operations in its order,
// each rounded once (no FMA contraction, IEEE division and square root), and
// every vector element with the reference's C expression, so the recurrence
// differs from the reference only through the dot products' summation order.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstring>
#include <map>
#include <memory>

#include "common.cuh"
#include "internal.h"
#include "persist.cuh"

namespace sfr {

namespace {

constexpr int kMrThreads = 256;
constexpr int kMrUnroll = 6;  // vector roles rotate with periods 3 and 2
constexpr int kMrCounters = 16;  // 0-4 last-block counters, 12-14 the grid barrier

struct MrState {
  // per call
  double tol;
  unsigned maxit;
  int newx;
  // recurrence
  double conv, beta, beta_old, alpha, t1, t2, t3;
  double c, c_old, s, s_old, ro1, neta, norm_r;
  double u1, u2, u3, u4;
  unsigned j;
  int active, upd, status, iters;
  // post-processing (Iters.c:540-557 with the solver's common epilogue)
  double xKx, norm_x, norm_r_true, norm_r_m;
};

struct MrArgs {
  int n, nslices;
  const int *sptr;
  SlotCols cols;
  const double *val;
  double *ad, *b, *x, *m;        // the graph's own copies of the diagonal, b and x
  double *V[3], *Z[2], *W[3];    // v0/v/p, z0/z, w00/w0/w by rotation
  double *part;
  unsigned *counter;
  MrState *st;
  cudaGraphConditionalHandle hwhile;
};

#define SFR_MR_FOR_ROWS(i) \
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += gridDim.x * blockDim.x)

// Row pairs (2i, 2i+1) with 16-byte loads; every vector of the graph's
// workspace has room for an even count, and its padding entries stay 0.
#define SFR_MR_FOR_PAIRS(i)                                                          \
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; 2 * i < a.n;                  \
       i += gridDim.x * blockDim.x)

__device__ __forceinline__ double2 ld2(const double *p) {
  return *reinterpret_cast<const double2 *>(p);
}
__device__ __forceinline__ void st2(double *p, double2 v) { *reinterpret_cast<double2 *>(p) = v; }


// Iters.c:1171-1211 (symOrtho): no branch taken leaves c, s, r as they were.
__device__ void sym_ortho_dev(double a, double b, double *c, double *s, double *r) {
  const double ma = fabs(a), mb = fabs(b);
  const double sa = a > 0.0 ? 1.0 : -1.0, sb = b > 0.0 ? 1.0 : -1.0;
  if (b == 0.0) {
    *s = 0.0;
    *r = ma;
    *c = a == 0.0 ? 1.0 : sa;
  } else if (a == 0.0) {
    *c = 0.0;
    *s = sb;
    *r = mb;
  } else if (mb > a) {
    const double t = xdiv(a, b);
    *s = xdiv(sb, xsqrt(xadd(1.0, xmul(t, t))));
    *c = xmul(*s, t);
    *r = xdiv(b, *s);
  } else if (ma > mb) {
    const double t = xdiv(b, a);
    *c = xdiv(sa, xsqrt(xadd(1.0, xmul(t, t))));
    *s = xmul(*c, t);
    *r = xdiv(a, *c);
  }
}

// m = 1/ad, x0, z = M^1/2 b; conv = tol ||z||  (Iters.c:355-372)
__global__ void __launch_bounds__(kMrThreads) k_mr_setup1(const MrArgs a) {
  SFR_SHARED_RED(1);
  MrState *st = a.st;
  const int newx = st->newx;
  double acc[1] = {0.0};
  double *z = a.Z[1];
  SFR_MR_FOR_ROWS(i) {
    const double mi = 1.0 / a.ad[i];
    a.m[i] = mi;
    if (newx) a.x[i] = 0.0;
    const double zi = xmul(a.b[i], sqrt(mi));
    z[i] = zi;
    acc[0] += zi * zi;
  }
  if (!last_block<1>(acc, a.part, a.counter + 0, sm)) return;
  if (threadIdx.x == 0) st->conv = xmul(st->tol, xsqrt(sm[0]));
}

// v = b - A x, v0 = w0 = w00 = 0, z0 = M v; beta = sqrt|(v, z0)|
// (Iters.c:374-398), with the iteration-0 roles.
template <typename I>
__global__ void __launch_bounds__(kMrThreads) k_mr_setup2(const MrArgs a) {
  SFR_SHARED_RED(1);
  MrState *st = a.st;
  const int n = a.n;
  const int lane = threadIdx.x & 31;
  int s0, s1;
  block_slices(a.nslices, &s0, &s1);
  const int all[1] = {1};
  const double *const diag[1] = {a.ad};
  double acc[1] = {0.0};
  SFR_FOR_OWN_ROWS(s0, s1) {
    double y[1];
    row_product<1, true, double>(a.sptr, cols_of<I>(a.cols), a.val, diag, s_, lane, all,
                                 [&](int, int c) { return ld_ro(a.x + c); }, y);
    const double vi = xsub(a.b[row_], y[0]);
    a.V[1][row_] = vi;  // v
    a.V[0][row_] = 0.0; // v0
    a.W[1][row_] = 0.0; // w0
    a.W[0][row_] = 0.0; // w00
    const double zi = xmul(vi, a.m[row_]);
    a.Z[0][row_] = zi;  // z0
    acc[0] += vi * zi;
  }
  if (!last_block<1>(acc, a.part, a.counter + 1, sm)) return;
  if (threadIdx.x == 0) {
    const double beta = xsqrt(fabs(sm[0]));
    st->beta = beta;
    st->beta_old = beta;
    st->norm_r = beta;
    st->neta = beta;
    st->c_old = 1.0;
    st->c = 1.0;
    st->s_old = 0.0;
    st->s = 0.0;
    st->ro1 = 1.0;
    st->j = 0;
    st->upd = 0;
    st->status = SFR_OK;
    st->active = st->maxit > 0 ? 1 : 0;
    if (!st->active) {
      st->status = SFR_MAXIT;
      st->iters = 1;
      cudaGraphSetConditional(a.hwhile, 0u);
    }
  }
}

// The previous iteration's w = u1 z0 + u2 w0 + u3 w00, x += u4 w
// (Iters.c:482-497) for one row, with that iteration's roles (pu).
__device__ __forceinline__ void mr_update_row(const MrArgs &a, const MrState *st, int pu,
                                              int row) {
  const double *z0 = a.Z[pu % 2];
  const double *w00 = a.W[pu % 3], *w0 = a.W[(pu + 1) % 3];
  double *w = a.W[(pu + 2) % 3];
  const double wi = xadd(xadd(xmul(st->u1, ld_ro(z0 + row)), xmul(st->u2, ld_ro(w0 + row))),
                         xmul(st->u3, ld_ro(w00 + row)));
  st_vec(w + row, wi);
  st_vec(a.x + row, xadd(ld_vec(a.x + row), xmul(st->u4, wi)));
}

// A row's operands in phase a: the previous iteration's z0, w0, w00 and x
// (for its pending update) and this iteration's z0 (for the dot).
struct MrRowIn {
  double zp, w0, w00, x, zc;
};

// a: the previous iteration's w and x update for this warp's rows (it waits
// for no reduction; its streaming loads overlap the product's gathers), then
// p = A z0, alpha and the three-term coefficients (Iters.c:402-411).  The
// update's operands are loaded with the slice's columns, before the gathers
// (slice_rows).
// Held to 64 registers (four blocks an SM): 77 us an iteration at 128^3
// against 81 us at the 76 registers it takes uncapped.
template <typename I>
__global__ void __launch_bounds__(kMrThreads, 4) k_mr_a(const MrArgs a, int u) {
  SFR_SHARED_RED(1);
  MrState *st = a.st;
  if (!st->active) return;
  const int n = a.n;
  const double *z0 = a.Z[u % 2];
  double *p = a.V[(u + 2) % 3];
  const bool pending = st->upd != 0;
  // the previous iteration's roles (Iters.c:482-497)
  const int pu = (u + kMrUnroll - 1) % kMrUnroll;
  const double *zprev = a.Z[pu % 2];
  const double *w00 = a.W[pu % 3], *w0 = a.W[(pu + 1) % 3];
  double *wn = a.W[(pu + 2) % 3];
  double u1 = 0.0, u2 = 0.0, u3 = 0.0, u4 = 0.0;
  if (pending) {
    u1 = st->u1;
    u2 = st->u2;
    u3 = st->u3;
    u4 = st->u4;
  }
  int s0, s1;
  block_slices(a.nslices, &s0, &s1);
  const int all[1] = {1};
  const double *const diag[1] = {a.ad};
  double acc[1] = {0.0};
  slice_rows<1, double, true, double, double, I>(
      n, a.sptr, cols_of<I>(a.cols), a.val, diag, s0, s1, 0, all,
      [&](int, int c) { return ld_ro(z0 + c); },
      [&](int, int row) {
        MrRowIn r{0.0, 0.0, 0.0, 0.0, ld_ro(z0 + row)};
        if (pending) {
          r.zp = ld_ro(zprev + row);
          r.w0 = ld_ro(w0 + row);
          r.w00 = ld_ro(w00 + row);
          r.x = ld_vec(a.x + row);
        }
        return r;
      },
      [&](int, int row, double y, MrRowIn r) {
        if (pending) {  // w = u1 z0 + u2 w0 + u3 w00, x += u4 w
          const double wi = xadd(xadd(xmul(u1, r.zp), xmul(u2, r.w0)), xmul(u3, r.w00));
          st_vec(wn + row, wi);
          st_vec(a.x + row, xadd(r.x, xmul(u4, wi)));
        }
        st_vec(p + row, y);
        acc[0] += r.zc * y;
      });
  if (!last_block<1>(acc, a.part, a.counter + 2, sm)) return;
  if (threadIdx.x == 0) {
    const double beta = st->beta;
    const double t1 = xdiv(1.0, xmul(beta, beta));
    const double alpha = xmul(sm[0], t1);
    st->alpha = alpha;
    st->t1 = xdiv(1.0, beta);
    st->t2 = xdiv(-alpha, beta);
    st->t3 = xdiv(-beta, st->beta_old);
  }
}

// The scalar part of one iteration (Iters.c:431-470) on a copy of the state:
// zp = (z, p) of the new Lanczos vector.  Sets beta, the rotation, u1..u4,
// |r|, the stop decision (convergence, breakdown -- a non-finite u, before
// the update, as the reference breaks -- or maxIt) and j + 1.
__device__ void mr_step(MrState &q, double alpha, double zp) {
  const unsigned j = q.j;
  const double beta_old = q.beta;
  const double beta = xsqrt(zp);
  double c = q.c, s = q.s, ro1 = q.ro1;
  const double c_old = q.c_old, s_old = q.s_old;
  const double delta = xsub(xmul(c, alpha), xmul(xmul(c_old, s), beta_old));
  const double ro2 = xadd(xmul(s, alpha), xmul(xmul(c_old, c), beta_old));
  const double ro3 = xmul(s_old, beta_old);
  q.c_old = c;
  q.s_old = s;
  sym_ortho_dev(delta, beta, &c, &s, &ro1);
  q.c = c;
  q.s = s;
  q.ro1 = ro1;
  q.beta_old = beta_old;
  q.beta = beta;
  const double u1 = xdiv(1.0, xmul(beta_old, ro1));
  const double u2 = xdiv(-ro2, ro1);
  const double u3 = xdiv(-ro3, ro1);
  const double u4 = xmul(c, q.neta);
  if (!isfinite(u1) || !isfinite(u2) || !isfinite(u3) || !isfinite(u4)) {
    q.status = SFR_BREAKDOWN;
    q.upd = 0;
    q.active = 0;
    q.iters = static_cast<int>(min(j + 1, q.maxit)) + 1;
  } else {
    q.u1 = u1;
    q.u2 = u2;
    q.u3 = u3;
    q.u4 = u4;
    q.upd = 1;
    const double norm_r = xmul(fabs(s), q.norm_r);
    q.norm_r = norm_r;
    if (norm_r < q.conv) {
      q.active = 0;
      q.iters = static_cast<int>(j) + 1;
    } else {
      q.neta = xmul(-s, q.neta);
      if (j + 1 >= q.maxit) {
        q.active = 0;
        q.status = SFR_MAXIT;
        q.iters = static_cast<int>(q.maxit) + 1;
      }
    }
  }
  q.j = j + 1;
}

// b: the new Lanczos vector and the scalar step (Iters.c:413-470)
__global__ void __launch_bounds__(kMrThreads) k_mr_b(const MrArgs a, int u) {
  SFR_SHARED_RED(1);
  MrState *st = a.st;
  if (!st->active) return;
  const double t1 = st->t1, t2 = st->t2, t3 = st->t3;
  const double *v0 = a.V[u % 3], *v = a.V[(u + 1) % 3];
  double *p = a.V[(u + 2) % 3];
  double *z = a.Z[(u + 1) % 2];
  double acc[1] = {0.0};
  SFR_MR_FOR_PAIRS(i) {
    const int r = 2 * i;
    const double2 pv = ld2(p + r), vv = ld2(v + r), v0v = ld2(v0 + r), mv = ld2(a.m + r);
    double2 pn, zn;
    pn.x = xadd(xadd(xmul(t1, pv.x), xmul(t2, vv.x)), xmul(t3, v0v.x));
    pn.y = xadd(xadd(xmul(t1, pv.y), xmul(t2, vv.y)), xmul(t3, v0v.y));
    zn.x = xmul(pn.x, mv.x);
    zn.y = xmul(pn.y, mv.y);
    st2(p + r, pn);
    st2(z + r, zn);
    acc[0] += zn.x * pn.x;
    if (r + 1 < a.n) acc[0] += zn.y * pn.y;
  }
  if (!last_block<1>(acc, a.part, a.counter + 3, sm)) return;
  if (threadIdx.x == 0) {
    MrState q = *st;
    mr_step(q, q.alpha, sm[0]);
    *st = q;
    if (!q.active) cudaGraphSetConditional(a.hwhile, 0u);
  }
}

// After the loop: the last iteration's w and x update (the reference breaks
// after it on convergence and at maxIt, before it on a breakdown), with that
// iteration's roles.
__global__ void __launch_bounds__(kMrThreads) k_mr_tail(const MrArgs a) {
  const MrState *st = a.st;
  if (!st->upd || st->j == 0) return;
  const int pu = static_cast<int>((st->j - 1) % kMrUnroll);
  SFR_MR_FOR_ROWS(i) mr_update_row(a, st, pu, i);
}

// One whole iteration in one cooperative launch: a, b and c above with two
// grid barriers between them.  A block keeps A z0 and z0 of its own rows in
// shared memory from phase a to phases b and c.  Each barrier's dot product
// is reduced by every block over all block partials in the same fixed
// order, and every block runs the scalar step itself on those totals, so all
// blocks take the same decisions; block 0 writes the state back.  Bounded
// barriers: a wait that gives up records SFR_TIMEOUT and the solve stops.
template <typename I>
__global__ void __launch_bounds__(kMrThreads) k_mr_fused(const MrArgs a, int u, GridSync gs) {
  __shared__ double sm[64];
  __shared__ MrState q;
  extern __shared__ double rows[];  // per own row: A z0, then z0
  MrState *st = a.st;
  if (!st->active) return;
  const int n = a.n;
  const int lane = threadIdx.x & 31;
  int s0, s1;
  block_slices(a.nslices, &s0, &s1);
  const int row0 = s0 * kWarp;
  const int nrow = (s1 - s0) * kWarp;
  const int G = gridDim.x;
  const double *z0 = a.Z[u % 2];
  const double *v0 = a.V[u % 3], *v = a.V[(u + 1) % 3];
  double *p = a.V[(u + 2) % 3];
  double *z = a.Z[(u + 1) % 2];
  const double *w00 = a.W[u % 3], *w0 = a.W[(u + 1) % 3];
  double *w = a.W[(u + 2) % 3];
  if (threadIdx.x == 0) q = *st;
  __syncthreads();
  auto fail = [&](int status) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      st->active = 0;
      st->upd = 0;
      st->status = status;
      st->iters = static_cast<int>(q.j) + 1;
      cudaGraphSetConditional(a.hwhile, 0u);
    }
  };
  // a: A z0, (z0, A z0)
  const int all[1] = {1};
  const double *const diag[1] = {a.ad};
  double acc[1] = {0.0};
  SFR_FOR_OWN_ROWS(s0, s1) {
    double y[1];
    row_product<1, true, double>(a.sptr, cols_of<I>(a.cols), a.val, diag, s_, lane, all,
                                 [&](int, int c) { return ld_ro(z0 + c); }, y);
    const double zr = ld_ro(z0 + row_);
    rows[row_ - row0] = y[0];
    rows[nrow + row_ - row0] = zr;
    acc[0] += zr * y[0];
  }
  block_partials<1>(acc, a.part, G, sm);
  if (!grid_sync(gs)) {
    fail(SFR_TIMEOUT);
    return;
  }
  double tot[1];
  grid_totals<1>(a.part, G, G, tot, sm);
  const double beta = q.beta;
  const double alpha = xmul(tot[0], xdiv(1.0, xmul(beta, beta)));
  const double t1 = xdiv(1.0, beta), t2 = xdiv(-alpha, beta), t3 = xdiv(-beta, q.beta_old);
  // b: p = t1 A z0 + t2 v + t3 v0, z = M p, (z, p)
  acc[0] = 0.0;
  SFR_FOR_OWN_ROWS(s0, s1) {
    const double pi = xadd(xadd(xmul(t1, rows[row_ - row0]), xmul(t2, ld_ro(v + row_))),
                           xmul(t3, ld_ro(v0 + row_)));
    st_vec(p + row_, pi);
    const double zi = xmul(pi, ld_ro(a.m + row_));
    st_vec(z + row_, zi);
    acc[0] += zi * pi;
  }
  block_partials<1>(acc, a.part + G, G, sm);
  if (!grid_sync(gs)) {
    fail(SFR_TIMEOUT);
    return;
  }
  grid_totals<1>(a.part + G, G, G, tot, sm);
  if (threadIdx.x == 0) {
    q.alpha = alpha;
    q.t1 = t1;
    q.t2 = t2;
    q.t3 = t3;
    mr_step(q, alpha, tot[0]);
    if (blockIdx.x == 0) {
      *st = q;
      if (!q.active) cudaGraphSetConditional(a.hwhile, 0u);
    }
  }
  __syncthreads();
  if (!q.upd) return;
  // c: w = u1 z0 + u2 w0 + u3 w00, x += u4 w
  const double u1 = q.u1, u2 = q.u2, u3 = q.u3, u4 = q.u4;
  SFR_FOR_OWN_ROWS(s0, s1) {
    const double wi = xadd(xadd(xmul(u1, rows[nrow + row_ - row0]), xmul(u2, ld_ro(w0 + row_))),
                           xmul(u3, ld_ro(w00 + row_)));
    st_vec(w + row_, wi);
    st_vec(a.x + row_, xadd(ld_vec(a.x + row_), xmul(u4, wi)));
  }
}

// post-processing: xKx, ||x||, ||b - A x||, ||M^1/2 (b - A x)||
template <typename I>
__global__ void __launch_bounds__(kMrThreads) k_mr_post(const MrArgs a) {
  SFR_SHARED_RED(4);
  MrState *st = a.st;
  const int n = a.n;
  const int lane = threadIdx.x & 31;
  int s0, s1;
  block_slices(a.nslices, &s0, &s1);
  const int all[1] = {1};
  const double *const diag[1] = {a.ad};
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  SFR_FOR_OWN_ROWS(s0, s1) {
    double y[1];
    row_product<1, true, double>(a.sptr, cols_of<I>(a.cols), a.val, diag, s_, lane, all,
                                 [&](int, int c) { return ld_ro(a.x + c); }, y);
    const double xi = a.x[row_];
    const double ri = xsub(a.b[row_], y[0]);
    const double ti = xmul(ri, sqrt(fabs(a.m[row_])));
    acc[0] += xi * y[0];
    acc[1] += xi * xi;
    acc[2] += ri * ri;
    acc[3] += ti * ti;
  }
  if (!last_block<4>(acc, a.part, a.counter + 4, sm)) return;
  if (threadIdx.x == 0) {
    st->xKx = sm[0];
    st->norm_x = sqrt(sm[1]);
    st->norm_r_true = sqrt(sm[2]);
    st->norm_r_m = sqrt(sm[3]);
  }
}

#define SFR_TRY(expr)                 \
  do {                                \
    cudaError_t e_ = (expr);          \
    if (e_ != cudaSuccess) return e_; \
  } while (0)

struct MrGraph {
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  void *ws = nullptr;
  MrArgs args{};
  int gs = 0, gv = 0;
  int gf = 0;         // fused iteration: co-resident blocks (0: three kernels)
  size_t smem_f = 0;  // fused iteration: dynamic shared memory a block
  int fused = 0;      // the handle's fused-iteration option this graph was built for
};

// The fused iteration's launch shape: the most co-resident blocks whose
// shared memory (16 bytes a row of the block's slices) still lets them all
// be resident at once; 0 when none does.
template <typename I>
int mr_fused_shape(const sfr_system *s, size_t *smem) {
  const int sms = std::max(1, num_sms(s->device));
  const int nsl = s->A.nslices;
  const int maxg = std::max(1, (nsl + 7) / 8);
  for (int per_sm = 8; per_sm >= 1; --per_sm) {
    const int G = std::min(maxg, per_sm * sms);
    const size_t bytes = static_cast<size_t>((nsl + G - 1) / G) * kWarp * 2 * sizeof(double);
    if (bytes > 200 * 1024) continue;
    if (cudaFuncSetAttribute(k_mr_fused<I>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(bytes)) != cudaSuccess)
      continue;
    int occ = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_mr_fused<I>, kMrThreads, bytes) !=
        cudaSuccess)
      continue;
    if (occ * sms >= G) {
      *smem = bytes;
      return G;
    }
  }
  return 0;
}

std::map<const sfr_system *, std::unique_ptr<MrGraph>> g_mr;

void free_mr(MrGraph *g) {
  if (g->exec) cudaGraphExecDestroy(g->exec);
  if (g->graph) cudaGraphDestroy(g->graph);
  cudaFree(g->ws);
  *g = MrGraph{};
}

cudaError_t node(cudaGraph_t g, cudaGraphNode_t *prev, void *func, int grid, void **params) {
  cudaKernelNodeParams p{};
  p.func = func;
  p.gridDim = dim3(grid);
  p.blockDim = dim3(kMrThreads);
  p.kernelParams = params;
  cudaGraphNode_t nd;
  const cudaError_t e = cudaGraphAddKernelNode(&nd, g, *prev ? prev : nullptr, *prev ? 1 : 0, &p);
  if (e == cudaSuccess) *prev = nd;
  return e;
}

template <typename I>
cudaError_t build(sfr_system *s, int fused, MrGraph *g) {
  g->fused = fused;
  const int n = s->n;
  const size_t vb = (sizeof(double) * static_cast<size_t>(std::max(n, 1)) + 255) & ~size_t{255};
  int occ = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_mr_a<I>, kMrThreads, 0) !=
          cudaSuccess ||
      occ < 1)
    occ = 1;
  const int sms = std::max(1, num_sms(s->device));
  g->gs = std::max(1, std::min((s->A.nslices + 7) / 8, occ * sms));
  const int npairs = (n + 1) / 2;  // the vector phases move row pairs
  g->gv = std::max(1, std::min(sms * (2048 / kMrThreads), (npairs + kMrThreads - 1) / kMrThreads));
  const int gmax = std::max(g->gs, g->gv);
  const size_t part_b = (sizeof(double) * 4 * static_cast<size_t>(gmax) + 255) & ~size_t{255};
  const size_t total = vb * 12 + part_b + 256 + sizeof(MrState);
  SFR_TRY(cudaMalloc(&g->ws, total));
  SFR_TRY(cudaMemset(g->ws, 0, total));
  char *base = static_cast<char *>(g->ws);
  auto V = [&](int i) { return reinterpret_cast<double *>(base + vb * i); };
  MrArgs &a = g->args;
  a.n = n;
  a.nslices = s->A.nslices;
  a.sptr = s->A.sptr;
  a.cols = SlotCols{s->A.col, s->A.off};
  a.val = s->A.val;
  a.ad = V(0);
  a.b = V(1);
  a.x = V(2);
  a.m = V(3);
  for (int i = 0; i < 3; ++i) a.V[i] = V(4 + i);
  for (int i = 0; i < 2; ++i) a.Z[i] = V(7 + i);
  for (int i = 0; i < 3; ++i) a.W[i] = V(9 + i);
  a.part = reinterpret_cast<double *>(base + vb * 12);
  a.counter = reinterpret_cast<unsigned *>(base + vb * 12 + part_b);
  a.st = reinterpret_cast<MrState *>(base + vb * 12 + part_b + 256);

  SFR_TRY(cudaGraphCreate(&g->graph, 0));
  SFR_TRY(cudaGraphConditionalHandleCreate(&a.hwhile, g->graph, 1, cudaGraphCondAssignDefault));
  cudaGraphNode_t prev = nullptr;
  {
    cudaMemsetParams mp{};
    mp.dst = a.counter;
    mp.value = 0;
    mp.elementSize = sizeof(unsigned);
    mp.width = kMrCounters;
    mp.height = 1;
    SFR_TRY(cudaGraphAddMemsetNode(&prev, g->graph, nullptr, 0, &mp));
  }
  void *p1[1] = {&a};
  SFR_TRY(node(g->graph, &prev, (void *)k_mr_setup1, g->gv, p1));
  SFR_TRY(node(g->graph, &prev, (void *)k_mr_setup2<I>, g->gs, p1));
  cudaGraphNodeParams cp{};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = a.hwhile;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  cudaGraphNode_t wn;
  SFR_TRY(cudaGraphAddNode(&wn, g->graph, &prev, 1, &cp));
  prev = wn;
  cudaGraph_t body = cp.conditional.phGraph_out[0];
  cudaGraphNode_t bp = nullptr;
  int us[kMrUnroll];
  void *pu[kMrUnroll][3];
  g->gf = fused ? mr_fused_shape<I>(s, &g->smem_f) : 0;
  GridSync gsync;
  gsync.count = a.counter + 12;
  gsync.gen = a.counter + 13;
  gsync.err = reinterpret_cast<int *>(a.counter + 14);
  gsync.nblocks = static_cast<unsigned>(g->gf);
  gsync.spin_limit = 1u << 22;
  for (int u = 0; u < kMrUnroll; ++u) {
    us[u] = u;
    pu[u][0] = &a;
    pu[u][1] = &us[u];
    pu[u][2] = &gsync;
    if (g->gf > 0) {
      // one cooperative kernel an iteration
      cudaKernelNodeParams kp{};
      kp.func = (void *)k_mr_fused<I>;
      kp.gridDim = dim3(g->gf);
      kp.blockDim = dim3(kMrThreads);
      kp.sharedMemBytes = static_cast<unsigned>(g->smem_f);
      kp.kernelParams = pu[u];
      cudaGraphNode_t fn;
      SFR_TRY(cudaGraphAddKernelNode(&fn, body, bp ? &bp : nullptr, bp ? 1 : 0, &kp));
      cudaKernelNodeAttrValue coop{};
      coop.cooperative = 1;
      SFR_TRY(cudaGraphKernelNodeSetAttribute(fn, cudaLaunchAttributeCooperative, &coop));
      bp = fn;
    } else {
      SFR_TRY(node(body, &bp, (void *)k_mr_a<I>, g->gs, pu[u]));
      SFR_TRY(node(body, &bp, (void *)k_mr_b, g->gv, pu[u]));
    }
  }
  // the fused kernel updates w and x itself; the two-kernel body leaves the
  // last iteration's update to the tail
  if (!g->gf) SFR_TRY(node(g->graph, &prev, (void *)k_mr_tail, g->gv, p1));
  SFR_TRY(node(g->graph, &prev, (void *)k_mr_post<I>, g->gs, p1));
  SFR_TRY(cudaGraphInstantiate(&g->exec, g->graph, 0));
  return cudaSuccess;
}

}  // namespace

int solve_minres_graph(sfr_system *s, const double *d_diag, const double *d_b, double *d_x,
                       double tol, uint32_t maxit, int32_t newx, cudaStream_t st,
                       sfr_solve_info *info) {
  auto &slot = g_mr[s];
  const int fused = s->graph_fused ? 1 : 0;
  if (slot && slot->fused != fused) {
    free_mr(slot.get());
    slot.reset();
  }
  if (!slot) {
    slot = std::make_unique<MrGraph>();
    const cudaError_t be =
        s->A.off ? build<int16_t>(s, fused, slot.get()) : build<int>(s, fused, slot.get());
    if (be != cudaSuccess) {
      set_last_error(cudaGetErrorString(be));
      free_mr(slot.get());
      g_mr.erase(s);
      return SFR_CUDA_ERROR;
    }
  }
  MrGraph *g = slot.get();
  const MrArgs &a = g->args;
  const size_t vb = sizeof(double) * static_cast<size_t>(s->n);
  MrState call{};
  call.tol = tol;
  call.maxit = maxit;
  call.newx = newx;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (cudaEventCreate(&e0) != cudaSuccess) return SFR_CUDA_ERROR;
  if (cudaEventCreate(&e1) != cudaSuccess) {
    cudaEventDestroy(e0);
    return SFR_CUDA_ERROR;
  }
  cudaError_t err = cudaEventRecord(e0, st);
  if (err == cudaSuccess)
    err = cudaMemcpyAsync(a.ad, d_diag ? d_diag : s->d_diag, vb, cudaMemcpyDeviceToDevice, st);
  if (err == cudaSuccess) err = cudaMemcpyAsync(a.b, d_b, vb, cudaMemcpyDeviceToDevice, st);
  if (err == cudaSuccess && !newx)
    err = cudaMemcpyAsync(a.x, d_x, vb, cudaMemcpyDeviceToDevice, st);
  if (err == cudaSuccess)
    err = cudaMemcpyAsync(a.st, &call, offsetof(MrState, conv), cudaMemcpyHostToDevice, st);
  if (err == cudaSuccess) err = cudaGraphLaunch(g->exec, st);
  if (err == cudaSuccess) err = cudaMemcpyAsync(d_x, a.x, vb, cudaMemcpyDeviceToDevice, st);
  if (err == cudaSuccess) err = cudaEventRecord(e1, st);
  MrState out{};
  if (err == cudaSuccess)
    err = cudaMemcpyAsync(&out, a.st, sizeof(MrState), cudaMemcpyDeviceToHost, st);
  if (err == cudaSuccess) err = cudaStreamSynchronize(st);
  float ms = 0.f;
  if (err == cudaSuccess) cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (err != cudaSuccess) {
    set_last_error(cudaGetErrorString(err));
    return SFR_CUDA_ERROR;
  }
  if (info) {
    std::memset(info, 0, sizeof(*info));
    info->iters = out.iters;
    info->status = out.status;
    info->xKx = out.xKx;
    info->norm_x = out.norm_x;
    info->norm_r = out.norm_r_true;
    info->norm_r_m = out.norm_r_m;
    info->conv = out.conv;
    info->seconds = ms * 1e-3;
    info->refinements = 0;
    info->inner_iters = out.iters;
    info->relres = std::nan("");
  }
  return out.status;
}

void release_minres_graph(const sfr_system *s) {
  auto it = g_mr.find(s);
  if (it == g_mr.end()) return;
  free_mr(it->second.get());
  g_mr.erase(it);
}

}  // namespace sfr
