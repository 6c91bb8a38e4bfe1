// BiCGSTAB(2) (Bicgstab.c:1172-1460, pbicgstabl2) with its scalar recurrence
// on the device: the whole solve is one CUDA graph whose iteration loop is a
// conditional WHILE node, like the graph engine's PCG (stream_solve.cu), so no
// dot product travels to the host.
//
// One iteration is nine kernels, four of them SpMV phases; every dot product
// is formed by the kernel that produces its operand and finished by the last
// block to arrive, which also computes the scalars the next kernel needs:
//   A. u = u - (w1 v + w2 w) (from the second iteration on), u = r - beta u,
//      z = M u;
//   B. v = A z, (v, r0) -> alpha = rr0 / (v, r0);
//   C. r = r - alpha v, p = M r, x = x + alpha z;
//   D. s = A p, (s, r0) -> beta = alpha (s, r0) / rr0, rr0 = (s, r0);
//   E. v = s - beta v, p = M v;
//   F. w = A p, (w, r0) -> alpha = rr0 / (w, r0);
//   G. u = r - beta u, r = r - alpha v, s = s - alpha w, p = M s, z = M u,
//      h = M r;
//   H. t = A p and the GCR(2) products (r,s), (s,s), (s,t), (t,t), (r,t) ->
//      tau, omega2, omega1; a non-finite omega or alpha is a breakdown (the
//      reference breaks before its update);
//   I. x = x + ((w1 h + w2 p) + alpha z), r = r - (w1 s + w2 t), (r, r) and
//      (r, r0) -> the stopping test sqrt(r, r) < tol ||b||, and the next
//      iteration's rr0 = -w2 rr0, beta = alpha (r, r0) / rr0, rr0 = (r, r0).
// Every scalar is the reference's expression in its order, each operation
// rounded once (no FMA contraction, IEEE division and square root), and every
// vector element the reference's C expression, so the recurrence differs from
// the reference only through the dot products' summation order.
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

constexpr int kBlThreads = 256;
constexpr int kBlCounters = 16;

struct BlState {
  // per call
  double tol;
  unsigned maxit;
  int newx;
  // recurrence
  double conv, rr0, alpha, beta, omega1, omega2;
  unsigned j;
  int active, status, iters;
  // post-processing
  double xKx, norm_x, norm_r;
};

struct BlArgs {
  int n, nslices;
  const int *sptr;
  SlotCols cols;
  const double *val;
  double *ad, *b, *x, *m;  // the graph's own copies of the diagonal, b and x
  double *t, *v, *r, *u, *r0, *w, *s, *p, *h, *z;
  double *part;
  unsigned *counter;
  BlState *st;
  cudaGraphConditionalHandle hwhile;
};

#define SFR_BL_FOR_ROWS(i) \
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += gridDim.x * blockDim.x)


// y = A g over this warp's rows (the reference's row rounding); defines y0
// for the body.  The diagonal is the graph's copy of the caller's.
#define SFR_BL_SPMV_ROWS(g, ...)                                                           \
  {                                                                                        \
    const int n = a.n;                                                                     \
    const int lane = threadIdx.x & 31;                                                     \
    int s0, s1;                                                                            \
    block_slices(a.nslices, &s0, &s1);                                                     \
    const int all[1] = {1};                                                                \
    const double *const diag[1] = {a.ad};                                                  \
    SFR_FOR_OWN_ROWS(s0, s1) {                                                             \
      double yv[1];                                                                        \
      row_product<1, true, double>(a.sptr, cols_of<I>(a.cols), a.val, diag, s_, lane, all, \
                                   [&](int, int c) { return ld_ro((g) + c); }, yv);        \
      const double y0 = yv[0];                                                             \
      const int i = row_;                                                                  \
      __VA_ARGS__                                                                          \
    }                                                                                      \
  }

// m = 1/ad, x0; conv = tol ||b||  (Bicgstab.c:1215-1232)
__global__ void __launch_bounds__(kBlThreads) k_bl_setup1(const BlArgs a) {
  SFR_SHARED_RED(1);
  BlState *st = a.st;
  const int newx = st->newx;
  double acc[1] = {0.0};
  SFR_BL_FOR_ROWS(i) {
    a.m[i] = 1.0 / a.ad[i];
    if (newx) a.x[i] = 0.0;
    const double bi = a.b[i];
    acc[0] += bi * bi;
  }
  if (!last_block<1>(acc, a.part, a.counter + 0, sm)) return;
  if (threadIdx.x == 0) st->conv = xmul(st->tol, sqrt(sm[0]));
}

// r0 = r = b - A x, u = 0 (Bicgstab.c:1234-1246); the first iteration's
// (r, r0) and its scalars (rr0 = 1, alpha = 0, omega2 = 1 before it)
template <typename I>
__global__ void __launch_bounds__(kBlThreads) k_bl_setup2(const BlArgs a) {
  SFR_SHARED_RED(1);
  BlState *st = a.st;
  double acc[1] = {0.0};
  SFR_BL_SPMV_ROWS(a.x, {
    const double ri = xsub(a.b[i], y0);
    a.r0[i] = ri;
    a.r[i] = ri;
    a.u[i] = 0.0;
    acc[0] += ri * ri;
  })
  if (!last_block<1>(acc, a.part, a.counter + 1, sm)) return;
  if (threadIdx.x == 0) {
    const double alpha = 0.0, omega2 = 1.0;
    const double rr0 = xmul(-omega2, 1.0);
    const double rr1 = sm[0];
    st->beta = xdiv(xmul(alpha, rr1), rr0);
    st->rr0 = rr1;
    st->alpha = alpha;
    st->omega2 = omega2;
    st->j = 0;
    st->status = SFR_OK;
    st->active = st->maxit > 0 ? 1 : 0;
    if (!st->active) {
      st->status = SFR_MAXIT;
      st->iters = 1;
      cudaGraphSetConditional(a.hwhile, 0u);
    }
  }
}

// A: the previous iteration's u update, then u = r - beta u, z = M u
__global__ void __launch_bounds__(kBlThreads) k_bl_a(const BlArgs a) {
  BlState *st = a.st;
  if (!st->active) return;
  const bool later = st->j > 0;
  const double o1 = st->omega1, o2 = st->omega2, beta = st->beta;
  SFR_BL_FOR_ROWS(i) {
    double ui = a.u[i];
    if (later) ui = xsub(ui, xadd(xmul(o1, ld_ro(a.v + i)), xmul(o2, ld_ro(a.w + i))));
    ui = xsub(ld_ro(a.r + i), xmul(beta, ui));
    a.u[i] = ui;
    a.z[i] = xmul(ui, ld_ro(a.m + i));
  }
}

// B: v = A z, alpha = rr0 / (v, r0)
template <typename I>
__global__ void __launch_bounds__(kBlThreads) k_bl_b(const BlArgs a) {
  SFR_SHARED_RED(1);
  BlState *st = a.st;
  if (!st->active) return;
  double acc[1] = {0.0};
  SFR_BL_SPMV_ROWS(a.z, {
    st_vec(a.v + i, y0);
    acc[0] += y0 * ld_ro(a.r0 + i);
  })
  if (!last_block<1>(acc, a.part, a.counter + 2, sm)) return;
  if (threadIdx.x == 0) st->alpha = xdiv(st->rr0, sm[0]);
}

// C: r = r - alpha v, p = M r, x = x + alpha z
__global__ void __launch_bounds__(kBlThreads) k_bl_c(const BlArgs a) {
  BlState *st = a.st;
  if (!st->active) return;
  const double alpha = st->alpha;
  SFR_BL_FOR_ROWS(i) {
    const double ri = xsub(a.r[i], xmul(alpha, ld_ro(a.v + i)));
    a.r[i] = ri;
    a.p[i] = xmul(ri, ld_ro(a.m + i));
    a.x[i] = xadd(a.x[i], xmul(alpha, ld_ro(a.z + i)));
  }
}

// D: s = A p, beta = alpha (s, r0) / rr0, rr0 = (s, r0)
template <typename I>
__global__ void __launch_bounds__(kBlThreads) k_bl_d(const BlArgs a) {
  SFR_SHARED_RED(1);
  BlState *st = a.st;
  if (!st->active) return;
  double acc[1] = {0.0};
  SFR_BL_SPMV_ROWS(a.p, {
    st_vec(a.s + i, y0);
    acc[0] += y0 * ld_ro(a.r0 + i);
  })
  if (!last_block<1>(acc, a.part, a.counter + 3, sm)) return;
  if (threadIdx.x == 0) {
    const double rr1 = sm[0];
    st->beta = xdiv(xmul(st->alpha, rr1), st->rr0);
    st->rr0 = rr1;
  }
}

// E: v = s - beta v, p = M v
__global__ void __launch_bounds__(kBlThreads) k_bl_e(const BlArgs a) {
  BlState *st = a.st;
  if (!st->active) return;
  const double beta = st->beta;
  SFR_BL_FOR_ROWS(i) {
    const double vi = xsub(ld_ro(a.s + i), xmul(beta, a.v[i]));
    a.v[i] = vi;
    a.p[i] = xmul(vi, ld_ro(a.m + i));
  }
}

// F: w = A p, alpha = rr0 / (w, r0)
template <typename I>
__global__ void __launch_bounds__(kBlThreads) k_bl_f(const BlArgs a) {
  SFR_SHARED_RED(1);
  BlState *st = a.st;
  if (!st->active) return;
  double acc[1] = {0.0};
  SFR_BL_SPMV_ROWS(a.p, {
    st_vec(a.w + i, y0);
    acc[0] += y0 * ld_ro(a.r0 + i);
  })
  if (!last_block<1>(acc, a.part, a.counter + 4, sm)) return;
  if (threadIdx.x == 0) st->alpha = xdiv(st->rr0, sm[0]);
}

// G: u = r - beta u, r = r - alpha v, s = s - alpha w, p = M s, z = M u,
// h = M r
__global__ void __launch_bounds__(kBlThreads) k_bl_g(const BlArgs a) {
  BlState *st = a.st;
  if (!st->active) return;
  const double alpha = st->alpha, beta = st->beta;
  SFR_BL_FOR_ROWS(i) {
    const double mi = ld_ro(a.m + i);
    const double ri = a.r[i];
    const double ui = xsub(ri, xmul(beta, a.u[i]));
    const double rn = xsub(ri, xmul(alpha, ld_ro(a.v + i)));
    const double si = xsub(a.s[i], xmul(alpha, ld_ro(a.w + i)));
    a.u[i] = ui;
    a.r[i] = rn;
    a.s[i] = si;
    a.p[i] = xmul(si, mi);
    a.z[i] = xmul(ui, mi);
    a.h[i] = xmul(rn, mi);
  }
}

// H: t = A p and the GCR(2) part (Bicgstab.c:1378-1398)
template <typename I>
__global__ void __launch_bounds__(kBlThreads) k_bl_h(const BlArgs a) {
  SFR_SHARED_RED(5);
  BlState *st = a.st;
  if (!st->active) return;
  double acc[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  SFR_BL_SPMV_ROWS(a.p, {
    st_vec(a.t + i, y0);
    const double ri = ld_ro(a.r + i), si = ld_ro(a.s + i);
    acc[0] += ri * si;
    acc[1] += si * si;
    acc[2] += si * y0;
    acc[3] += y0 * y0;
    acc[4] += ri * y0;
  })
  if (!last_block<5>(acc, a.part, a.counter + 5, sm)) return;
  if (threadIdx.x == 0) {
    double omega1 = sm[0];
    const double mi = sm[1], ni = sm[2];
    double tau = sm[3];
    double omega2 = sm[4];
    tau = xsub(tau, xdiv(xmul(ni, ni), mi));
    omega2 = xdiv(xsub(omega2, xdiv(xmul(ni, omega1), mi)), tau);
    omega1 = xdiv(xsub(omega1, xmul(ni, omega2)), mi);
    st->omega1 = omega1;
    st->omega2 = omega2;
    if (!isfinite(omega1) || !isfinite(omega2) || !isfinite(st->alpha)) {
      const unsigned j = st->j;
      st->status = SFR_BREAKDOWN;
      st->active = 0;
      st->iters = static_cast<int>(min(j + 1, st->maxit)) + 1;
      cudaGraphSetConditional(a.hwhile, 0u);
    }
  }
}

// I: the x and r updates, the stopping test and the next iteration's
// scalars (Bicgstab.c:1400-1424, then 1297-1302)
__global__ void __launch_bounds__(kBlThreads) k_bl_i(const BlArgs a) {
  SFR_SHARED_RED(2);
  BlState *st = a.st;
  if (!st->active) return;
  const double o1 = st->omega1, o2 = st->omega2, alpha = st->alpha;
  double acc[2] = {0.0, 0.0};
  SFR_BL_FOR_ROWS(i) {
    const double xi =
        xadd(a.x[i], xadd(xadd(xmul(o1, ld_ro(a.h + i)), xmul(o2, ld_ro(a.p + i))),
                          xmul(alpha, ld_ro(a.z + i))));
    a.x[i] = xi;
    const double ri =
        xsub(a.r[i], xadd(xmul(o1, ld_ro(a.s + i)), xmul(o2, ld_ro(a.t + i))));
    a.r[i] = ri;
    acc[0] += ri * ri;
    acc[1] += ri * ld_ro(a.r0 + i);
  }
  if (!last_block<2>(acc, a.part, a.counter + 6, sm)) return;
  if (threadIdx.x == 0) {
    const unsigned j = st->j;
    if (sqrt(sm[0]) < st->conv) {
      st->active = 0;
      st->iters = static_cast<int>(j) + 1;
    } else if (j + 1 >= st->maxit) {
      st->active = 0;
      st->status = SFR_MAXIT;
      st->iters = static_cast<int>(st->maxit) + 1;
    } else {
      // the next iteration's first scalars (rr0 = -omega2 rr0; beta)
      const double rr0 = xmul(-o2, st->rr0);
      const double rr1 = sm[1];
      st->beta = xdiv(xmul(alpha, rr1), rr0);
      st->rr0 = rr1;
    }
    st->j = j + 1;
    if (!st->active) cudaGraphSetConditional(a.hwhile, 0u);
  }
}

// post-processing: xKx, ||x||, ||b - A x||
template <typename I>
__global__ void __launch_bounds__(kBlThreads) k_bl_post(const BlArgs a) {
  SFR_SHARED_RED(3);
  BlState *st = a.st;
  double acc[3] = {0.0, 0.0, 0.0};
  SFR_BL_SPMV_ROWS(a.x, {
    const double xi = a.x[i];
    const double ri = xsub(a.b[i], y0);
    acc[0] += xi * y0;
    acc[1] += xi * xi;
    acc[2] += ri * ri;
  })
  if (!last_block<3>(acc, a.part, a.counter + 7, sm)) return;
  if (threadIdx.x == 0) {
    st->xKx = sm[0];
    st->norm_x = sqrt(sm[1]);
    st->norm_r = sqrt(sm[2]);
  }
}

#define SFR_TRY(expr)                 \
  do {                                \
    cudaError_t e_ = (expr);          \
    if (e_ != cudaSuccess) return e_; \
  } while (0)

struct BlGraph {
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  void *ws = nullptr;
  BlArgs args{};
  int gs = 0, gv = 0;
};

std::map<const sfr_system *, std::unique_ptr<BlGraph>> g_bl;

void free_bl(BlGraph *g) {
  if (g->exec) cudaGraphExecDestroy(g->exec);
  if (g->graph) cudaGraphDestroy(g->graph);
  cudaFree(g->ws);
  *g = BlGraph{};
}

cudaError_t node(cudaGraph_t g, cudaGraphNode_t *prev, void *func, int grid, void **params) {
  cudaKernelNodeParams p{};
  p.func = func;
  p.gridDim = dim3(grid);
  p.blockDim = dim3(kBlThreads);
  p.kernelParams = params;
  cudaGraphNode_t nd;
  const cudaError_t e = cudaGraphAddKernelNode(&nd, g, *prev ? prev : nullptr, *prev ? 1 : 0, &p);
  if (e == cudaSuccess) *prev = nd;
  return e;
}

template <typename I>
cudaError_t build(sfr_system *s, BlGraph *g) {
  const int n = s->n;
  const size_t vb = (sizeof(double) * static_cast<size_t>(std::max(n, 1)) + 255) & ~size_t{255};
  int occ = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_bl_h<I>, kBlThreads, 0) !=
          cudaSuccess ||
      occ < 1)
    occ = 1;
  const int sms = std::max(1, num_sms(s->device));
  g->gs = std::max(1, std::min((s->A.nslices + 7) / 8, occ * sms));
  g->gv = std::max(1, std::min(sms * (2048 / kBlThreads), (n + kBlThreads - 1) / kBlThreads));
  const int gmax = std::max(g->gs, g->gv);
  constexpr int kVecs = 14;
  const size_t part_b = (sizeof(double) * 5 * static_cast<size_t>(gmax) + 255) & ~size_t{255};
  const size_t total = vb * kVecs + part_b + 256 + sizeof(BlState);
  SFR_TRY(cudaMalloc(&g->ws, total));
  SFR_TRY(cudaMemset(g->ws, 0, total));
  char *base = static_cast<char *>(g->ws);
  auto V = [&](int i) { return reinterpret_cast<double *>(base + vb * i); };
  BlArgs &a = g->args;
  a.n = n;
  a.nslices = s->A.nslices;
  a.sptr = s->A.sptr;
  a.cols = SlotCols{s->A.col, s->A.off};
  a.val = s->A.val;
  a.ad = V(0);
  a.b = V(1);
  a.x = V(2);
  a.m = V(3);
  a.t = V(4);
  a.v = V(5);
  a.r = V(6);
  a.u = V(7);
  a.r0 = V(8);
  a.w = V(9);
  a.s = V(10);
  a.p = V(11);
  a.h = V(12);
  a.z = V(13);
  a.part = reinterpret_cast<double *>(base + vb * kVecs);
  a.counter = reinterpret_cast<unsigned *>(base + vb * kVecs + part_b);
  a.st = reinterpret_cast<BlState *>(base + vb * kVecs + part_b + 256);

  SFR_TRY(cudaGraphCreate(&g->graph, 0));
  SFR_TRY(cudaGraphConditionalHandleCreate(&a.hwhile, g->graph, 1, cudaGraphCondAssignDefault));
  cudaGraphNode_t prev = nullptr;
  {
    cudaMemsetParams mp{};
    mp.dst = a.counter;
    mp.value = 0;
    mp.elementSize = sizeof(unsigned);
    mp.width = kBlCounters;
    mp.height = 1;
    SFR_TRY(cudaGraphAddMemsetNode(&prev, g->graph, nullptr, 0, &mp));
  }
  void *p1[1] = {&a};
  SFR_TRY(node(g->graph, &prev, (void *)k_bl_setup1, g->gv, p1));
  SFR_TRY(node(g->graph, &prev, (void *)k_bl_setup2<I>, g->gs, p1));
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
  SFR_TRY(node(body, &bp, (void *)k_bl_a, g->gv, p1));
  SFR_TRY(node(body, &bp, (void *)k_bl_b<I>, g->gs, p1));
  SFR_TRY(node(body, &bp, (void *)k_bl_c, g->gv, p1));
  SFR_TRY(node(body, &bp, (void *)k_bl_d<I>, g->gs, p1));
  SFR_TRY(node(body, &bp, (void *)k_bl_e, g->gv, p1));
  SFR_TRY(node(body, &bp, (void *)k_bl_f<I>, g->gs, p1));
  SFR_TRY(node(body, &bp, (void *)k_bl_g, g->gv, p1));
  SFR_TRY(node(body, &bp, (void *)k_bl_h<I>, g->gs, p1));
  SFR_TRY(node(body, &bp, (void *)k_bl_i, g->gv, p1));
  SFR_TRY(node(g->graph, &prev, (void *)k_bl_post<I>, g->gs, p1));
  SFR_TRY(cudaGraphInstantiate(&g->exec, g->graph, 0));
  return cudaSuccess;
}

}  // namespace

int solve_bicgstabl2_graph(sfr_system *s, const double *d_diag, const double *d_b, double *d_x,
                           double tol, uint32_t maxit, int32_t newx, cudaStream_t st,
                           sfr_solve_info *info) {
  auto &slot = g_bl[s];
  if (!slot) {
    slot = std::make_unique<BlGraph>();
    const cudaError_t be = s->A.off ? build<int16_t>(s, slot.get()) : build<int>(s, slot.get());
    if (be != cudaSuccess) {
      set_last_error(cudaGetErrorString(be));
      free_bl(slot.get());
      g_bl.erase(s);
      return SFR_CUDA_ERROR;
    }
  }
  BlGraph *g = slot.get();
  const BlArgs &a = g->args;
  const size_t vb = sizeof(double) * static_cast<size_t>(s->n);
  BlState call{};
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
    err = cudaMemcpyAsync(a.st, &call, offsetof(BlState, conv), cudaMemcpyHostToDevice, st);
  if (err == cudaSuccess) err = cudaGraphLaunch(g->exec, st);
  if (err == cudaSuccess) err = cudaMemcpyAsync(d_x, a.x, vb, cudaMemcpyDeviceToDevice, st);
  if (err == cudaSuccess) err = cudaEventRecord(e1, st);
  BlState out{};
  if (err == cudaSuccess)
    err = cudaMemcpyAsync(&out, a.st, sizeof(BlState), cudaMemcpyDeviceToHost, st);
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
    info->norm_r = out.norm_r;
    info->norm_r_m = 0.0;
    info->conv = out.conv;
    info->seconds = ms * 1e-3;
    info->refinements = 0;
    info->inner_iters = out.iters;
    info->relres = std::nan("");
  }
  return out.status;
}

void release_bicgstabl2_graph(const sfr_system *s) {
  auto it = g_bl.find(s);
  if (it == g_bl.end()) return;
  free_bl(it->second.get());
  g_bl.erase(it);
}

}  // namespace sfr
