// Restarted GMRES(15) (Iters.c:587-800, gmres) with its scalar recurrence on
// the device: the whole solve is one CUDA graph whose restart loop is a
// conditional WHILE node, like the graph engine's PCG (stream_solve.cu), so
// no Gram-Schmidt coefficient travels to the host.
//
// A cycle of the graph:
//   res.   t = M (b - A x), (t, t) -> e_0 = sqrt, inv = 1 / e_0;
//   step ni = 0..14, ni + 2 kernels each:
//     spmv.  g_ni = inv src (src: t, or the previous step's raw vector),
//            w = M A g_ni (the gathers scale src on the fly, so they see the
//            same rounded g_ni the row stores), (w, g_0) -> H(0, ni);
//     mgs jj = 1..ni.  w -= H(jj-1, ni) g_(jj-1), (w, g_jj) -> H(jj, ni);
//     last.  w -= H(ni, ni) g_ni, (w, w) -> H(ni+1, ni) = sqrt, inv = 1 / it,
//            the earlier Givens rotations applied to column ni, the new one
//            formed, e_(ni+1) = -s e_ni, e_ni = c e_ni;
//   y.     back substitution over the first 14 directions and the restart
//          test |e_15| < eConv, the cycle cap, a non-finite y (breakdown);
//   x.     x += sum_(k<14) y_k g_k, unless y broke down.
// The raw Arnoldi vector alternates between two buffers from step to step,
// so a step's gathers never read a row its own kernel rewrites.  Every
// dot product is finished by the last block of the kernel that forms it.
// The reference's quirks are kept: a cycle always runs all 15 Arnoldi
// steps, x is updated with the first nk - 1 = 14 directions, the back
// substitution of y_i runs over j < ni, maxit counts cycles and the
// iteration count is 15 cycles + 1.  Every scalar is the reference's
// expression in its order with one rounding per operation (xmul/xadd/xdiv,
// IEEE square root), every vector element the reference's C expression, so
// the solve differs from the reference only through the dot products'
// summation order.
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

constexpr int kGmThreads = 256;
constexpr int kGmNk = 15;  // solverC's nKrylov (Solv.c:82)
constexpr int kGmCounters = 4;

struct GmState {
  // per call
  double tol;
  unsigned maxit;
  int newx;
  // recurrence
  double conv;
  double h[(kGmNk + 1) * kGmNk];  // H(row, col) = h[row * nk + col]
  double c[kGmNk], s[kGmNk], e[kGmNk + 1], y[kGmNk];
  double inv;  // 1 / the norm of the vector the next step normalises
  unsigned l;  // cycles done
  int nit;     // Arnoldi steps done
  int active, broke, status, iters;
  // post-processing
  double xKx, norm_x, norm_r;
};

struct GmArgs {
  int n, nslices;
  const int *sptr;
  SlotCols cols;
  const double *val;
  double *ad, *b, *x, *m;  // the graph's own copies of the diagonal, b and x
  double *g[kGmNk + 1];    // the cycle's Krylov basis
  double *w[2];            // the raw Arnoldi vector, alternating by step
  double *t;               // M (b - A x), before its normalisation
  double *part;
  unsigned *counter;
  GmState *st;
  cudaGraphConditionalHandle hwhile;
};

#define SFR_GM_FOR_ROWS(i) \
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += gridDim.x * blockDim.x)

__device__ __forceinline__ double &H(GmState *st, int row, int col) {
  return st->h[row * kGmNk + col];
}

// m = 1/ad, x0, eConv = tol ||M b||  (Iters.c:618-631)
__global__ void __launch_bounds__(kGmThreads) k_gm_setup(const GmArgs a) {
  SFR_SHARED_RED(1);
  GmState *st = a.st;
  const int newx = st->newx;
  double acc[1] = {0.0};
  SFR_GM_FOR_ROWS(i) {
    const double mi = 1.0 / a.ad[i];
    a.m[i] = mi;
    if (newx) a.x[i] = 0.0;
    const double gi = xmul(a.b[i], mi);
    acc[0] += gi * gi;
  }
  if (!last_block<1>(acc, a.part, a.counter, sm)) return;
  if (threadIdx.x == 0) {
    st->conv = xmul(st->tol, xsqrt(sm[0]));
    st->l = 0;
    st->nit = 0;
    st->broke = 0;
    st->status = SFR_OK;
    st->active = st->maxit > 0 ? 1 : 0;
    for (int k = 0; k < kGmNk; ++k) {
      st->c[k] = 0.0;
      st->s[k] = 0.0;
      st->y[k] = 0.0;
    }
    for (int k = 0; k < (kGmNk + 1) * kGmNk; ++k) st->h[k] = 0.0;
    if (!st->active) {
      st->status = SFR_MAXIT;
      st->iters = 1;
      cudaGraphSetConditional(a.hwhile, 0u);
    }
  }
}

// res: t = M (b - A x), e_0 = ||t||, inv = 1 / e_0 (Iters.c:634-640)
template <typename I>
__global__ void __launch_bounds__(kGmThreads) k_gm_res(const GmArgs a) {
  SFR_SHARED_RED(1);
  GmState *st = a.st;
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
    const double ti = xmul(xsub(a.b[row_], y[0]), a.m[row_]);
    st_vec(a.t + row_, ti);
    acc[0] += ti * ti;
  }
  if (!last_block<1>(acc, a.part, a.counter, sm)) return;
  if (threadIdx.x == 0) {
    const double e0 = xsqrt(sm[0]);
    st->e[0] = e0;
    st->inv = xdiv(1.0, e0);
  }
}

// spmv of step ni: g_ni = inv src for this warp's rows, w = M A g_ni with
// the gathers scaled the same way, (w, g_0) -> H(0, ni)  (Iters.c:644-655)
template <typename I>
__global__ void __launch_bounds__(kGmThreads) k_gm_spmv(const GmArgs a, int ni) {
  SFR_SHARED_RED(1);
  GmState *st = a.st;
  const int n = a.n;
  const int lane = threadIdx.x & 31;
  int s0, s1;
  block_slices(a.nslices, &s0, &s1);
  const int all[1] = {1};
  const double *const diag[1] = {a.ad};
  const double *src = ni == 0 ? a.t : a.w[(ni - 1) & 1];
  double *gk = a.g[ni];
  const double *g0 = a.g[0];
  double *w = a.w[ni & 1];
  const double inv = st->inv;
  double acc[1] = {0.0};
  SFR_FOR_OWN_ROWS(s0, s1) {
    double y[1];
    row_product<1, true, double>(a.sptr, cols_of<I>(a.cols), a.val, diag, s_, lane, all,
                                 [&](int, int c) { return xmul(ld_ro(src + c), inv); }, y);
    const double gi = xmul(ld_ro(src + row_), inv);
    st_vec(gk + row_, gi);
    const double wi = xmul(y[0], a.m[row_]);
    st_vec(w + row_, wi);
    acc[0] += wi * (ni == 0 ? gi : ld_ro(g0 + row_));
  }
  if (!last_block<1>(acc, a.part, a.counter, sm)) return;
  if (threadIdx.x == 0) H(st, 0, ni) = sm[0];
}

// mgs jj of step ni: w -= H(jj-1, ni) g_(jj-1), (w, g_jj) -> H(jj, ni)
// (Iters.c:656-663, one modified Gram-Schmidt step and the next one's dot)
__global__ void __launch_bounds__(kGmThreads) k_gm_mgs(const GmArgs a, int ni, int jj) {
  SFR_SHARED_RED(1);
  GmState *st = a.st;
  double *w = a.w[ni & 1];
  const double *gp = a.g[jj - 1], *gj = a.g[jj];
  const double beta = H(st, jj - 1, ni);
  double acc[1] = {0.0};
  SFR_GM_FOR_ROWS(i) {
    const double wi = xsub(w[i], xmul(beta, ld_ro(gp + i)));
    w[i] = wi;
    acc[0] += wi * ld_ro(gj + i);
  }
  if (!last_block<1>(acc, a.part, a.counter, sm)) return;
  if (threadIdx.x == 0) H(st, jj, ni) = sm[0];
}

// last of step ni: w -= H(ni, ni) g_ni, H(ni+1, ni) = ||w||, inv, and the
// Givens rotations of column ni (Iters.c:664-690)
__global__ void __launch_bounds__(kGmThreads) k_gm_last(const GmArgs a, int ni) {
  SFR_SHARED_RED(1);
  GmState *st = a.st;
  double *w = a.w[ni & 1];
  const double *gn = a.g[ni];
  const double beta = H(st, ni, ni);
  double acc[1] = {0.0};
  SFR_GM_FOR_ROWS(i) {
    const double wi = xsub(w[i], xmul(beta, ld_ro(gn + i)));
    w[i] = wi;
    acc[0] += wi * wi;
  }
  if (!last_block<1>(acc, a.part, a.counter, sm)) return;
  if (threadIdx.x == 0) {
    const double norm = xsqrt(sm[0]);
    H(st, ni + 1, ni) = norm;
    st->inv = xdiv(1.0, norm);
    for (int j = 0; j < ni; ++j) {
      const double h1 = H(st, j, ni), h2 = H(st, j + 1, ni);
      const double aux1 = xadd(xmul(st->c[j], h1), xmul(st->s[j], h2));
      const double aux2 = xadd(xmul(-st->s[j], h1), xmul(st->c[j], h2));
      H(st, j, ni) = aux1;
      H(st, j + 1, ni) = aux2;
    }
    const double h1 = H(st, ni, ni), h2 = H(st, ni + 1, ni);
    const double r = xsqrt(xadd(xmul(h1, h1), xmul(h2, h2)));
    const double tmp = xdiv(1.0, r);
    st->c[ni] = xmul(h1, tmp);
    st->s[ni] = xmul(h2, tmp);
    H(st, ni, ni) = r;
    H(st, ni + 1, ni) = 0.0;
    st->e[ni + 1] = xmul(-st->s[ni], st->e[ni]);
    st->e[ni] = xmul(st->c[ni], st->e[ni]);
    st->nit += 1;
  }
}

// y: the back substitution and the restart test (Iters.c:692-712)
__global__ void k_gm_y(const GmArgs a) {
  GmState *st = a.st;
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const int ni = kGmNk - 1;  // the cycle ran all nk steps
  double *y = st->y;
  y[ni] = xdiv(st->e[ni], H(st, ni, ni));
  for (int i = ni - 1; i >= 0; --i) {
    double yi = 0.0;
    for (int j = i + 1; j < ni; ++j) yi = xsub(yi, xmul(H(st, i, j), y[j]));
    y[i] = xdiv(xadd(yi, st->e[i]), H(st, i, i));
  }
  bool finite = true;
  for (int k = 0; k <= ni; ++k) finite = finite && isfinite(y[k]);
  const unsigned l = st->l + 1;
  st->l = l;
  bool stop = false;
  if (!finite) {
    st->broke = 1;
    st->status = SFR_BREAKDOWN;
    stop = true;
  } else if (fabs(st->e[ni + 1]) < st->conv) {
    stop = true;
  } else if (l >= st->maxit) {
    st->status = SFR_MAXIT;
    stop = true;
  }
  if (stop) {
    st->active = 0;
    st->iters = st->nit + 1;
    cudaGraphSetConditional(a.hwhile, 0u);
  }
}

// x: x += sum_(k < nk-1) g_k y_k  (Iters.c:713-719), after a finite y
__global__ void __launch_bounds__(kGmThreads) k_gm_x(const GmArgs a) {
  const GmState *st = a.st;
  if (st->broke) return;
  double y[kGmNk - 1];
#pragma unroll
  for (int k = 0; k < kGmNk - 1; ++k) y[k] = st->y[k];
  SFR_GM_FOR_ROWS(i) {
    double xi = a.x[i];
#pragma unroll
    for (int k = 0; k < kGmNk - 1; ++k) xi = xadd(xi, xmul(ld_ro(a.g[k] + i), y[k]));
    a.x[i] = xi;
  }
}

// post-processing: xKx, ||x||, ||b - A x|| (Iters.c:746-760)
template <typename I>
__global__ void __launch_bounds__(kGmThreads) k_gm_post(const GmArgs a) {
  SFR_SHARED_RED(3);
  GmState *st = a.st;
  const int n = a.n;
  const int lane = threadIdx.x & 31;
  int s0, s1;
  block_slices(a.nslices, &s0, &s1);
  const int all[1] = {1};
  const double *const diag[1] = {a.ad};
  double acc[3] = {0.0, 0.0, 0.0};
  SFR_FOR_OWN_ROWS(s0, s1) {
    double y[1];
    row_product<1, true, double>(a.sptr, cols_of<I>(a.cols), a.val, diag, s_, lane, all,
                                 [&](int, int c) { return ld_ro(a.x + c); }, y);
    const double xi = a.x[row_];
    const double ri = xsub(a.b[row_], y[0]);
    acc[0] += xi * y[0];
    acc[1] += xi * xi;
    acc[2] += ri * ri;
  }
  if (!last_block<3>(acc, a.part, a.counter, sm)) return;
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

struct GmGraph {
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  void *ws = nullptr;
  GmArgs args{};
  int gs = 0, gv = 0;
};

std::map<const sfr_system *, std::unique_ptr<GmGraph>> g_gm;

void free_gm(GmGraph *g) {
  if (g->exec) cudaGraphExecDestroy(g->exec);
  if (g->graph) cudaGraphDestroy(g->graph);
  cudaFree(g->ws);
  *g = GmGraph{};
}

cudaError_t node(cudaGraph_t g, cudaGraphNode_t *prev, void *func, int grid, int threads,
                 void **params) {
  cudaKernelNodeParams p{};
  p.func = func;
  p.gridDim = dim3(grid);
  p.blockDim = dim3(threads);
  p.kernelParams = params;
  cudaGraphNode_t nd;
  const cudaError_t e = cudaGraphAddKernelNode(&nd, g, *prev ? prev : nullptr, *prev ? 1 : 0, &p);
  if (e == cudaSuccess) *prev = nd;
  return e;
}

template <typename I>
cudaError_t build(sfr_system *s, GmGraph *g) {
  const int n = s->n;
  const size_t vb = (sizeof(double) * static_cast<size_t>(std::max(n, 1)) + 255) & ~size_t{255};
  int occ = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_gm_spmv<I>, kGmThreads, 0) !=
          cudaSuccess ||
      occ < 1)
    occ = 1;
  const int sms = std::max(1, num_sms(s->device));
  g->gs = std::max(1, std::min((s->A.nslices + 7) / 8, occ * sms));
  g->gv = std::max(1, std::min(sms * (2048 / kGmThreads), (n + kGmThreads - 1) / kGmThreads));
  const int gmax = std::max(g->gs, g->gv);
  constexpr int kVecs = 4 + (kGmNk + 1) + 2 + 1;  // ad, b, x, m; g; w; t
  const size_t part_b = (sizeof(double) * 3 * static_cast<size_t>(gmax) + 255) & ~size_t{255};
  const size_t total = vb * kVecs + part_b + 256 + sizeof(GmState);
  SFR_TRY(cudaMalloc(&g->ws, total));
  SFR_TRY(cudaMemset(g->ws, 0, total));
  char *base = static_cast<char *>(g->ws);
  auto V = [&](int i) { return reinterpret_cast<double *>(base + vb * i); };
  GmArgs &a = g->args;
  a.n = n;
  a.nslices = s->A.nslices;
  a.sptr = s->A.sptr;
  a.cols = SlotCols{s->A.col, s->A.off};
  a.val = s->A.val;
  a.ad = V(0);
  a.b = V(1);
  a.x = V(2);
  a.m = V(3);
  for (int k = 0; k <= kGmNk; ++k) a.g[k] = V(4 + k);
  a.w[0] = V(5 + kGmNk);
  a.w[1] = V(6 + kGmNk);
  a.t = V(7 + kGmNk);
  a.part = reinterpret_cast<double *>(base + vb * kVecs);
  a.counter = reinterpret_cast<unsigned *>(base + vb * kVecs + part_b);
  a.st = reinterpret_cast<GmState *>(base + vb * kVecs + part_b + 256);

  SFR_TRY(cudaGraphCreate(&g->graph, 0));
  SFR_TRY(cudaGraphConditionalHandleCreate(&a.hwhile, g->graph, 1, cudaGraphCondAssignDefault));
  cudaGraphNode_t prev = nullptr;
  {
    cudaMemsetParams mp{};
    mp.dst = a.counter;
    mp.value = 0;
    mp.elementSize = sizeof(unsigned);
    mp.width = kGmCounters;
    mp.height = 1;
    SFR_TRY(cudaGraphAddMemsetNode(&prev, g->graph, nullptr, 0, &mp));
  }
  void *p1[1] = {&a};
  SFR_TRY(node(g->graph, &prev, (void *)k_gm_setup, g->gv, kGmThreads, p1));
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
  SFR_TRY(node(body, &bp, (void *)k_gm_res<I>, g->gs, kGmThreads, p1));
  for (int ni = 0; ni < kGmNk; ++ni) {
    int vni = ni;  // copied into the node's parameters when it is added
    void *p2[2] = {&a, &vni};
    SFR_TRY(node(body, &bp, (void *)k_gm_spmv<I>, g->gs, kGmThreads, p2));
    for (int jj = 1; jj <= ni; ++jj) {
      int vjj = jj;
      void *p3[3] = {&a, &vni, &vjj};
      SFR_TRY(node(body, &bp, (void *)k_gm_mgs, g->gv, kGmThreads, p3));
    }
    SFR_TRY(node(body, &bp, (void *)k_gm_last, g->gv, kGmThreads, p2));
  }
  SFR_TRY(node(body, &bp, (void *)k_gm_y, 1, 32, p1));
  SFR_TRY(node(body, &bp, (void *)k_gm_x, g->gv, kGmThreads, p1));
  SFR_TRY(node(g->graph, &prev, (void *)k_gm_post<I>, g->gs, kGmThreads, p1));
  SFR_TRY(cudaGraphInstantiate(&g->exec, g->graph, 0));
  return cudaSuccess;
}

}  // namespace

int solve_gmres_graph(sfr_system *s, const double *d_diag, const double *d_b, double *d_x,
                      double tol, uint32_t maxit, int32_t newx, cudaStream_t st,
                      sfr_solve_info *info) {
  auto &slot = g_gm[s];
  if (!slot) {
    slot = std::make_unique<GmGraph>();
    const cudaError_t be = s->A.off ? build<int16_t>(s, slot.get()) : build<int>(s, slot.get());
    if (be != cudaSuccess) {
      set_last_error(cudaGetErrorString(be));
      free_gm(slot.get());
      g_gm.erase(s);
      return SFR_CUDA_ERROR;
    }
  }
  GmGraph *g = slot.get();
  const GmArgs &a = g->args;
  const size_t vb = sizeof(double) * static_cast<size_t>(s->n);
  GmState call{};
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
    err = cudaMemcpyAsync(a.st, &call, offsetof(GmState, conv), cudaMemcpyHostToDevice, st);
  if (err == cudaSuccess) err = cudaGraphLaunch(g->exec, st);
  if (err == cudaSuccess) err = cudaMemcpyAsync(d_x, a.x, vb, cudaMemcpyDeviceToDevice, st);
  if (err == cudaSuccess) err = cudaEventRecord(e1, st);
  GmState out{};
  if (err == cudaSuccess)
    err = cudaMemcpyAsync(&out, a.st, sizeof(GmState), cudaMemcpyDeviceToHost, st);
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

void release_gmres_graph(const sfr_system *s) {
  auto it = g_gm.find(s);
  if (it == g_gm.end()) return;
  free_gm(it->second.get());
  g_gm.erase(it);
}

}  // namespace sfr
