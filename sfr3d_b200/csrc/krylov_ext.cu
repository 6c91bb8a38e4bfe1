// The other Krylov methods behind the reference's solverC (Solv.c:217-440):
// BiCGSTAB(2) (Bicgstab.c:1172-1460), restarted GMRES(15) (Iters.c:587-800)
// and MINRES (Iters.c:309-558), all with the Jacobi preconditioner, FP64.
//
// With engine 3 the three run as host loops over device work (otherwise
// each is one CUDA graph: minres_graph.cu, bicgl2_graph.cu,
// gmres_graph.cu): the SpMV with the reference's row rounding
// (spmv_kernel), deterministic dot products (fixed block
// partition, fixed reduction tree), and element-wise updates that round in
// the order of the reference's expressions (no FMA contraction).  The scalar
// recurrences -- MINRES's Givens rotations (symOrtho), the GCR(2) part of
// BiCGSTAB(2), GMRES's rotations and back substitution -- run on the host in
// double precision, as in the reference, from dot products read back.
// GMRES keeps its Gram-Schmidt coefficients on the device for a whole
// restart cycle, so a cycle costs one host round trip plus one per restart
// norm.  The reference's quirks are kept: GMRES always runs the full cycle
// and updates x with its first nk-1 directions; symOrtho tests |b| against
// a, not |a|.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "internal.h"
#include "persist.cuh"

namespace sfr {

namespace {

constexpr int kExtThreads = 256;
constexpr int kGmresRestart = 15;  // solverC's nKrylov (Solv.c:82)
constexpr int kExtMaxDots = 8;

template <typename F>
__global__ void __launch_bounds__(kExtThreads) each_kernel(int n, F f) {
  const int stride = gridDim.x * blockDim.x;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) f(i);
}

template <int NV>
struct DotPairs {
  const double *a[NV];
  const double *b[NV];
};

// NV dot products (a_v, b_v) in one pass; the last block to finish sums the
// block partials in block order into out[0..NV) and resets the counter.
template <int NV>
__global__ void __launch_bounds__(kExtThreads) mdot_kernel(DotPairs<NV> d, int n, double *part,
                                                           unsigned *counter, double *out) {
  __shared__ double sm[(NV + 1) * 32];
  __shared__ bool s_last;
  double acc[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) acc[v] = 0.0;
  const int stride = gridDim.x * blockDim.x;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
#pragma unroll
    for (int v = 0; v < NV; ++v) acc[v] += d.a[v][i] * d.b[v][i];
  }
  block_partials<NV>(acc, part, gridDim.x, sm);
  if (threadIdx.x == 0) {
    __threadfence();
    s_last = atomicAdd(counter, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  double tot[NV];
  grid_totals<NV>(part, gridDim.x, gridDim.x, tot, sm);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int v = 0; v < NV; ++v) out[v] = tot[v];
    *counter = 0u;
  }
}

// One solve's device context: vectors in the system's workspace, reduction
// scratch, and the launch helpers.
struct Ext {
  sfr_system *s;
  cudaStream_t st;
  int n;
  int grid;
  const double *diag;
  double *part;       // block partials, kExtMaxDots * grid
  unsigned *counter;
  double *dout;       // device results of reductions
  std::vector<double *> vec;
  cudaError_t err = cudaSuccess;

  template <typename F>
  void each(F f) {
    if (err != cudaSuccess) return;
    each_kernel<<<grid, kExtThreads, 0, st>>>(n, f);
    err = cudaGetLastError();
  }
  void spmv(const double *x, double *y) {
    if (err != cudaSuccess) return;
    if (spmv_device(s, s->A, diag, x, y, nullptr, st) != SFR_OK) err = cudaErrorLaunchFailure;
  }
  // NV dot products into device memory at out
  template <int NV>
  void dots_dev(const DotPairs<NV> &d, double *out) {
    if (err != cudaSuccess) return;
    mdot_kernel<NV><<<grid, kExtThreads, 0, st>>>(d, n, part, counter, out);
    err = cudaGetLastError();
  }
  // NV dot products read back to the host
  template <int NV>
  bool dots(const DotPairs<NV> &d, double (&h)[NV]) {
    dots_dev<NV>(d, dout);
    if (err == cudaSuccess) err = cudaMemcpyAsync(h, dout, sizeof(double) * NV,
                                                  cudaMemcpyDeviceToHost, st);
    if (err == cudaSuccess) err = cudaStreamSynchronize(st);
    return err == cudaSuccess;
  }
  double dot(const double *a, const double *b) {
    double h[1] = {0.0};
    dots<1>(DotPairs<1>{{a}, {b}}, h);
    return h[0];
  }
};

// Workspace: nv vectors of n, the reduction scratch and `extra` result words.
int make_ext(sfr_system *s, cudaStream_t st, int nv, int extra, Ext *e) {
  const int n = s->n;
  auto align = [](size_t v) { return (v + 255) & ~static_cast<size_t>(255); };
  const int grid = std::max(1, std::min(4 * std::max(1, num_sms(s->device)),
                                        (n + kExtThreads - 1) / kExtThreads));
  const size_t vb = align(sizeof(double) * static_cast<size_t>(std::max(n, 1)));
  const size_t part_b = align(sizeof(double) * kExtMaxDots * grid);
  const size_t ctl_b = 256;
  const size_t out_b = align(sizeof(double) * (kExtMaxDots + extra));
  int rc = ensure_workspace(s, vb * nv + part_b + ctl_b + out_b);
  if (rc != SFR_OK) return rc;
  char *base = static_cast<char *>(s->ws.base);
  e->s = s;
  e->st = st;
  e->n = n;
  e->grid = grid;
  e->vec.resize(nv);
  for (int i = 0; i < nv; ++i) e->vec[i] = reinterpret_cast<double *>(base + vb * i);
  base += vb * nv;
  e->part = reinterpret_cast<double *>(base);
  e->counter = reinterpret_cast<unsigned *>(base + part_b);
  e->dout = reinterpret_cast<double *>(base + part_b + ctl_b);
  if (cudaMemsetAsync(e->counter, 0, ctl_b, st) != cudaSuccess) return SFR_CUDA_ERROR;
  return SFR_OK;
}

// xKx, ||x||, ||b - Ax|| (and, for MINRES, ||M^1/2 (b - Ax)||) as the
// reference's post-processing computes them.
void post(Ext &e, const double *b, const double *x, const double *m, double *t, double *r,
          bool minres_norm, sfr_solve_info *info) {
  e.spmv(x, t);
  double h[2] = {0.0, 0.0};
  e.dots<2>(DotPairs<2>{{x, x}, {t, x}}, h);
  info->xKx = h[0];
  info->norm_x = std::sqrt(h[1]);
  const double *tc = t;
  if (minres_norm) {
    e.each([=] __device__(int i) {
      const double ri = xsub(b[i], tc[i]);
      r[i] = ri;
      t[i] = xmul(ri, sqrt(fabs(m[i])));
    });
    e.dots<2>(DotPairs<2>{{r, t}, {r, t}}, h);
    info->norm_r = std::sqrt(h[0]);
    info->norm_r_m = std::sqrt(h[1]);
  } else {
    e.each([=] __device__(int i) { r[i] = xsub(b[i], tc[i]); });
    info->norm_r = std::sqrt(e.dot(r, r));
    info->norm_r_m = 0.0;
  }
}

// Iters.c:1171-1211 (symOrtho), branch tests as the reference writes them.
void sym_ortho(double a, double b, double *c, double *s, double *r) {
  const double ma = std::fabs(a), mb = std::fabs(b);
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
    const double t = a / b;
    *s = sb / std::sqrt(1.0 + t * t);
    *c = *s * t;
    *r = b / *s;
  } else if (ma > mb) {
    const double t = b / a;
    *c = sa / std::sqrt(1.0 + t * t);
    *s = *c * t;
    *r = a / *c;
  }
}

// Iters.c:309-558 (pminres).
int run_minres(Ext &e, const double *b, double *x, double tol, uint32_t maxit, int newx,
               sfr_solve_info *info) {
  double *m = e.vec[0], *v0 = e.vec[1], *v = e.vec[2], *w = e.vec[3], *w0 = e.vec[4],
         *w00 = e.vec[5], *z = e.vec[6], *z0 = e.vec[7], *p = e.vec[8];
  const double *ad = e.diag;
  e.each([=] __device__(int i) {
    const double mi = 1.0 / ad[i];
    m[i] = mi;
    if (newx) x[i] = 0.0;
    z[i] = xmul(b[i], sqrt(mi));
  });
  const double conv = tol * std::sqrt(e.dot(z, z));
  e.spmv(x, z);
  e.each([=] __device__(int i) {
    const double vi = xsub(b[i], z[i]);
    v[i] = vi;
    v0[i] = w0[i] = w00[i] = 0.0;
    z0[i] = xmul(vi, m[i]);
  });
  double beta = std::sqrt(std::fabs(e.dot(v, z0)));
  double norm_r = beta, neta = beta, beta_old = beta;
  double c_old = 1.0, c = 1.0, s_old = 0.0, s = 0.0, ro1 = 1.0;
  int status = SFR_OK;
  uint32_t j = 0;
  for (; j < maxit && e.err == cudaSuccess; ++j) {
    e.spmv(z0, p);
    double t1 = 1.0 / (beta * beta);
    const double alpha = e.dot(z0, p) * t1;
    t1 = 1.0 / beta;
    const double t2 = -alpha / beta, t3 = -beta / beta_old;
    {
      const double *vc = v, *v0c = v0;
      double *pc = p, *zc = z;
      e.each([=] __device__(int i) {
        const double pi = xadd(xadd(xmul(t1, pc[i]), xmul(t2, vc[i])), xmul(t3, v0c[i]));
        pc[i] = pi;
        zc[i] = xmul(pi, m[i]);
      });
    }
    beta_old = beta;
    beta = std::sqrt(e.dot(z, p));
    const double delta = c * alpha - c_old * s * beta_old;
    const double ro2 = s * alpha + c_old * c * beta_old;
    const double ro3 = s_old * beta_old;
    c_old = c;
    s_old = s;
    sym_ortho(delta, beta, &c, &s, &ro1);
    const double u1 = 1.0 / (beta_old * ro1), u2 = -ro2 / ro1, u3 = -ro3 / ro1, u4 = c * neta;
    if (!std::isfinite(u1) || !std::isfinite(u2) || !std::isfinite(u3) || !std::isfinite(u4)) {
      status = SFR_BREAKDOWN;
      ++j;
      break;
    }
    {
      const double *z0c = z0, *w0c = w0, *w00c = w00;
      double *wc = w;
      e.each([=] __device__(int i) {
        const double wi = xadd(xadd(xmul(u1, z0c[i]), xmul(u2, w0c[i])), xmul(u3, w00c[i]));
        wc[i] = wi;
        x[i] = xadd(x[i], xmul(u4, wi));
      });
    }
    // v0 <- v, v <- p, z0 <- z, w00 <- w0, w0 <- w: by rotation
    double *tmp = v0;
    v0 = v;
    v = p;
    p = tmp;
    tmp = z0;
    z0 = z;
    z = tmp;
    tmp = w00;
    w00 = w0;
    w0 = w;
    w = tmp;
    norm_r = std::fabs(s) * norm_r;
    if (norm_r < conv) break;
    neta = -s * neta;
  }
  if (status == SFR_OK && j == maxit) status = SFR_MAXIT;
  post(e, b, x, m, z, v, true, info);
  info->iters = static_cast<int>(std::min<uint32_t>(j, maxit)) + 1;
  info->conv = conv;
  return status;
}

// Bicgstab.c:1172-1460 (pbicgstabl2).
int run_bicgstabl2(Ext &e, const double *b, double *x, double tol, uint32_t maxit, int newx,
                   sfr_solve_info *info) {
  double *m = e.vec[0], *t = e.vec[1], *v = e.vec[2], *r = e.vec[3], *u = e.vec[4],
         *r0 = e.vec[5], *w = e.vec[6], *s = e.vec[7], *p = e.vec[8], *h = e.vec[9],
         *z = e.vec[10];
  const double *ad = e.diag;
  e.each([=] __device__(int i) {
    m[i] = 1.0 / ad[i];
    if (newx) x[i] = 0.0;
  });
  const double conv = tol * std::sqrt(e.dot(b, b));
  e.spmv(x, t);
  e.each([=] __device__(int i) {
    const double ri = xsub(b[i], t[i]);
    r0[i] = ri;
    r[i] = ri;
    u[i] = 0.0;
  });
  double rr0 = 1.0, alpha = 0.0, omega2 = 1.0;
  int status = SFR_OK;
  uint32_t j = 0;
  for (; j < maxit && e.err == cudaSuccess; ++j) {
    rr0 = -omega2 * rr0;
    // even BiCG step
    double rr1 = e.dot(r, r0);
    double beta = alpha * rr1 / rr0;
    rr0 = rr1;
    e.each([=] __device__(int i) {
      const double ui = xsub(r[i], xmul(beta, u[i]));
      u[i] = ui;
      z[i] = xmul(ui, m[i]);
    });
    e.spmv(z, v);
    alpha = rr0 / e.dot(v, r0);
    {
      const double a = alpha;
      e.each([=] __device__(int i) {
        const double ri = xsub(r[i], xmul(a, v[i]));
        r[i] = ri;
        p[i] = xmul(ri, m[i]);
      });
    }
    e.spmv(p, s);
    {
      const double a = alpha;
      e.each([=] __device__(int i) { x[i] = xadd(x[i], xmul(a, z[i])); });
    }
    // odd BiCG step
    rr1 = e.dot(s, r0);
    beta = alpha * rr1 / rr0;
    rr0 = rr1;
    e.each([=] __device__(int i) {
      const double vi = xsub(s[i], xmul(beta, v[i]));
      v[i] = vi;
      p[i] = xmul(vi, m[i]);
    });
    e.spmv(p, w);
    alpha = rr0 / e.dot(w, r0);
    {
      const double a = alpha, bt = beta;
      e.each([=] __device__(int i) {
        const double ui = xsub(r[i], xmul(bt, u[i]));
        const double ri = xsub(r[i], xmul(a, v[i]));
        const double si = xsub(s[i], xmul(a, w[i]));
        u[i] = ui;
        r[i] = ri;
        s[i] = si;
        p[i] = xmul(si, m[i]);
        z[i] = xmul(ui, m[i]);
        h[i] = xmul(ri, m[i]);
      });
    }
    e.spmv(p, t);
    // GCR(2) part
    double g5[5] = {0, 0, 0, 0, 0};
    e.dots<5>(DotPairs<5>{{r, s, s, t, r}, {s, s, t, t, t}}, g5);
    double omega1 = g5[0];
    const double mi = g5[1], ni = g5[2];
    double tau = g5[3];
    omega2 = g5[4];
    tau = tau - ni * ni / mi;
    omega2 = (omega2 - ni * omega1 / mi) / tau;
    omega1 = (omega1 - ni * omega2) / mi;
    if (!std::isfinite(omega1) || !std::isfinite(omega2) || !std::isfinite(alpha)) {
      status = SFR_BREAKDOWN;
      ++j;
      break;
    }
    {
      const double o1 = omega1, o2 = omega2, a = alpha;
      e.each([=] __device__(int i) {
        x[i] = xadd(x[i], xadd(xadd(xmul(o1, h[i]), xmul(o2, p[i])), xmul(a, z[i])));
        r[i] = xsub(r[i], xadd(xmul(o1, s[i]), xmul(o2, t[i])));
      });
    }
    const double d = e.dot(r, r);
    if (std::sqrt(d) < conv) break;
    {
      const double o1 = omega1, o2 = omega2;
      e.each([=] __device__(int i) { u[i] = xsub(u[i], xadd(xmul(o1, v[i]), xmul(o2, w[i]))); });
    }
  }
  if (status == SFR_OK && j == maxit) status = SFR_MAXIT;
  post(e, b, x, m, z, r, false, info);
  info->iters = static_cast<int>(std::min<uint32_t>(j, maxit)) + 1;
  info->conv = conv;
  return status;
}

// The Krylov basis of a GMRES cycle, passed by value to the update kernel.
struct GmresBasis {
  double *v[kGmresRestart];
};

// Iters.c:587-800 (gmres) with nk = 15 Krylov vectors a cycle; maxit counts
// cycles.
int run_gmres(Ext &e, const double *b, double *x, double tol, uint32_t maxit, int newx,
              sfr_solve_info *info) {
  constexpr int nk = kGmresRestart;
  double *m = e.vec[0];
  double *g[nk + 1];
  for (int k = 0; k <= nk; ++k) g[k] = e.vec[1 + k];
  double *t = e.vec[nk + 2];
  double *dh = e.dout + kExtMaxDots;        // Gram-Schmidt coefficients, (nk+1) x nk
  double *dn = dh + (nk + 1) * nk;          // (g2, g2) of each Arnoldi step
  double *dy = dn + nk;                     // the cycle's update coefficients
  std::vector<double> hh((nk + 1) * nk, 0.0), hn(nk, 0.0), y(nk, 0.0), c(nk, 0.0),
      sn(nk, 0.0), ev(nk + 1, 0.0);
  auto H = [&](int row, int col) -> double & { return hh[row * nk + col]; };
  const double *ad = e.diag;
  double *g0 = g[0];
  e.each([=] __device__(int i) {
    const double mi = 1.0 / ad[i];
    m[i] = mi;
    if (newx) x[i] = 0.0;
    g0[i] = xmul(b[i], mi);
  });
  const double eConv = tol * std::sqrt(e.dot(g0, g0));
  int status = SFR_OK, nIt = 0, ni = 0;
  uint32_t l = 0;
  for (; l < maxit && e.err == cudaSuccess; ++l) {
    e.spmv(x, g0);
    e.each([=] __device__(int i) { g0[i] = xmul(xsub(b[i], g0[i]), m[i]); });
    ev[0] = std::sqrt(e.dot(g0, g0));
    {
      const double tmp = 1.0 / ev[0];
      e.each([=] __device__(int i) { g0[i] = xmul(g0[i], tmp); });
    }
    for (ni = 0; ni < nk; ++ni, ++nIt) {
      double *g1 = g[ni], *g2 = g[ni + 1];
      e.spmv(g1, g2);
      e.each([=] __device__(int i) { g2[i] = xmul(g2[i], m[i]); });
      for (int jj = 0; jj <= ni; ++jj) {  // modified Gram-Schmidt
        const double *gj = g[jj];
        double *hp = dh + jj * nk + ni;
        e.dots_dev<1>(DotPairs<1>{{g2}, {gj}}, hp);
        e.each([=] __device__(int i) { g2[i] = xsub(g2[i], xmul(*hp, gj[i])); });
      }
      double *np = dn + ni;
      e.dots_dev<1>(DotPairs<1>{{g2}, {g2}}, np);
      e.each([=] __device__(int i) { g2[i] = xmul(g2[i], 1.0 / sqrt(*np)); });
    }
    // the cycle's coefficients: rotations and back substitution on the host
    if (e.err == cudaSuccess)
      e.err = cudaMemcpyAsync(hh.data(), dh, sizeof(double) * hh.size(), cudaMemcpyDeviceToHost,
                              e.st);
    if (e.err == cudaSuccess)
      e.err = cudaMemcpyAsync(hn.data(), dn, sizeof(double) * nk, cudaMemcpyDeviceToHost, e.st);
    if (e.err == cudaSuccess) e.err = cudaStreamSynchronize(e.st);
    if (e.err != cudaSuccess) break;
    for (int k = 0; k < nk; ++k) {
      H(k + 1, k) = std::sqrt(hn[k]);
      for (int jj = 0; jj < k; ++jj) {
        const double h1 = H(jj, k), h2 = H(jj + 1, k);
        const double aux1 = c[jj] * h1 + sn[jj] * h2;
        const double aux2 = -sn[jj] * h1 + c[jj] * h2;
        H(jj, k) = aux1;
        H(jj + 1, k) = aux2;
      }
      const double h1 = H(k, k), h2 = H(k + 1, k);
      const double r = std::sqrt(h1 * h1 + h2 * h2);
      const double tmp = 1.0 / r;
      c[k] = h1 * tmp;
      sn[k] = h2 * tmp;
      H(k, k) = r;
      H(k + 1, k) = 0.0;
      ev[k + 1] = -sn[k] * ev[k];
      ev[k] = c[k] * ev[k];
    }
    if (ni == nk) ni--;
    y[ni] = ev[ni] / H(ni, ni);
    for (int i = ni - 1; i >= 0; i--) {
      y[i] = 0.0;
      for (int jj = i + 1; jj < ni; jj++) y[i] -= H(i, jj) * y[jj];
      y[i] = (y[i] + ev[i]) / H(i, i);
    }
    bool finite = true;
    for (int k = 0; k <= ni; ++k) finite = finite && std::isfinite(y[k]);
    if (!finite) {
      status = SFR_BREAKDOWN;
      ++l;
      break;
    }
    e.err = cudaMemcpyAsync(dy, y.data(), sizeof(double) * nk, cudaMemcpyHostToDevice, e.st);
    {
      const int nu = ni;
      GmresBasis basis;
      for (int k = 0; k < nk; ++k) basis.v[k] = g[k];
      e.each([=] __device__(int i) {
        double xi = x[i];
        for (int k = 0; k < nu; ++k) xi = xadd(xi, xmul(basis.v[k][i], dy[k]));
        x[i] = xi;
      });
    }
    if (std::fabs(ev[ni + 1]) < eConv) break;
  }
  if (status == SFR_OK && l == maxit) status = SFR_MAXIT;
  post(e, b, x, m, t, g[1], false, info);
  info->iters = nIt + 1;
  info->conv = eConv;
  return status;
}

}  // namespace

int solve_ext(sfr_system *s, int32_t solver, const double *d_diag, const double *d_b, double *d_x,
              double tol, uint32_t maxit, int32_t newx, cudaStream_t st, sfr_solve_info *info) {
  if (maxit == 0) return SFR_BAD_INPUT;
  // MINRES, BiCGSTAB(2) and GMRES run as one CUDA graph with their
  // recurrences on the device (minres_graph.cu, bicgl2_graph.cu,
  // gmres_graph.cu); engine 3 keeps the host loops below, for profilers
  if (solver == SFR_MINRES && s->engine != 3)
    return solve_minres_graph(s, d_diag, d_b, d_x, tol, maxit, newx, st, info);
  if (solver == SFR_PBICGSTABL2 && s->engine != 3)
    return solve_bicgstabl2_graph(s, d_diag, d_b, d_x, tol, maxit, newx, st, info);
  if (solver == SFR_GMRES && s->engine != 3)
    return solve_gmres_graph(s, d_diag, d_b, d_x, tol, maxit, newx, st, info);
  int nv = 0, extra = 0;
  switch (solver) {
    case SFR_MINRES: nv = 9; break;
    case SFR_PBICGSTABL2: nv = 11; break;
    case SFR_GMRES:
      nv = kGmresRestart + 3;
      extra = (kGmresRestart + 1) * kGmresRestart + 2 * kGmresRestart;
      break;
    default: return SFR_UNSUPPORTED;
  }
  Ext e;
  int rc = make_ext(s, st, nv, extra, &e);
  if (rc != SFR_OK) return rc;
  e.diag = d_diag ? d_diag : s->d_diag;
  cudaEvent_t e0, e1;
  if (cudaEventCreate(&e0) != cudaSuccess) return SFR_CUDA_ERROR;
  if (cudaEventCreate(&e1) != cudaSuccess) {
    cudaEventDestroy(e0);
    return SFR_CUDA_ERROR;
  }
  sfr_solve_info out;
  std::memset(&out, 0, sizeof(out));
  cudaEventRecord(e0, st);
  int status = SFR_OK;
  if (solver == SFR_MINRES)
    status = run_minres(e, d_b, d_x, tol, maxit, newx, &out);
  else if (solver == SFR_PBICGSTABL2)
    status = run_bicgstabl2(e, d_b, d_x, tol, maxit, newx, &out);
  else
    status = run_gmres(e, d_b, d_x, tol, maxit, newx, &out);
  cudaEventRecord(e1, st);
  cudaError_t ce = e.err;
  if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
  float ms = 0.f;
  if (ce == cudaSuccess) cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (ce != cudaSuccess) {
    set_last_error(cudaGetErrorString(ce));
    return SFR_CUDA_ERROR;
  }
  if (info) {
    *info = out;
    info->status = status;
    info->seconds = ms * 1e-3;
    info->refinements = 0;
    info->inner_iters = out.iters;
    info->relres = std::nan("");
  }
  return status;
}

}  // namespace sfr
