/*
 * Test infrastructure, not product code: plain-C restatement of SFR3D's
 * Jacobi-PCG / Jacobi-BiCGSTAB path (the parity oracle).  Compiled with
 * -ffp-contract=off so every product and sum rounds exactly where the
 * reference's (gcc -std=c99 -O3, no FMA) does.
 */
#include "sfr3d_oracle.h"

#include <math.h>
#include <stdlib.h>

/* Summation order of orc_dot: 0 is the reference's; 1 (right to left) and
 * 2 (pairwise over blocks of 64) exist only to measure how far the
 * reference's own algorithms move when nothing but the order of a sum
 * changes. */
static int g_dot_order = 0;

void orc_set_dot_order(int order) { g_dot_order = order; }

static double dot_pairwise(const double *a, const double *b, int n)
{
  if (n <= 64) {
    double s = 0.0;
    for (int i = 0; i < n; i++) s += a[i] * b[i];
    return s;
  }
  const int h = n / 2;
  return dot_pairwise(a, b, h) + dot_pairwise(a + h, b + h, n - h);
}

/* HccaBlas.c:393-437 (dot): one accumulator, left to right. */
double orc_dot(const double *a, const double *b, int n)
{
  double s = 0.0;
  if (g_dot_order == 1) {
    for (int i = n - 1; i >= 0; i--) s += a[i] * b[i];
    return s;
  }
  if (g_dot_order == 2) return dot_pairwise(a, b, n);
  for (int i = 0; i < n; i++) s += a[i] * b[i];
  return s;
}

/* HccaBlas.c:3358-3400 (matVecCsrD): full off-diagonal rows, diagonal first. */
static void mv_csrd(int neq, const int *ia, const int *ja, const double *a,
                    const double *ad, const double *x, double *y)
{
  for (int i = 0; i < neq; i++) {
    double t = ad[i] * x[i];
    for (int k = ia[i]; k < ia[i + 1]; k++) t += a[k] * x[ja[k]];
    y[i] = t;
  }
}

/* HccaBlas.c:2620-2655 (matVecCsrDSym) when au == al, and HccaBlas.c:4223-4258
 * (matVecCsrC) with au = a + nad: strict-lower rows plus the mirrored
 * scatter into y[ja[k]] in row order. */
static void mv_lower(int neq, const int *ia, const int *ja, const double *al,
                     const double *au, const double *ad, const double *x,
                     double *y)
{
  if (neq <= 0) return;
  y[0] = ad[0] * x[0];
  for (int i = 1; i < neq; i++) {
    const double xi = x[i];
    double t = ad[i] * xi;
    for (int k = ia[i]; k < ia[i + 1]; k++) {
      const int j = ja[k];
      t += al[k] * x[j];
      y[j] += au[k] * xi;
    }
    y[i] = t;
  }
}

/* HccaBlas.c:4700-4755 (matVecEllPack), for any width: diagonal, then the
 * slots in order.  The reference unrolls widths 6, 4 and 3 only; the sum
 * order is the same. */
static void mv_ell(int neq, int width, const int *ja, const double *a,
                   const double *ad, const double *x, double *y)
{
  for (int i = 0; i < neq; i++) {
    double t = ad[i] * x[i];
    for (int k = 0; k < width; k++)
      t += a[(long)i * width + k] * x[ja[(long)i * width + k]];
    y[i] = t;
  }
}

/* setMatVec, Solv.c:732-919 (serial branches). */
void orc_matvec(int storage, int unsym, int neq, const int *ia, const int *ja,
                const double *al, const double *ad, const double *x, double *y)
{
  if (storage == ORC_ELLPACK) {
    mv_ell(neq, ia[0], ja, al, ad, x, y);
  } else if (storage == ORC_CSRD && unsym) {
    mv_csrd(neq, ia, ja, al, ad, x, y);
  } else if (storage == ORC_CSRC && unsym) {
    const int nad = ia[neq] - ia[0];
    mv_lower(neq, ia, ja, al, al + nad, ad, x, y);
  } else {
    mv_lower(neq, ia, ja, al, al, ad, x, y);
  }
}

/* Cg.c:47-209 (pcg) with the diagonal preconditioner of PreCond.c:18-26. */
int orc_pcg(int storage, int unsym, int neq, const int *ia, const int *ja,
            const double *al, const double *ad, const double *b, double *x,
            double tol, unsigned maxit, int newx, orc_stats *st)
{
  double *m = malloc(sizeof(double) * (size_t)neq * 4);
  double *z = m + neq, *r = z + neq, *p = r + neq;
  double alpha, beta, d, di, conv;
  unsigned j;
  int i;
  if (!m) return -1;
  for (i = 0; i < neq; i++) m[i] = 1.0 / ad[i];
  if (newx)
    for (i = 0; i < neq; i++) x[i] = 0.0;
  for (i = 0; i < neq; i++) z[i] = b[i] * m[i];
  d = orc_dot(b, z, neq);
  conv = tol * sqrt(fabs(d));
  orc_matvec(storage, unsym, neq, ia, ja, al, ad, x, z);
  for (i = 0; i < neq; i++) {
    r[i] = b[i] - z[i];
    z[i] = r[i] * m[i];
    p[i] = z[i];
  }
  d = orc_dot(r, z, neq);
  for (j = 0; j < maxit; j++) {
    orc_matvec(storage, unsym, neq, ia, ja, al, ad, p, z);
    alpha = d / orc_dot(z, p, neq);
    for (i = 0; i < neq; i++) {
      x[i] += alpha * p[i];
      r[i] -= alpha * z[i];
      z[i] = r[i] * m[i];
    }
    di = orc_dot(r, z, neq);
    beta = di / d;
    for (i = 0; i < neq; i++) p[i] = z[i] + beta * p[i];
    d = di;
    if (sqrt(fabs(d)) < conv) break;
  }
  /* post-processing, Cg.c:155-176 */
  orc_matvec(storage, unsym, neq, ia, ja, al, ad, x, z);
  st->xKx = orc_dot(x, z, neq);
  st->norm_x = sqrt(orc_dot(x, x, neq));
  for (i = 0; i < neq; i++) {
    r[i] = b[i] - z[i];
    z[i] = r[i] * m[i];
  }
  st->norm_r_m = sqrt(fabs(orc_dot(r, z, neq)));
  st->norm_r = sqrt(orc_dot(r, r, neq));
  st->conv = conv;
  st->iters = (int)j + 1;
  st->status = j == maxit ? 1 : 0;
  free(m);
  return st->status;
}

/* Bicgstab.c:50-245 (pbicgstab), right-preconditioned. */
int orc_pbicgstab(int storage, int unsym, int neq, const int *ia,
                  const int *ja, const double *al, const double *ad,
                  const double *b, double *x, double tol, unsigned maxit,
                  int newx, orc_stats *st)
{
  double *m = malloc(sizeof(double) * (size_t)neq * 7);
  double *t = m + neq, *v = t + neq, *r = v + neq, *p = r + neq, *z = p + neq,
         *r0 = z + neq;
  double alpha, beta, d, conv, w, rr0;
  unsigned j;
  int i;
  if (!m) return -1;
  for (i = 0; i < neq; i++) m[i] = 1.0 / ad[i];
  if (newx)
    for (i = 0; i < neq; i++) x[i] = 0.0;
  d = orc_dot(b, b, neq);
  conv = tol * sqrt(d);
  orc_matvec(storage, unsym, neq, ia, ja, al, ad, x, z);
  for (i = 0; i < neq; i++) {
    r0[i] = b[i] - z[i];
    p[i] = r0[i];
    r[i] = r0[i];
    z[i] = p[i] * m[i];
  }
  for (j = 0; j < maxit; j++) {
    orc_matvec(storage, unsym, neq, ia, ja, al, ad, z, v);
    rr0 = orc_dot(r, r0, neq);
    alpha = rr0 / orc_dot(v, r0, neq);
    for (i = 0; i < neq; i++) {
      x[i] += alpha * z[i];
      r[i] -= alpha * v[i];
      z[i] = r[i] * m[i];
    }
    d = orc_dot(r, r, neq);
    if (sqrt(d) < conv) break;
    orc_matvec(storage, unsym, neq, ia, ja, al, ad, z, t);
    w = orc_dot(t, r, neq) / orc_dot(t, t, neq);
    for (i = 0; i < neq; i++) {
      x[i] += w * z[i];
      r[i] -= w * t[i];
    }
    d = orc_dot(r, r, neq);
    if (sqrt(d) < conv) break;
    beta = (orc_dot(r, r0, neq) / rr0) * (alpha / w);
    for (i = 0; i < neq; i++) {
      p[i] = r[i] + beta * (p[i] - w * v[i]);
      z[i] = p[i] * m[i];
    }
  }
  /* post-processing, Bicgstab.c:188-204 */
  orc_matvec(storage, unsym, neq, ia, ja, al, ad, x, z);
  st->xKx = orc_dot(x, z, neq);
  st->norm_x = sqrt(orc_dot(x, x, neq));
  for (i = 0; i < neq; i++) r[i] = b[i] - z[i];
  st->norm_r = sqrt(orc_dot(r, r, neq));
  st->norm_r_m = 0.0;
  st->conv = conv;
  st->iters = (int)j + 1;
  st->status = j == maxit ? 1 : 0;
  free(m);
  return st->status;
}

/* Iters.c:1171-1211 (symOrtho): Givens rotation for (a, b), with the
 * reference's branch tests as written (the third compares |b| with a, not
 * |a|; when no branch applies c, s and r keep their values). */
static void orc_sym_ortho(double a, double b, double *c, double *s, double *r)
{
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
    const double t = a / b;
    *s = sb / sqrt(1.0 + t * t);
    *c = *s * t;
    *r = b / *s;
  } else if (ma > mb) {
    const double t = b / a;
    *c = sa / sqrt(1.0 + t * t);
    *s = *c * t;
    *r = a / *c;
  }
}

/* Iters.c:309-558 (pminres): MINRES on the Jacobi-preconditioned system
 * D^-1/2 A D^-1/2, with the Lanczos vectors kept in the unscaled space.
 * The reference only warns when maxIt is reached; status 1 reports it. */
int orc_minres(int storage, int unsym, int neq, const int *ia, const int *ja,
               const double *al, const double *ad, const double *b, double *x,
               double tol, unsigned maxit, int newx, orc_stats *st)
{
  double *m = malloc(sizeof(double) * (size_t)neq * 10);
  double *v0 = m + neq, *v = v0 + neq, *w = v + neq, *w0 = w + neq,
         *w00 = w0 + neq, *z = w00 + neq, *z0 = z + neq, *p = z0 + neq, *tmp;
  double t1, t2, t3, t4, conv, beta, beta_old, neta, c, c_old, s, s_old,
         ro1 = 1.0, ro2, ro3, alpha, delta, norm_r;
  unsigned j;
  int i;
  if (!m) return -1;
  for (i = 0; i < neq; i++) m[i] = 1.0 / ad[i];
  if (newx)
    for (i = 0; i < neq; i++) x[i] = 0.0;
  for (i = 0; i < neq; i++) z[i] = b[i] * sqrt(m[i]);
  conv = tol * sqrt(orc_dot(z, z, neq));
  orc_matvec(storage, unsym, neq, ia, ja, al, ad, x, z);
  for (i = 0; i < neq; i++) {
    v[i] = b[i] - z[i];
    v0[i] = w0[i] = w00[i] = 0.0;
    z0[i] = v[i] * m[i];
  }
  beta = sqrt(fabs(orc_dot(v, z0, neq)));
  norm_r = beta;
  neta = beta;
  beta_old = beta;
  c_old = c = 1.0;
  s_old = s = 0.0;
  for (j = 0; j < maxit; j++) {
    orc_matvec(storage, unsym, neq, ia, ja, al, ad, z0, p);
    t1 = 1.0 / (beta * beta);
    alpha = orc_dot(z0, p, neq) * t1;
    t1 = 1.0 / beta;
    t2 = -alpha / beta;
    t3 = -beta / beta_old;
    for (i = 0; i < neq; i++) {
      p[i] = t1 * p[i] + t2 * v[i] + t3 * v0[i];
      z[i] = p[i] * m[i];
    }
    beta_old = beta;
    beta = sqrt(orc_dot(z, p, neq));
    delta = c * alpha - c_old * s * beta_old;
    ro2 = s * alpha + c_old * c * beta_old;
    ro3 = s_old * beta_old;
    c_old = c;
    s_old = s;
    orc_sym_ortho(delta, beta, &c, &s, &ro1);
    t1 = 1.0 / (beta_old * ro1);
    t2 = -ro2 / ro1;
    t3 = -ro3 / ro1;
    t4 = c * neta;
    for (i = 0; i < neq; i++) {
      w[i] = t1 * z0[i] + t2 * w0[i] + t3 * w00[i];
      x[i] += t4 * w[i];
    }
    /* v0 <- v, v <- p, z0 <- z, w00 <- w0, w0 <- w (by rotation) */
    tmp = v0; v0 = v; v = p; p = tmp;
    tmp = z0; z0 = z; z = tmp;
    tmp = w00; w00 = w0; w0 = w; w = tmp;
    norm_r = fabs(s) * norm_r;
    if (norm_r < conv) break;
    neta = -s * neta;
  }
  /* post-processing, Iters.c:481-497 */
  orc_matvec(storage, unsym, neq, ia, ja, al, ad, x, z);
  st->xKx = orc_dot(x, z, neq);
  st->norm_x = sqrt(orc_dot(x, x, neq));
  for (i = 0; i < neq; i++) {
    v[i] = b[i] - z[i];
    z[i] = v[i] * sqrt(fabs(m[i]));
  }
  st->norm_r = sqrt(orc_dot(v, v, neq));
  st->norm_r_m = sqrt(orc_dot(z, z, neq));
  st->conv = conv;
  st->iters = (int)j + 1;
  st->status = j == maxit ? 1 : 0;
  free(m);
  return st->status;
}

/* Bicgstab.c:1172-1460 (pbicgstabl2): BiCGSTAB(2), right-preconditioned. */
int orc_pbicgstabl2(int storage, int unsym, int neq, const int *ia,
                    const int *ja, const double *al, const double *ad,
                    const double *b, double *x, double tol, unsigned maxit,
                    int newx, orc_stats *st)
{
  double *m = malloc(sizeof(double) * (size_t)neq * 12);
  double *t = m + neq, *v = t + neq, *r = v + neq, *u = r + neq,
         *r0 = u + neq, *w = r0 + neq, *s = w + neq, *p = s + neq,
         *h = p + neq, *z = h + neq;
  double alpha, beta, d, conv, rr0, rr1, omega1, omega2, gamma, mi, ni, tau;
  unsigned j;
  int i;
  if (!m) return -1;
  for (i = 0; i < neq; i++) m[i] = 1.0 / ad[i];
  if (newx)
    for (i = 0; i < neq; i++) x[i] = 0.0;
  d = orc_dot(b, b, neq);
  conv = tol * sqrt(d);
  orc_matvec(storage, unsym, neq, ia, ja, al, ad, x, t);
  for (i = 0; i < neq; i++) {
    r0[i] = b[i] - t[i];
    r[i] = r0[i];
    u[i] = 0.0;
  }
  rr0 = 1.0;
  alpha = 0.0;
  omega2 = 1.0;
  for (j = 0; j < maxit; j++) {
    rr0 = -omega2 * rr0;
    /* even BiCG step */
    rr1 = orc_dot(r, r0, neq);
    beta = alpha * rr1 / rr0;
    rr0 = rr1;
    for (i = 0; i < neq; i++) {
      u[i] = r[i] - beta * u[i];
      z[i] = u[i] * m[i];
    }
    orc_matvec(storage, unsym, neq, ia, ja, al, ad, z, v);
    gamma = orc_dot(v, r0, neq);
    alpha = rr0 / gamma;
    for (i = 0; i < neq; i++) {
      r[i] -= alpha * v[i];
      p[i] = r[i] * m[i];
    }
    orc_matvec(storage, unsym, neq, ia, ja, al, ad, p, s);
    for (i = 0; i < neq; i++) x[i] += alpha * z[i];
    /* odd BiCG step */
    rr1 = orc_dot(s, r0, neq);
    beta = alpha * rr1 / rr0;
    rr0 = rr1;
    for (i = 0; i < neq; i++) {
      v[i] = s[i] - beta * v[i];
      p[i] = v[i] * m[i];
    }
    orc_matvec(storage, unsym, neq, ia, ja, al, ad, p, w);
    gamma = orc_dot(w, r0, neq);
    alpha = rr0 / gamma;
    for (i = 0; i < neq; i++) {
      u[i] = r[i] - beta * u[i];
      r[i] -= alpha * v[i];
      s[i] -= alpha * w[i];
      p[i] = s[i] * m[i];
      z[i] = u[i] * m[i];
      h[i] = r[i] * m[i];
    }
    orc_matvec(storage, unsym, neq, ia, ja, al, ad, p, t);
    /* GCR(2) part */
    omega1 = orc_dot(r, s, neq);
    mi = orc_dot(s, s, neq);
    ni = orc_dot(s, t, neq);
    tau = orc_dot(t, t, neq);
    omega2 = orc_dot(r, t, neq);
    tau = tau - ni * ni / mi;
    omega2 = (omega2 - ni * omega1 / mi) / tau;
    omega1 = (omega1 - ni * omega2) / mi;
    for (i = 0; i < neq; i++) {
      x[i] += omega1 * h[i] + omega2 * p[i] + alpha * z[i];
      r[i] -= (omega1 * s[i] + omega2 * t[i]);
    }
    d = orc_dot(r, r, neq);
    if (sqrt(d) < conv) break;
    for (i = 0; i < neq; i++) u[i] -= (omega1 * v[i] + omega2 * w[i]);
  }
  /* post-processing, Bicgstab.c:1395-1410 */
  orc_matvec(storage, unsym, neq, ia, ja, al, ad, x, z);
  st->xKx = orc_dot(x, z, neq);
  st->norm_x = sqrt(orc_dot(x, x, neq));
  for (i = 0; i < neq; i++) r[i] = b[i] - z[i];
  st->norm_r = sqrt(orc_dot(r, r, neq));
  st->norm_r_m = 0.0;
  st->conv = conv;
  st->iters = (int)j + 1;
  st->status = j == maxit ? 1 : 0;
  free(m);
  return st->status;
}

/* Iters.c:587-800 (gmres): restarted GMRES(nk) with the Jacobi
 * preconditioner on the left, modified Gram-Schmidt and Givens rotations.
 * As in the reference, a cycle always runs all nk Arnoldi steps, and the
 * update uses the first nk-1 of them (the back substitution and the sum
 * x += V y stop before the last column); convergence is tested on |e[nk]|
 * after each cycle, and maxit counts cycles.  iters = nk * cycles + 1. */
int orc_gmres(int storage, int unsym, int neq, const int *ia, const int *ja,
              const double *al, const double *ad, const double *b, double *x,
              double tol, unsigned maxit, int newx, int nk, orc_stats *st)
{
  double *m = malloc(sizeof(double) * (size_t)neq * (size_t)(nk + 2));
  double *g = m + neq, *g1, *g2;
  double *hh = malloc(sizeof(double) * (size_t)(nk + 1) * (size_t)nk);
  double *y = malloc(sizeof(double) * (size_t)nk * 3 + sizeof(double) * (nk + 1));
  double *c = y + nk, *s = c + nk, *e = s + nk;
  double tmp, norm, eConv, beta, h1, h2, aux1, aux2, r;
  unsigned l;
  int i, j, ni = 0, nIt = 0;
  long k;
#define HH(row, col) hh[(long)(row) * nk + (col)]
  if (!m || !hh || !y) {
    free(m); free(hh); free(y);
    return -1;
  }
  for (k = 0; k < (long)(nk + 1) * nk; k++) hh[k] = 0.0;
  for (k = 0; k < 3L * nk + nk + 1; k++) y[k] = 0.0;
  for (i = 0; i < neq; i++) m[i] = 1.0 / ad[i];
  if (newx)
    for (i = 0; i < neq; i++) x[i] = 0.0;
  for (i = 0; i < neq; i++) g[i] = b[i] * m[i];
  norm = sqrt(orc_dot(g, g, neq));
  eConv = tol * norm;
  for (l = 0; l < maxit; l++) {
    orc_matvec(storage, unsym, neq, ia, ja, al, ad, x, g);
    for (i = 0; i < neq; i++) g[i] = (b[i] - g[i]) * m[i];
    e[0] = sqrt(orc_dot(g, g, neq));
    tmp = 1.0 / e[0];
    for (i = 0; i < neq; i++) g[i] *= tmp;
    for (ni = 0; ni < nk; ni++, nIt++) {
      g1 = g + (long)ni * neq;
      g2 = g + (long)(ni + 1) * neq;
      orc_matvec(storage, unsym, neq, ia, ja, al, ad, g1, g2);
      for (i = 0; i < neq; i++) g2[i] *= m[i];
      for (j = 0; j <= ni; j++) {
        g1 = g + (long)j * neq;
        beta = orc_dot(g2, g1, neq);
        for (i = 0; i < neq; i++) g2[i] -= beta * g1[i];
        HH(j, ni) = beta;
      }
      norm = sqrt(orc_dot(g2, g2, neq));
      HH(ni + 1, ni) = norm;
      tmp = 1.0 / norm;
      for (i = 0; i < neq; i++) g2[i] *= tmp;
      for (j = 0; j < ni; j++) {
        h1 = HH(j, ni);
        h2 = HH(j + 1, ni);
        aux1 = c[j] * h1 + s[j] * h2;
        aux2 = -s[j] * h1 + c[j] * h2;
        HH(j, ni) = aux1;
        HH(j + 1, ni) = aux2;
      }
      h1 = HH(ni, ni);
      h2 = HH(ni + 1, ni);
      r = sqrt(h1 * h1 + h2 * h2);
      tmp = 1.0 / r;
      c[ni] = h1 * tmp;
      s[ni] = h2 * tmp;
      HH(ni, ni) = r;
      HH(ni + 1, ni) = 0.0;
      e[ni + 1] = -s[ni] * e[ni];
      e[ni] = c[ni] * e[ni];
    }
    if (ni == nk) ni--;
    y[ni] = e[ni] / HH(ni, ni);
    for (i = ni - 1; i >= 0; i--) {
      y[i] = 0.0;
      for (j = i + 1; j < ni; j++) y[i] -= HH(i, j) * y[j];
      y[i] = (y[i] + e[i]) / HH(i, i);
    }
    for (j = 0; j < ni; j++) {
      tmp = y[j];
      g1 = g + (long)j * neq;
      for (i = 0; i < neq; i++) x[i] += g1[i] * tmp;
    }
    if (fabs(e[ni + 1]) < eConv) break;
  }
#undef HH
  /* post-processing, Iters.c:746-760 */
  g1 = g;
  g2 = g + neq;
  orc_matvec(storage, unsym, neq, ia, ja, al, ad, x, g1);
  st->xKx = orc_dot(x, g1, neq);
  st->norm_x = sqrt(orc_dot(x, x, neq));
  for (i = 0; i < neq; i++) g2[i] = b[i] - g1[i];
  st->norm_r = sqrt(orc_dot(g2, g2, neq));
  st->norm_r_m = 0.0;
  st->conv = eConv;
  st->iters = nIt + 1;
  st->status = l == maxit ? 1 : 0;
  free(m);
  free(hh);
  free(y);
  return st->status;
}

/* ======================================================================
 * Diffusion system assembly: systFormDif (CellLoop.c:285-455) calling
 * cellDif3D (CellDif.c:312-537) per cell, then csr()/ellPack() (Csr.c:549,
 * EllPack.c:113).  Every floating-point expression keeps the reference's
 * operand order (C evaluates a + b + c as (a + b) + c).
 * ====================================================================== */

/* difusionSchemeNew, ndm = 3 (CellLib.c:5824-6000): split of the area
 * vector s into the implicit part e along ksi and the explicit rest t. */
static int dif_scheme(const double s[3], const double k[3], double e[3], double t[3], int icod)
{
  double ss, nk, tmp;
  int j;
  switch (icod) {
  case 1: /* ORTHOGONAL */
    ss = sqrt(s[0] * s[0] + s[1] * s[1] + s[2] * s[2]);
    for (j = 0; j < 3; j++) { e[j] = ss * k[j]; t[j] = 0.0; }
    return 0;
  case 2: /* MINIMAL */
    nk = s[0] * k[0] + s[1] * k[1] + s[2] * k[2];
    tmp = nk;
    for (j = 0; j < 3; j++) e[j] = tmp * k[j];
    for (j = 0; j < 3; j++) t[j] = s[j] - e[j];
    return 0;
  case 3: /* ORTHOGONALC */
    ss = sqrt(s[0] * s[0] + s[1] * s[1] + s[2] * s[2]);
    for (j = 0; j < 3; j++) e[j] = ss * k[j];
    for (j = 0; j < 3; j++) t[j] = s[j] - e[j];
    return 0;
  case 4: /* OVERRELAXED */
    ss = s[0] * s[0] + s[1] * s[1] + s[2] * s[2];
    nk = s[0] * k[0] + s[1] * k[1] + s[2] * k[2];
    tmp = ss / nk;
    for (j = 0; j < 3; j++) e[j] = tmp * k[j];
    for (j = 0; j < 3; j++) t[j] = s[j] - e[j];
    return 0;
  }
  return -1;
}

/* pLoad for constant loads (Loads.c:881-990, getLoads Loads.c:122-169):
 * adds the boundary face's share to the diagonal sP and the force p. */
static int dif_load(const orc_load *ld, double *sP, double *p, const double n[3], double kc,
                    double area, double dcca)
{
  double aP, h, tA, wfn, rhoEnv;
  switch (ld->type) {
  case 1: /* DIRICHLETBC */
    if (ld->var != 0) return -2;
    if (ld->np < 1) return -1;
    tA = ld->par[0];
    aP = kc * area / dcca;
    *sP += aP;
    *p += aP * tA;
    return 0;
  case 3: /* ROBINBC: par[0] = h, par[1] = the far value */
    h = ld->par[0];
    tA = ld->par[1];
    aP = ((kc * h) / (kc + h * dcca)) * area;
    *sP += aP;
    *p += aP * tA;
    return 0;
  case 2: /* NEUMANNBC */
    if (ld->np < 1) return -1;
    tA = ld->par[0];
    *p += area * tA;
    return 0;
  case 4: /* SINBC: sin products of the face centre */
    return -2;
  case 6: /* INLET: par[0] value, par[1..3] velocity, par[4] density */
    if (ld->var != 0) return -2;
    if (ld->np < 5) return -1;
    tA = ld->par[0];
    rhoEnv = ld->par[4];
    wfn = ld->par[1] * n[0] + ld->par[2] * n[1];
    wfn += ld->par[3] * n[2];
    *p -= wfn * rhoEnv * area * tA;
    aP = kc * area / dcca;
    *sP += aP;
    *p += aP * tA;
    return 0;
  case 7: /* OUTLET reads the cell velocity, which the diffusion cell has not */
    return -1;
  }
  return 0; /* other codes add nothing (pLoad's chain of tests falls through) */
}

/* the slot of column c in row r of a CSR pattern; writes every match as the
 * reference's search loop does */
static void dif_put(const int *ia, const int *ja, int r, int c, double *dst, double v)
{
  int k;
  for (k = ia[r]; k < ia[r + 1]; k++)
    if (ja[k] == c) dst[k] = v;
}

int orc_dif_assemble(const orc_dif_mesh *m, const orc_load *loads, int nloads,
                     const orc_dif_opts *o, const double *density,
                     const double *cdiff, const double *u0,
                     const double *gradu0, int storage, int unsym, int neq,
                     int nad, const int *ia, const int *ja, double *a,
                     double *ad, double *b, double *rcell, int forces,
                     int matrix, int calrcell)
{
  enum { MAXF = 32 };
  const int mv = m->maxviz;
  int nel, f, j, rc;
  (void)neq;
  if (mv < 1 || mv > MAXF - 1) return -1;
  for (nel = 0; nel < m->numel; nel++) {
    double lA[MAXF], ksi[3], nrm[3], s[3], e[3], t[3], gf[3], gc[3], v[3];
    int viz[MAXF], lid[MAXF];
    const int nf = m->nface[nel];
    const short *fr = m->facer + (long)nel * (mv + 1);
    double p = 0.0, sP = 0.0, r = 0.0, kc, rho, vol, lB;
    int row;
    if (calrcell) rcell[nel] = 0.0;
    if (nf < 1 || nf > mv) return -1;
    if (fr[nf] >= 1) continue; /* no equation in this cell */
    if (m->caltype[m->mat[nel] - 1] != 1) return -1;
    row = m->id[nel] - 1;
    kc = cdiff[nel];
    rho = density[nel];
    vol = m->volume[nel];
    for (f = 0; f < nf; f++) {
      const long q = (long)nel * mv + f;
      const int face = m->cellface[q] - 1;
      const double ch = (m->owner[2 * face] - 1 == nel) ? 1.0 : -1.0;
      const double mk = m->mksi[face], area = m->area[face];
      const double *xmcc = m->xmcc + 3 * q;
      viz[f] = m->nelcon[q] - 1;
      lid[f] = viz[f] != -2 ? m->id[viz[f]] - 1 : -1;
      for (j = 0; j < 3; j++) {
        ksi[j] = ch * m->ksi[3 * face + j];
        nrm[j] = ch * m->normal[3 * face + j];
      }
      if (viz[f] > -1) {
        const int nb = viz[f];
        double duDksi, alpha, am1, coef, modE, dfd, gfk, du;
        duDksi = (u0[nb] - u0[nel]) / mk;
        for (j = 0; j < 3; j++) s[j] = area * nrm[j];
        if (dif_scheme(s, ksi, e, t, o->icod)) return -1;
        /* interpolFace, INTPOLFACELINEAR (CellLib.c:7174-7200) */
        for (j = 0; j < 3; j++) v[j] = m->vskew[3 * face + j] + xmcc[j];
        alpha = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]) / mk;
        am1 = 1.0 - alpha;
        coef = alpha / kc + am1 / cdiff[nb];
        coef = 1.0 / coef;
        modE = sqrt(e[0] * e[0] + e[1] * e[1] + e[2] * e[2]);
        dfd = coef * modE / mk;
        for (j = 0; j < 3; j++) gf[j] = am1 * gradu0[3 * nel + j] + alpha * gradu0[3 * nb + j];
        gfk = gf[0] * ksi[0] + gf[1] * ksi[1] + gf[2] * ksi[2];
        du = duDksi - gfk;
        for (j = 0; j < 3; j++) gc[j] = gf[j] + du * ksi[j];
        gfk = gc[0] * t[0] + gc[1] * t[1] + gc[2] * t[2];
        lA[f] = dfd;
        p += coef * gfk;
      } else {
        lA[f] = 0.0;
        if (fr[f]) {
          const int l = fr[f] - 1;
          if (l < 0 || l >= nloads) return -1;
          rc = dif_load(&loads[l], &sP, &p, nrm, kc, area, m->dcca[q]);
          if (rc) return rc;
        }
      }
    }
    /* implicit time term, CellDif.c:485-497 */
    if (o->time_flag) {
      if (o->time_type == 0)
        sP += rho * vol / o->dt;
      else if (o->time_type == 1) {
        const double tmp = 1.e0 / o->dt + 1.e0 / (o->dt + o->dt0);
        sP += tmp * rho * vol;
      }
    }
    lA[nf] = sP;
    for (f = 0; f < nf; f++) lA[nf] += lA[f];
    for (f = 0; f < nf; f++)
      if (viz[f] > -1) {
        if (lid[f] == -2)
          p += lA[f] * u0[viz[f]];
        else
          r += lA[f] * u0[viz[f]];
      }
    r += p - lA[nf] * u0[nel];
    for (f = 0; f < nf; f++) lA[f] *= -1.e0;
    lB = o->fres ? r : p;
    if (calrcell) rcell[nel] = r;
    /* csr() / ellPack(), ndf = 1 */
    if (forces) b[row] = lB;
    if (!matrix) continue;
    ad[row] = lA[nf];
    if (storage == ORC_ELLPACK) {
      const int w = ia[0];
      for (f = 0; f < nf; f++) a[(long)row * w + f] = lA[f];
      continue;
    }
    for (f = 0; f < nf; f++) {
      const int c = lid[f];
      if (c <= -1) continue;
      if (storage == ORC_CSRC && unsym) {
        if (c < row)
          dif_put(ia, ja, row, c, a, lA[f]);
        else if (c > row)
          dif_put(ia, ja, c, row, a + nad, lA[f]);
      } else {
        dif_put(ia, ja, row, c, a, lA[f]);
      }
    }
  }
  return 0;
}

/* ======================================================================
 * Pressure-correction assembly: systFormSimplePres (CellLoopInc.c:471-700)
 * calling cellSimplePres3D (CellPres.c:903-1218) per cell.
 * ====================================================================== */

/* difusionSchemeAnisotropic, ndm = 3 (CellLib.c:6054-6170): only ORTHOGONAL
 * and OVERRELAXED set e and t */
static int pres_scheme(const double s[3], const double k[3], double e[3], double t[3], int icod)
{
  double ss, nk, tmp;
  int j;
  if (icod == 1) {
    ss = sqrt(s[0] * s[0] + s[1] * s[1] + s[2] * s[2]);
    for (j = 0; j < 3; j++) { e[j] = ss * k[j]; t[j] = 0.0; }
    return 0;
  }
  if (icod == 4) {
    ss = s[0] * s[0] + s[1] * s[1] + s[2] * s[2];
    nk = s[0] * k[0] + s[1] * k[1] + s[2] * k[2];
    tmp = ss / nk;
    for (j = 0; j < 3; j++) e[j] = tmp * k[j];
    for (j = 0; j < 3; j++) t[j] = s[j] - e[j];
    return 0;
  }
  return -1;
}

static double dot3c(const double a[3], const double b[3])
{
  return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}

/* pLoadSimplePres with fCal, no buoyancy (Loads.c:728-845): the pressure
 * load's share of the diagonal */
static int pres_load(const orc_load *ld, double *sP, const double e[3], const double n[3],
                     const double velC[3], double rhoC, double area, double dd)
{
  double tmp0, tmp1, modE, dc, m, modVel, rhoEnv;
  tmp0 = e[0] * e[0] + e[1] * e[1];
  tmp0 += e[2] * e[2];
  modE = sqrt(tmp0);
  switch (ld->type) {
  case 1: /* DIRICHLETBC */
    *sP += rhoC * modE / dd;
    return 0;
  case 13: /* INLETTOTALPRES: par = density, total pressure, direction
            * (getLoads copies the first five whatever np says) */
    rhoEnv = ld->par[0];
    dc = modE / dd;
    tmp0 = velC[0] * n[0] + velC[1] * n[1] + velC[2] * n[2];
    tmp1 = (ld->par[2] * n[0] + ld->par[3] * n[1] + ld->par[4] * n[2]) * area;
    m = rhoEnv * tmp0 * area;
    modVel = m / (rhoEnv * tmp1);
    tmp0 = rhoEnv * modVel;
    tmp1 = m - dc * tmp0 * tmp0;
    *sP += rhoEnv * m * dc / tmp1;
    return 0;
  case 10: /* OPEN: outflow only, added twice as the reference does */
    tmp0 = velC[0] * n[0] + velC[1] * n[1];
    tmp0 += velC[2] * n[2];
    if (tmp0 > 0.e0) {
      *sP += rhoC * modE / dd;
      *sP += rhoC * modE / dd;
    }
    return 0;
  }
  return 0; /* FLUXPRES without buoyancy and the other codes add nothing */
}

/* pLoadSimple with fCalVel = false, fCalPres = true (Loads.c:265-720): the
 * velocity load's mass flux in the pressure equation */
static int vel_load(const orc_load *ld, double *p, const double n[3], const double velC[3],
                    double rhoC, double area)
{
  double wfn, m, rho;
  switch (ld->type) {
  case 9:  /* INLETSTAICTPRES */
  case 7:  /* OUTLET */
    wfn = velC[0] * n[0] + velC[1] * n[1] + velC[2] * n[2];
    if (ld->type == 7) {
      wfn = velC[0] * n[0] + velC[1] * n[1];
      wfn += velC[2] * n[2];
    }
    m = rhoC * wfn * area;
    *p -= m;
    return 0;
  case 6: /* INLET: par[0..2] velocity, par[np-1] density (getLoads copies
           * np parameters) */
    if (ld->var != 0) return -2;
    if (ld->np < 3) return -1;
    wfn = ld->par[0] * n[0] + ld->par[1] * n[1];
    wfn += ld->par[2] * n[2];
    m = ld->par[ld->np - 1] * wfn * area;
    *p -= m;
    return 0;
  case 10: /* OPEN */
    wfn = velC[0] * n[0] + velC[1] * n[1];
    wfn += velC[2] * n[2];
    rho = wfn >= 0.e0 ? rhoC : ld->density;
    m = rho * wfn * area;
    *p -= m;
    return 0;
  case 13: /* INLETTOTALPRES */
    wfn = velC[0] * n[0] + velC[1] * n[1] + velC[2] * n[2];
    m = ld->par[0] * wfn * area;
    *p -= m;
    return 0;
  }
  return 0; /* MOVEWALL, STATICWALL, ...: nothing in the pressure equation */
}

int orc_pres_assemble(const orc_dif_mesh *m, const short *facevelr,
                      const orc_load *lvel, int nlvel, const orc_load *lpres,
                      int nlpres, int icod, const double *prop,
                      const double *pres, const double *gradpres,
                      const double *vel, const double *dfield, int storage,
                      int unsym, int neq, int nad, const int *ia,
                      const int *ja, double *a, double *ad, double *b,
                      double *rcell, int forces, int matrix, int calrcell)
{
  enum { MAXF = 32 };
  const int mv = m->maxviz;
  int nel, f, j, rc;
  (void)neq;
  if (mv < 1 || mv > MAXF - 1) return -1;
  if (icod != 1 && icod != 4) return -1;
  for (nel = 0; nel < m->numel; nel++) {
    double lA[MAXF], ksi[3], nrm[3], s[3], e[3], t[3], dF[3], wf[3], gf[3], v[3];
    int viz[MAXF], lid[MAXF];
    const int nf = m->nface[nel];
    const short *fr = m->facer + (long)nel * (mv + 1);
    const short *fv = facevelr + (long)nel * (mv + 1);
    const double *velC = vel + 3 * (long)nel, *gpC = gradpres + 3 * (long)nel;
    const double *dC = dfield + 3 * (long)nel;
    double p = 0.0, sP = 0.0, rhoC, presC;
    int row, lm;
    if (calrcell) rcell[nel] = 0.0;
    if (nf < 1 || nf > mv) return -1;
    if (fr[nf] > 0) continue; /* prescribed pressure: no equation */
    lm = m->mat[nel] - 1;
    if (m->caltype[lm] != 1) return -1;
    row = m->id[nel] - 1;
    rhoC = prop[lm * ORC_MAXPROP + ORC_DENSITY];
    presC = pres[nel];
    for (f = 0; f < nf; f++) {
      const long q = (long)nel * mv + f;
      const int face = m->cellface[q] - 1;
      const double ch = (m->owner[2 * face] - 1 == nel) ? 1.0 : -1.0;
      const double mk = m->mksi[face], area = m->area[face];
      const double *xmcc = m->xmcc + 3 * q;
      viz[f] = m->nelcon[q] - 1;
      lid[f] = viz[f] != -2 ? m->id[viz[f]] - 1 : -1;
      for (j = 0; j < 3; j++) {
        ksi[j] = ch * m->ksi[3 * face + j];
        nrm[j] = ch * m->normal[3 * face + j];
      }
      if (viz[f] > -1) {
        const int nb = viz[f];
        const double *velV = vel + 3 * (long)nb, *gpV = gradpres + 3 * (long)nb;
        const double *dV = dfield + 3 * (long)nb;
        const double rhoV = prop[(m->mat[nb] - 1) * ORC_MAXPROP + ORC_DENSITY];
        double alpha, am1, rho, modE, dfd, wfn, nk, g0, g1;
        /* interpolFace, INTPOLFACELINEAR (CellLib.c:7174-7200) */
        for (j = 0; j < 3; j++) v[j] = m->vskew[3 * face + j] + xmcc[j];
        alpha = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]) / mk;
        am1 = 1.0e0 - alpha;
        rho = am1 * rhoC + alpha * rhoV;
        for (j = 0; j < 3; j++) dF[j] = am1 * dC[j] + alpha * dV[j];
        for (j = 0; j < 3; j++) s[j] = dF[j] * area * nrm[j];
        if (pres_scheme(s, ksi, e, t, icod)) return -1;
        modE = sqrt(e[0] * e[0] + e[1] * e[1] + e[2] * e[2]);
        dfd = rho * modE / mk;
        lA[f] = dfd;
        /* interpolFaceVel, ndm = 3 (CellLib.c:6853-6960): Rhie-Chow face
         * velocity */
        for (j = 0; j < 3; j++) wf[j] = am1 * velC[j] + alpha * velV[j];
        wfn = dot3c(wf, nrm);
        for (j = 0; j < 3; j++) gf[j] = am1 * gpC[j] + alpha * gpV[j];
        g0 = (pres[nb] - presC) / mk;
        nk = dF[0] * ksi[0] * nrm[0] + dF[1] * ksi[1] * nrm[1] + dF[2] * ksi[2] * nrm[2];
        g1 = dot3c(gf, ksi);
        g1 = (g1 - g0) * nk;
        wfn += g1;
        p -= rho * wfn * area;
      } else {
        lA[f] = 0.0;
        if (fr[f]) {
          const int l = fr[f] - 1;
          if (l < 0 || l >= nlpres) return -1;
          for (j = 0; j < 3; j++) s[j] = dC[j] * area * nrm[j];
          if (pres_scheme(s, ksi, e, t, icod)) return -1;
          rc = pres_load(&lpres[l], &sP, e, nrm, velC, rhoC, area, m->dcca[q]);
          if (rc) return rc;
        }
        if (fv[f]) {
          const int l = fv[f] - 1;
          if (l < 0 || l >= nlvel) return -1;
          rc = vel_load(&lvel[l], &p, nrm, velC, rhoC, area);
          if (rc) return rc;
        }
      }
    }
    lA[nf] = sP;
    for (f = 0; f < nf; f++) lA[nf] += lA[f];
    for (f = 0; f < nf; f++) lA[f] *= -1.e0;
    if (calrcell) rcell[nel] = p;
    if (forces) b[row] = p;
    if (!matrix) continue;
    ad[row] = lA[nf];
    if (storage == ORC_ELLPACK) {
      const int w = ia[0];
      for (f = 0; f < nf; f++) a[(long)row * w + f] = lA[f];
      continue;
    }
    for (f = 0; f < nf; f++) {
      const int c = lid[f];
      if (c <= -1) continue;
      if (storage == ORC_CSRC && unsym) {
        if (c < row)
          dif_put(ia, ja, row, c, a, lA[f]);
        else if (c > row)
          dif_put(ia, ja, c, row, a + nad, lA[f]);
      } else {
        dif_put(ia, ja, row, c, a, lA[f]);
      }
    }
  }
  return 0;
}

/* ======================================================================
 * Momentum assembly: systFormSimpleVel (CellLoopInc.c:98-470) calling
 * cellSimpleVel3D (CellSimple.c:106-727) per cell, placed by csrSimple
 * (Csr.c:1024-1200): laminar (no eddy viscosity, no structural stress, no
 * wall model), first-order upwind (advectiveScheme FOUP, CellLib.c:6394:
 * no deferred correction), face velocity without Rhie-Chow.
 * ====================================================================== */

/* moveWall, not Dirichlet (CellLib.c:7715-7770): the wall's tangential
 * stress on the diagonals sPc and the force p */
static void move_wall(const double vC[3], const double vB[3], const double n[3], double sPc[3],
                      double p[3], double dcca, double visc, double area)
{
  const double aP = visc * area / dcca;
  sPc[0] += aP * (1.e0 - n[0] * n[0]);
  sPc[1] += aP * (1.e0 - n[1] * n[1]);
  sPc[2] += aP * (1.e0 - n[2] * n[2]);
  p[0] += aP * (vB[0] * (1.0 - n[0] * n[0]) + (vC[1] - vB[1]) * n[1] * n[0] +
                (vC[2] - vB[2]) * n[2] * n[0]);
  p[1] += aP * (vB[1] * (1.0 - n[1] * n[1]) + (vC[0] - vB[0]) * n[0] * n[1] +
                (vC[2] - vB[2]) * n[2] * n[1]);
  p[2] += aP * (vB[2] * (1.0 - n[2] * n[2]) + (vC[0] - vB[0]) * n[0] * n[2] +
                (vC[1] - vB[1]) * n[1] * n[2]);
}

/* nvd (CellLib.c): the weights of NVD function fn at phi~, as its table
 * gives them; MUSCL (2) and STOIC (7) have empty bodies there: (0, 0) */
static void nvd_table(double ph, int fn, double *w)
{
  const double third = 3.33333333333333333333E-1, two3 = 6.66666666666666666666E-1;
  w[0] = 0.0;
  w[1] = 0.0;
  if (fn == 2 || fn == 7) return;
  w[0] = 1.0;
  if (fn == 1) {
    if (ph >= 0 && ph <= 1.e0) { w[0] = 0.5; w[1] = 0.5; }
  } else if (fn == 3) {
    if (ph >= 0 && ph <= 5.0 / 6.0) { w[0] = 3.0 / 4.0; w[1] = 3.0 / 8.0; }
    else if (ph > 5.0 / 6.0 && ph <= 1.0) { w[0] = 0.0; w[1] = 1.0; }
  } else if (fn == 4) {
    if (ph >= 0 && ph <= 1.0 / 6.0) { w[0] = 3.0; w[1] = 0.0; }
    else if (ph > 1.0 / 6.0 && ph <= 0.7) { w[0] = 3.0 / 4.0; w[1] = 3.0 / 8.0; }
    else if (ph > 0.7 && ph <= 1.0) { w[0] = third; w[1] = two3; }
  } else if (fn == 5) {
    if (ph >= 0 && ph <= 5.e-1) { w[0] = 0.5; w[1] = 0.5; }
    else if (ph > 5e-1 && ph <= two3) { w[0] = 1.5; w[1] = 0.0; }
    else if (ph > two3 && ph <= 1.e0) { w[0] = 0.0; w[1] = 1.0; }
  } else if (fn == 6) {
    if (ph >= 0 && ph <= third) { w[0] = 2.0; w[1] = 0.0; }
    else if (ph > third && ph <= 0.5) { w[0] = 0.5; w[1] = 0.5; }
    else if (ph > 0.5 && ph <= two3) { w[0] = 1.5; w[1] = 0.0; }
    else if (ph > two3 && ph <= 1) { w[0] = 0.0; w[1] = 1.0; }
  } else if (fn == 8) {
    if (ph >= 0 && ph <= 5.e-1) { w[0] = 1.5; w[1] = 0.0; }
    else if (ph > 5e-1 && ph <= 1.0) { w[0] = 0.5; w[1] = 0.5; }
  } else if (fn == 9) {
    if (ph >= 0.e0 && ph <= 1.0 / 4.0) { w[0] = 2.5; w[1] = 0.0; }
    else if (ph > 1.0 / 4.0 && ph <= 1.e0) { w[0] = 0.5; w[1] = 0.5; }
  }
}

/* turbStructIntegral (CellLib.c:7586-7626); rv NULL on a boundary face */
static void struct_integral(const double *rc, const double *rv, const double *n, double *p,
                            double area, double g1, double g2)
{
  const double third = 3.33333333333333333333E-1; /* D1DIV3, Define.h:179 */
  double s[6], tmp;
  int k;
  if (!rv) {
    tmp = third * (rc[0] + rc[1] + rc[2]);
    for (k = 0; k < 3; k++) s[k] = rc[k] - tmp;
    for (k = 3; k < 6; k++) s[k] = rc[k];
  } else {
    for (k = 0; k < 3; k++) s[k] = g1 * rc[k] + g2 * rv[k];
    tmp = third * (s[0] + s[1] + s[2]);
    for (k = 0; k < 3; k++) s[k] -= tmp;
    for (k = 3; k < 6; k++) s[k] = g1 * rc[k] + g2 * rv[k];
  }
  p[0] -= area * (s[0] * n[0] + s[3] * n[1] + s[5] * n[2]);
  p[1] -= area * (s[3] * n[0] + s[1] * n[1] + s[4] * n[2]);
  p[2] -= area * (s[5] * n[0] + s[4] * n[1] + s[2] * n[2]);
}

/* dsnap: the D field at the call's start (Rhie-Chow), else NULL */
static int vel_assemble(const orc_dif_mesh *m, const short *facepresr, const double *cc,
                        const double *xm, const orc_load *lvel, int nlvel,
                        const orc_vel_opts *o, const double *prop, const double *pres,
                        const double *gradpres, const double *vel, const double *gradvel,
                        double *dfield, int storage, int unsym, int neq, int nad,
                        const int *ia, const int *ja, double *a, double *ad, double *b,
                        double *rcell, int forces, int matrix, int calrcell,
                        const double *dsnap)
{
  enum { MAXF = 32 };
  const int mv = m->maxviz, numel = m->numel;
  int nel, f, i, j, k;
  (void)facepresr;
  if (mv < 1 || mv > MAXF - 1 || storage == ORC_ELLPACK) return -1;
  /* any other typeSimple leaves D as the first neighbour's copy */
  if (o->type_simple != 1 && o->type_simple != 2) return -1;
  if (o->adv < 0 || o->adv > 6) return -1;
  if (o->adv == 4 && (o->adv_fn < 1 || o->adv_fn > 5)) return -1;
  if (o->adv == 5 && (o->adv_fn < 1 || o->adv_fn > 9)) return -1;
  for (nel = 0; nel < numel; nel++) {
    double lA[MAXF + 3], ksi[3], nrm[3], s[3], e[3], t[3];
    double p[3] = {0.0, 0.0, 0.0}, pf[3] = {0.0, 0.0, 0.0}, sPc[3] = {0.0, 0.0, 0.0};
    double rc[3], lB[3], gvC[3][3], velC[3], gpC[3], sP = 0.0, lAn, rhoC, muC, effC, presC;
    int viz[MAXF], lid[MAXF], lm, row;
    const int nf = m->nface[nel];
    const short *fr = m->facer + (long)nel * (mv + 1);
    if (calrcell) {
      rcell[nel] = 0.e0;
      rcell[numel + nel] = 0.e0;
      rcell[2 * numel + nel] = 0.e0;
    }
    if (nf < 1 || nf > mv) return -1;
    if (fr[nf] > 0) continue; /* prescribed velocity: no equation */
    lm = m->mat[nel] - 1;
    if (m->caltype[lm] != 1) return -1;
    row = m->id[nel] - 1;
    rhoC = prop[lm * ORC_MAXPROP + ORC_DENSITY];
    muC = prop[lm * ORC_MAXPROP + 0];
    effC = muC + (o->fturb ? o->eddy[nel] : 0.0e0); /* CellSimple.c:207-209 */
    presC = pres[nel];
    for (i = 0; i < 3; i++) {
      for (j = 0; j < 3; j++) gvC[i][j] = gradvel[9 * (long)nel + 3 * i + j];
      gpC[i] = gradpres[3 * (long)nel + i];
      velC[i] = vel[3 * (long)nel + i];
    }
    for (f = 0; f < nf; f++) {
      const long q = (long)nel * mv + f;
      const int face = m->cellface[q] - 1;
      const double ch = (m->owner[2 * face] - 1 == nel) ? 1.0 : -1.0;
      const double mk = m->mksi[face], area = m->area[face];
      const double *xmcc = m->xmcc + 3 * q;
      viz[f] = m->nelcon[q] - 1;
      lid[f] = viz[f] != -2 ? m->id[viz[f]] - 1 : -1;
      for (j = 0; j < 3; j++) {
        ksi[j] = ch * m->ksi[3 * face + j];
        nrm[j] = ch * m->normal[3 * face + j];
      }
      if (viz[f] > -1) {
        const int nb = viz[f];
        const int lmv = m->mat[nb] - 1;
        const double rhoV = prop[lmv * ORC_MAXPROP + ORC_DENSITY];
        const double effV = prop[lmv * ORC_MAXPROP + 0] + (o->fturb ? o->eddy[nb] : 0.0e0);
        const double presV = pres[nb];
        double velV[3], gpV[3], duDksi[3], gvV[3][3], ccV[3], lXm[3], v[3];
        double alpha, am1, visc, modE, dfd, density, wfn, cv, gf[3][3], wf[3], gvc[3][3];
        double dfdc[3], gk, du, p1, p2, pFace, tmp;
        for (i = 0; i < 3; i++) {
          velV[i] = vel[3 * (long)nb + i];
          gpV[i] = gradpres[3 * (long)nb + i];
          duDksi[i] = (velV[i] - velC[i]) / mk;
          for (j = 0; j < 3; j++) gvV[i][j] = gradvel[9 * (long)nb + 3 * i + j];
          ccV[i] = cc[3 * (long)nb + i];
          lXm[i] = xm[3 * (long)face + i];
        }
        for (j = 0; j < 3; j++) s[j] = area * nrm[j];
        if (dif_scheme(s, ksi, e, t, o->icod)) return -1;
        for (j = 0; j < 3; j++) v[j] = m->vskew[3 * face + j] + xmcc[j];
        alpha = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]) / mk;
        am1 = 1.0e0 - alpha;
        /* mediaHarmonica (CellLib.c:7879) */
        visc = (effC == 0.e0 || effV == 0.e0) ? 0.e0 : 1.e0 / (alpha / effC + am1 / effV);
        modE = sqrt(e[0] * e[0] + e[1] * e[1] + e[2] * e[2]);
        dfd = visc * modE / mk;
        for (i = 0; i < 3; i++) {
          for (j = 0; j < 3; j++) gf[i][j] = am1 * gvC[i][j] + alpha * gvV[i][j];
          wf[i] = am1 * velC[i] + alpha * velV[i];
        }
        density = am1 * rhoC + alpha * rhoV;
        wfn = wf[0] * nrm[0] + wf[1] * nrm[1] + wf[2] * nrm[2];
        if (o->rhie) {
          /* interpolFaceVel, ndm = 3 (CellLib.c:6853-6960) with the face D
           * of CellSimple.c:339-350, both D values from the call's start */
          const double *dd = dsnap ? dsnap : dfield;
          double dF[3], gp[3], g0, g1, nk;
          for (j = 0; j < 3; j++) {
            dF[j] = am1 * dd[3 * (long)nel + j] + alpha * dd[3 * (long)nb + j];
            gp[j] = am1 * gpC[j] + alpha * gpV[j];
          }
          g0 = (presV - presC) / mk;
          nk = dF[0] * ksi[0] * nrm[0] + dF[1] * ksi[1] * nrm[1] + dF[2] * ksi[2] * nrm[2];
          g1 = gp[0] * ksi[0] + gp[1] * ksi[1] + gp[2] * ksi[2];
          g1 = (g1 - g0) * nk;
          wfn += g1;
        }
        for (i = 0; i < 3; i++) {
          gk = gf[i][0] * ksi[0] + gf[i][1] * ksi[1] + gf[i][2] * ksi[2];
          du = duDksi[i] - gk;
          for (j = 0; j < 3; j++) gvc[i][j] = gf[i][j] + du * ksi[j];
          gk = gvc[i][0] * t[0] + gvc[i][1] * t[1] + gvc[i][2] * t[2];
          dfdc[i] = visc * gk;
        }
        cv = density * wfn * area;
        lA[f] = dfd - (cv < 0.0e0 ? cv : 0.0e0);
        sP += cv;
        /* advectiveScheme (CellLib.c:6394-6480), cv in the place of wfn */
        {
          double cvc[3] = {0.e0, 0.e0, 0.e0}, rV[3];
          for (j = 0; j < 3; j++) rV[j] = lXm[j] - ccV[j];
          for (i = 0; i < 3; i++) {
            if (o->adv == 2) { /* deferredCd, CellLib.c:5113-5127 */
              const double cd = am1 * velC[i] + alpha * velV[i];
              cvc[i] = cd - (cv < 0.e0 ? velV[i] : velC[i]);
            } else if (o->adv == 3) { /* upwindLinearV1, CellLib.c:5072-5090 */
              if (cv < 0.e0)
                cvc[i] = gvV[i][0] * rV[0] + gvV[i][1] * rV[1] + gvV[i][2] * rV[2];
              else
                cvc[i] = gvC[i][0] * xmcc[0] + gvC[i][1] * xmcc[1] + gvC[i][2] * xmcc[2];
            } else if (o->adv == 4) { /* faceBaseTvdV1, CellLib.c:4845-4875 */
              double du, gf, r, lim = 0.e0, a, b, c;
              const double *vs = m->vskew + 3 * face;
              if (cv < 0.e0) {
                du = velC[i] - velV[i] + 1.e-14;
                gf = gvV[i][0] * ksi[0] + gvV[i][1] * ksi[1];
                gf += gvV[i][2] * ksi[2];
                gf = -2.e0 * gf * mk;
              } else {
                du = velV[i] - velC[i] + 1.e-14;
                gf = gvC[i][0] * ksi[0] + gvC[i][1] * ksi[1];
                gf += gvC[i][2] * ksi[2];
                gf = 2.e0 * gf * mk;
              }
              r = gf / du - 1.0e0;
              /* limitFaceBase, CellLib.c:4482-4530 (min/max of Define.h:455-456) */
              switch (o->adv_fn) {
                case 1: a = fabs(r); lim = (r + a) / (1.0e0 + a); break;
                case 2: if (r > 0.e0) { a = r * r; lim = (r + a) / (1.0e0 + a); } break;
                case 3: a = r < 1.e0 ? r : 1.e0; lim = 0.e0 > a ? 0.e0 : a; break;
                case 4: a = r < 2.e0 ? r : 2.e0; lim = 0.e0 > a ? 0.e0 : a; break;
                default:
                  a = 2.e0 * r < 1.e0 ? 2.e0 * r : 1.e0;
                  b = r < 2.e0 ? r : 2.e0;
                  c = a > b ? a : b;
                  lim = 0.e0 > c ? 0.e0 : c;
                  break;
              }
              cvc[i] = 0.5e0 * lim * du;
              cvc[i] -= gvc[i][0] * vs[0] + gvc[i][1] * vs[1] + gvc[i][2] * vs[2];
            } else if (o->adv == 5) { /* faceBaseNvd, CellLib.c:4900-4937 */
              double gf, phi, w[2];
              if (cv < 0.e0) {
                gf = gvV[i][0] * ksi[0] + gvV[i][1] * ksi[1];
                gf += gvV[i][2] * ksi[2];
                gf = -2.e0 * gf * mk + 1.e-32;
                phi = (velV[i] - velC[i]) / gf + 1.e0;
                nvd_table(phi, o->adv_fn, w);
                cvc[i] = (w[0] - 1.0) * velV[i] + w[1] * velC[i] +
                         (1.0 - w[0] - w[1]) * (velC[i] - gf);
              } else {
                gf = gvC[i][0] * ksi[0] + gvC[i][1] * ksi[1];
                gf += gvC[i][2] * ksi[2];
                gf = 2.e0 * gf * mk + 1.e-32;
                phi = (velC[i] - velV[i]) / gf + 1.e0;
                nvd_table(phi, o->adv_fn, w);
                cvc[i] = (w[0] - 1.0) * velC[i] + w[1] * velV[i] +
                         (1.0 - w[0] - w[1]) * (velV[i] - gf);
              }
            } else if (o->adv == 6) { /* deferredLust, CellLib.c:5162-5198 */
              double gf, up, ul, uf1, uf2, cd;
              if (cv < 0.e0) {
                gf = gvV[i][0] * rV[0] + gvV[i][1] * rV[1];
                gf += gvV[i][2] * rV[2];
                up = velV[i];
              } else {
                gf = gvC[i][0] * xmcc[0] + gvC[i][1] * xmcc[1];
                gf += gvC[i][2] * xmcc[2];
                up = velC[i];
              }
              ul = up + gf;
              uf1 = velC[i] + gvC[i][0] * xmcc[0] + gvC[i][1] * xmcc[1];
              uf2 = velV[i] + gvV[i][0] * rV[0] + gvV[i][1] * rV[1];
              uf1 += gvC[i][2] * xmcc[2];
              uf2 += gvV[i][2] * rV[2];
              cd = am1 * uf1 + alpha * uf2;
              cvc[i] = o->adv_beta * ul + (1.e0 - o->adv_beta) * cd - up;
            }
          }
          for (i = 0; i < 3; i++) p[i] += dfdc[i] - cv * cvc[i];
        }
        /* facePressure (CellLib.c:7499), interior */
        if (o->fso) {
          for (j = 0; j < 3; j++) v[j] = lXm[j] - ccV[j];
          p1 = presC + gpC[0] * xmcc[0] + gpC[1] * xmcc[1] + gpC[2] * xmcc[2];
          p2 = presV + gpV[0] * v[0] + gpV[1] * v[1] + gpV[2] * v[2];
          pFace = 0.5e0 * (p1 + p2);
        } else {
          pFace = am1 * presC + alpha * presV;
        }
        tmp = pFace * area;
        for (i = 0; i < 3; i++) pf[i] += tmp * nrm[i];
        /* viscosityPartExp (CellLib.c:7439), fDiv false */
        if (o->fvisc) {
          const double aP = muC * area;
          for (i = 0; i < 3; i++)
            p[i] += aP * (gvc[0][i] * nrm[0] + gvc[1][i] * nrm[1] + gvc[2][i] * nrm[2]);
        }
        if (o->fstruc)
          struct_integral(o->stress + 6 * (long)nel, o->stress + 6 * (long)nb, nrm, p, area,
                          am1, alpha);
      } else {
        double tmp;
        lA[f] = 0.0e0;
        /* facePressure, boundary: the cell's own pressure on the face */
        tmp = presC * area;
        for (i = 0; i < 3; i++) pf[i] += tmp * nrm[i];
        if (o->fstruc) struct_integral(o->stress + 6 * (long)nel, 0, nrm, p, area, 0.0, 0.0);
        for (j = 0; j < 3; j++) s[j] = area * nrm[j];
        if (dif_scheme(s, ksi, e, t, o->icod)) return -1;
        if (fr[f]) {
          const int l = fr[f] - 1;
          const orc_load *ld;
          double tA[3] = {0.0, 0.0, 0.0};
          if (l < 0 || l >= nlvel) return -1;
          ld = &lvel[l];
          if (ld->type == 8 || ld->type == 14) { /* MOVEWALL, STATICWALL */
            double visc = effC;
            if (o->fwall) { /* Loads.c:300-313: the wall model's viscosity */
              const double yp = o->wallpar[4 * (long)nel], up = o->wallpar[4 * (long)nel + 1];
              visc = yp > 0.01e0 ? muC * yp / up : muC;
            }
            if (ld->type == 8)
              for (j = 0; j < 3; j++) tA[j] = ld->par[j];
            move_wall(velC, tA, nrm, sPc, p, m->dcca[q], visc, area);
          } else if (ld->type == 6) { /* INLET */
            double wfn, ss[6], tr, mflux;
            if (ld->var != 0) return -2;
            if (ld->np < 3) return -1;
            for (j = 0; j < 3; j++) tA[j] = ld->par[j];
            wfn = tA[0] * nrm[0] + tA[1] * nrm[1];
            wfn += tA[2] * nrm[2];
            mflux = ld->par[ld->np - 1] * wfn * area;
            /* stress (CellLib.c:7013), lambda = 0 */
            tr = gvC[0][0] + gvC[1][1] + gvC[2][2];
            ss[0] = 2.e0 * muC * gvC[0][0] + 0.0 * tr;
            ss[1] = 2.e0 * muC * gvC[1][1] + 0.0 * tr;
            ss[2] = 2.e0 * muC * gvC[2][2] + 0.0 * tr;
            ss[3] = muC * (gvC[1][0] + gvC[0][1]);
            ss[4] = muC * (gvC[2][1] + gvC[1][2]);
            ss[5] = muC * (gvC[2][0] + gvC[0][2]);
            p[0] += ss[0] * s[0] + ss[3] * s[1] + ss[5] * s[2];
            p[1] += ss[3] * s[0] + ss[1] * s[1] + ss[4] * s[2];
            p[2] += ss[5] * s[0] + ss[4] * s[1] + ss[2] * s[2];
            p[0] -= mflux * tA[0];
            p[1] -= mflux * tA[1];
            p[2] -= mflux * tA[2];
          } else if (ld->type == 7 || ld->type == 10) { /* OUTLET, OPEN */
            const double wfn = dot3c(velC, nrm);
            if (ld->type == 10 && wfn < 0.e0) {
              /* OPEN inflow (Loads.c:604-627): the cell's own direction */
              const double mflux = ld->density * wfn * area;
              double modv = velC[0] * velC[0] + velC[1] * velC[1];
              double aP;
              modv += velC[2] * velC[2];
              modv = 1.e0 / sqrt(modv);
              aP = mflux * wfn * modv;
              for (k = 0; k < 3; k++) p[k] -= aP * velC[k];
            } else {
              /* OUTLET (Loads.c:436-518) and OPEN outflow (Loads.c:531-600) */
              const double mflux = rhoC * wfn * area;
              double ef[3], prod[3], gvf[3][3], mod, tf;
              if (ld->type == 7) { /* stress (CellLib.c:7013), lambda = 0 */
                const double tr = gvC[0][0] + gvC[1][1] + gvC[2][2];
                double ss[6];
                ss[0] = 2.e0 * muC * gvC[0][0] + 0.0 * tr;
                ss[1] = 2.e0 * muC * gvC[1][1] + 0.0 * tr;
                ss[2] = 2.e0 * muC * gvC[2][2] + 0.0 * tr;
                ss[3] = muC * (gvC[1][0] + gvC[0][1]);
                ss[4] = muC * (gvC[2][1] + gvC[1][2]);
                ss[5] = muC * (gvC[2][0] + gvC[0][2]);
                p[0] += ss[0] * s[0] + ss[3] * s[1] + ss[5] * s[2];
                p[1] += ss[3] * s[0] + ss[1] * s[1] + ss[4] * s[2];
                p[2] += ss[5] * s[0] + ss[4] * s[1] + ss[2] * s[2];
              }
              /* gradFaceNull (CellLib.c:5477-5600): the cell gradient less
               * its part along the centroid-to-face direction */
              mod = sqrt(xmcc[0] * xmcc[0] + xmcc[1] * xmcc[1] + xmcc[2] * xmcc[2]);
              for (j = 0; j < 3; j++) ef[j] = xmcc[j] / mod;
              for (i = 0; i < 3; i++)
                prod[i] = gvC[i][0] * ef[0] + gvC[i][1] * ef[1] + gvC[i][2] * ef[2];
              for (i = 0; i < 3; i++)
                for (j = 0; j < 3; j++) gvf[i][j] = gvC[i][j] - prod[i] * ef[j];
              for (i = 0; i < 3; i++) {
                tf = gvf[i][0] * xmcc[0] + gvf[i][1] * xmcc[1] + gvf[i][2] * xmcc[2];
                p[i] -= mflux * tf;
              }
              for (i = 0; i < 3; i++) sPc[i] += mflux;
            }
          } else if (ld->type == 9) {
            /* INLETSTAICTPRES (Loads.c:364-392).  getLoads copies nothing
             * for this type (Loads.c:148-150), so the reference reads an
             * uninitialised par[]; this restatement reads the load's own
             * par[0..2] as the inflow direction. */
            const double wfn = dot3c(velC, nrm);
            const double dn = ld->par[0] * nrm[0] + ld->par[1] * nrm[1] + ld->par[2] * nrm[2];
            const double t3 = wfn / dn, mflux = rhoC * wfn * area;
            for (k = 0; k < 3; k++) p[k] -= mflux * ld->par[k] * t3;
          } else if (ld->type == 13) {
            /* INLETTOTALPRES (Loads.c:634-672): density par[0], direction
             * par[2..4] (getLoads copies 5 parameters) */
            const double rho = ld->par[0];
            const double ev[3] = {ld->par[2], ld->par[3], ld->par[4]};
            const double t0 = dot3c(velC, nrm), t1 = dot3c(ev, nrm) * area;
            const double mflux = rho * t0 * area;
            const double modv = mflux / (rho * t1), tm = mflux * modv;
            for (k = 0; k < 3; k++) p[k] -= tm * ev[k];
          }
        }
      }
    }
    /* implicit time term, CellSimple.c:606-617 */
    if (o->time_flag) {
      if (o->time_type == 0)
        sP += rhoC * m->volume[nel] / o->dt;
      else if (o->time_type == 1) {
        const double tmp = 1.e0 / o->dt + 1.e0 / (o->dt + o->dt0);
        sP += tmp * rhoC * m->volume[nel];
      }
    }
    lAn = 0.e0;
    for (f = 0; f < nf; f++) lAn += lA[f];
    for (k = 0; k < 3; k++) lA[nf + k] = sP + sPc[k] + lAn;
    for (k = 0; k < 3; k++) lA[nf + k] = lA[nf + k] / o->under;
    for (k = 0; k < 3; k++) p[k] += (1 - o->under) * lA[nf + k] * velC[k];
    for (k = 0; k < 3; k++) p[k] -= pf[k];
    for (k = 0; k < 3; k++) rc[k] = 0.0e0;
    for (f = 0; f < nf; f++)
      if (viz[f] > -1)
        for (k = 0; k < 3; k++) {
          if (lid[f] == -2)
            p[k] += lA[f] * vel[3 * (long)viz[f] + k];
          else
            rc[k] += lA[f] * vel[3 * (long)viz[f] + k];
        }
    for (k = 0; k < 3; k++) rc[k] += p[k] - lA[nf + k] * velC[k];
    /* the momentum D field, written back in place (CellLoopInc.c, after
     * cellLibSimpleVel) */
    for (k = 0; k < 3; k++)
      dfield[3 * (long)nel + k] = o->type_simple == 2
                                      ? m->volume[nel] / (lA[nf + k] - lAn)
                                      : m->volume[nel] / lA[nf + k];
    for (f = 0; f < nf; f++) lA[f] *= -1.e0;
    for (k = 0; k < 3; k++) lB[k] = o->fres ? rc[k] : p[k];
    if (calrcell)
      for (k = 0; k < 3; k++) rcell[(long)k * numel + nel] = rc[k];
    /* csrSimple (Csr.c:1024), ndf = 3 */
    if (forces)
      for (k = 0; k < 3; k++) b[(long)k * neq + row] = lB[k];
    if (!matrix) continue;
    for (k = 0; k < 3; k++) ad[(long)k * neq + row] = lA[nf + k];
    for (f = 0; f < nf; f++) {
      const int c = lid[f];
      if (c <= -1) continue;
      if (storage == ORC_CSRC && unsym) {
        if (c < row)
          dif_put(ia, ja, row, c, a, lA[f]);
        else if (c > row)
          dif_put(ia, ja, c, row, a + nad, lA[f]);
      } else {
        dif_put(ia, ja, row, c, a, lA[f]);
      }
    }
  }
  return 0;
}

int orc_vel_assemble(const orc_dif_mesh *m, const short *facepresr, const double *cc,
                     const double *xm, const orc_load *lvel, int nlvel,
                     const orc_vel_opts *o, const double *prop, const double *pres,
                     const double *gradpres, const double *vel, const double *gradvel,
                     double *dfield, int storage, int unsym, int neq, int nad,
                     const int *ia, const int *ja, double *a, double *ad, double *b,
                     double *rcell, int forces, int matrix, int calrcell)
{
  double *dsnap = NULL;
  int rc, i;
  if (o->rhie == 1) { /* the D field every face velocity reads: the call's start */
    dsnap = (double *)malloc(sizeof(double) * 3 * (size_t)(m->numel > 0 ? m->numel : 1));
    if (!dsnap) return -1;
    for (i = 0; i < 3 * m->numel; i++) dsnap[i] = dfield[i];
  }
  rc = vel_assemble(m, facepresr, cc, xm, lvel, nlvel, o, prop, pres, gradpres, vel, gradvel,
                    dfield, storage, unsym, neq, nad, ia, ja, a, ad, b, rcell, forces, matrix,
                    calrcell, dsnap);
  free(dsnap);
  return rc;
}

/* ---- the MPI path (test infrastructure) ------------------------------- */

typedef struct {
  int nranks;
  const orc_rank *rk;
  double **xb;   /* per rank: nRcvs + nSends */
  int **peer;    /* per rank and neighbour n: the neighbour's index of this rank */
} orc_comm;

static int comm_init(orc_comm *c, int nranks, const orc_rank *rk)
{
  int r, n, m;
  c->nranks = nranks;
  c->rk = rk;
  c->xb = calloc((size_t)nranks, sizeof(double *));
  c->peer = calloc((size_t)nranks, sizeof(int *));
  if (!c->xb || !c->peer) return -1;
  for (r = 0; r < nranks; r++) {
    const orc_rank *q = &rk[r];
    c->xb[r] = malloc(sizeof(double) * (size_t)(q->nRcvs + q->nSends + 1));
    c->peer[r] = malloc(sizeof(int) * (size_t)(q->nVizPart + 1));
    if (!c->xb[r] || !c->peer[r]) return -1;
    for (n = 0; n < q->nVizPart; n++) {
      const int p = q->vizPart[n];
      const orc_rank *o;
      if (p < 0 || p >= nranks) return -1;
      o = &rk[p];
      c->peer[r][n] = -1;
      for (m = 0; m < o->nVizPart; m++)
        if (o->vizPart[m] == r) c->peer[r][n] = m;
      if (c->peer[r][n] < 0) {
        if (q->iaRcvs[n + 1] != q->iaRcvs[n]) return -1;
      } else if (o->iaSends[c->peer[r][n] + 1] - o->iaSends[c->peer[r][n]] !=
                 q->iaRcvs[n + 1] - q->iaRcvs[n]) {
        return -1;
      }
    }
  }
  return 0;
}

static void comm_free(orc_comm *c)
{
  int r;
  for (r = 0; r < c->nranks; r++) {
    if (c->xb) free(c->xb[r]);
    if (c->peer) free(c->peer[r]);
  }
  free(c->xb);
  free(c->peer);
}

/* comunicateNeq (ParallelMpi.c:3346-3418) on every rank: makeBuffer, the
 * sends and receives, getBuffer */
static void comunicate(const orc_comm *c, double *const *v)
{
  int r, n, i;
  for (r = 0; r < c->nranks; r++) {
    const orc_rank *q = &c->rk[r];
    for (i = 0; i < q->nSends; i++)
      c->xb[r][q->nRcvs + i] = v[r][q->fMap[q->nRcvs + i]];
  }
  for (r = 0; r < c->nranks; r++) {
    const orc_rank *q = &c->rk[r];
    for (n = 0; n < q->nVizPart; n++) {
      const int p = q->vizPart[n], m = c->peer[r][n];
      if (m < 0) continue;
      for (i = 0; i < q->iaRcvs[n + 1] - q->iaRcvs[n]; i++)
        c->xb[r][q->iaRcvs[n] + i] = c->xb[p][c->rk[p].iaSends[m] + i];
    }
  }
  for (r = 0; r < c->nranks; r++) {
    const orc_rank *q = &c->rk[r];
    for (i = 0; i < q->nRcvs; i++) v[r][q->fMap[i]] = c->xb[r][i];
  }
}

/* The storage's MPI product of every rank, after comunicateNeq */
static void mpi_matvec(const orc_comm *c, double *const *x, double *const *y)
{
  int r, i, k;
  comunicate(c, x);
  for (r = 0; r < c->nranks; r++) {
    const orc_rank *q = &c->rk[r];
    const double *xr = x[r];
    double *yr = y[r];
    const int split = (q->storage == 3 || q->storage == 6) && q->unsym;
    if (q->storage == 4) {
      /* mpiMatVecEllPack: ia[0] slots a row, row-major (MAT2D) */
      const int w = q->ia[0];
      for (i = 0; i < q->nEqNov; i++) {
        double ti = q->ad[i] * xr[i];
        for (k = 0; k < w; k++) ti += q->al[i * w + k] * xr[q->ja[i * w + k]];
        yr[i] = ti;
      }
    } else if (q->storage == 5 || q->storage == 6) {
      /* mpiMatVecCsrDcooSym / mpiMatVecCsrCcoo: the square part with the
       * mirrored scatter, then the ghost terms in COO order */
      const double *au = split ? q->al + q->nAd : q->al;
      const int *iar = q->ia + 2 * (q->nEqNov + 1), *jar = q->ja + q->nAd;
      const double *ar = q->al + (split ? 2 * q->nAd : q->nAd);
      for (i = 0; i < q->nEqNov; i++) {
        const double xi = xr[i];
        double tmp = q->ad[i] * xi;
        for (k = q->ia[i]; k < q->ia[i + 1]; k++) {
          const int j = q->ja[k];
          tmp += q->al[k] * xr[j];
          yr[j] += au[k] * xi;
        }
        yr[i] = tmp;
      }
      for (k = 0; k < q->nAdR; k++) yr[iar[k]] += ar[k] * xr[jar[k]];
    } else if (q->unsym && q->storage != 3) {
      for (i = 0; i < q->nEqNov; i++) {
        double tmp = q->ad[i] * xr[i];
        for (k = q->ia[i]; k < q->ia[i + 1]; k++) tmp += q->al[k] * xr[q->ja[k]];
        yr[i] = tmp;
      }
    } else {
      /* mpiMatVecCsrDSym, or mpiMatVecCsrC (au = al + nAd) */
      const int *iar = q->ia + q->nEqNov + 1, *jar = q->ja + q->nAd;
      const double *au = split ? q->al + q->nAd : q->al;
      const double *ar = q->al + (split ? 2 * q->nAd : q->nAd);
      for (i = 0; i < q->nEqNov; i++) {
        const double xi = xr[i];
        double tmp = q->ad[i] * xi;
        for (k = q->ia[i]; k < q->ia[i + 1]; k++) {
          const int j = q->ja[k];
          tmp += q->al[k] * xr[j];
          yr[j] += au[k] * xi;
        }
        for (k = iar[i]; k < iar[i + 1]; k++) tmp += ar[k] * xr[jar[k]];
        yr[i] = tmp;
      }
    }
  }
}

/* dot under MPI: each rank's sum, then the sum over the ranks in rank order */
static double mpi_dot(const orc_comm *c, double *const *a, double *const *b)
{
  double t = 0.0;
  int r;
  for (r = 0; r < c->nranks; r++) {
    const double l = orc_dot(a[r], b[r], c->rk[r].nEqNov);
    t = r == 0 ? l : t + l;
  }
  return t;
}

int orc_mpi_solve(int solver, int nranks, const orc_rank *rk, const double *const *b,
                  double *const *x, double tol, unsigned maxit, int newx, orc_stats *st)
{
  enum { NV = 8 };
  orc_comm c = {0, 0, 0, 0};
  double **w[NV];
  double alpha, beta, d, di, conv, rr0, om;
  unsigned j = 0;
  int q, i, k, rc = 0;
  if (nranks <= 0 || (solver != 1 && solver != 2)) return -1;
  for (k = 0; k < NV; k++) {
    w[k] = calloc((size_t)nranks, sizeof(double *));
    if (!w[k]) return -1;
  }
  if (comm_init(&c, nranks, rk) != 0) { rc = -1; goto done; }
  for (k = 0; k < NV; k++)
    for (q = 0; q < nranks; q++) {
      w[k][q] = calloc((size_t)rk[q].nEq + 1, sizeof(double));
      if (!w[k][q]) { rc = -1; goto done; }
    }
  {
    double **m = w[0], **z = w[1], **r = w[2], **p = w[3], **t = w[4], **v = w[5],
           **r0 = w[6], **bb = w[7];
    for (q = 0; q < nranks; q++) {
      for (i = 0; i < rk[q].nEqNov; i++) {
        m[q][i] = 1.0 / rk[q].ad[i];
        bb[q][i] = b[q][i];
      }
      if (newx)
        for (i = 0; i < rk[q].nEq; i++) x[q][i] = 0.0;
    }
    if (solver == 1) {
      /* mpiPcg, Cg.c:283-366 */
      for (q = 0; q < nranks; q++)
        for (i = 0; i < rk[q].nEqNov; i++) z[q][i] = bb[q][i] * m[q][i];
      d = mpi_dot(&c, bb, z);
      conv = tol * sqrt(fabs(d));
      mpi_matvec(&c, x, z);
      for (q = 0; q < nranks; q++)
        for (i = 0; i < rk[q].nEqNov; i++) {
          r[q][i] = bb[q][i] - z[q][i];
          z[q][i] = r[q][i] * m[q][i];
          p[q][i] = z[q][i];
        }
      d = mpi_dot(&c, r, z);
      for (j = 0; j < maxit; j++) {
        mpi_matvec(&c, p, z);
        alpha = d / mpi_dot(&c, z, p);
        for (q = 0; q < nranks; q++)
          for (i = 0; i < rk[q].nEqNov; i++) {
            x[q][i] += alpha * p[q][i];
            r[q][i] -= alpha * z[q][i];
            z[q][i] = r[q][i] * m[q][i];
          }
        di = mpi_dot(&c, r, z);
        beta = di / d;
        for (q = 0; q < nranks; q++)
          for (i = 0; i < rk[q].nEqNov; i++) p[q][i] = z[q][i] + beta * p[q][i];
        d = di;
        if (sqrt(fabs(d)) < conv) break;
      }
    } else {
      /* mpiPbicgstab, Bicgstab.c:325-437 */
      d = mpi_dot(&c, bb, bb);
      conv = tol * sqrt(d);
      mpi_matvec(&c, x, z);
      for (q = 0; q < nranks; q++)
        for (i = 0; i < rk[q].nEqNov; i++) {
          r0[q][i] = bb[q][i] - z[q][i];
          p[q][i] = r0[q][i];
          r[q][i] = r0[q][i];
          z[q][i] = p[q][i] * m[q][i];
        }
      for (j = 0; j < maxit; j++) {
        mpi_matvec(&c, z, v);
        rr0 = mpi_dot(&c, r, r0);
        alpha = rr0 / mpi_dot(&c, v, r0);
        for (q = 0; q < nranks; q++)
          for (i = 0; i < rk[q].nEqNov; i++) {
            x[q][i] += alpha * z[q][i];
            r[q][i] -= alpha * v[q][i];
            z[q][i] = r[q][i] * m[q][i];
          }
        d = mpi_dot(&c, r, r);
        if (sqrt(d) < conv) break;
        mpi_matvec(&c, z, t);
        om = mpi_dot(&c, t, r) / mpi_dot(&c, t, t);
        for (q = 0; q < nranks; q++)
          for (i = 0; i < rk[q].nEqNov; i++) {
            x[q][i] += om * z[q][i];
            r[q][i] -= om * t[q][i];
          }
        d = mpi_dot(&c, r, r);
        if (sqrt(fabs(d)) < conv) break;
        beta = (mpi_dot(&c, r, r0) / rr0) * (alpha / om);
        for (q = 0; q < nranks; q++)
          for (i = 0; i < rk[q].nEqNov; i++) {
            p[q][i] = r[q][i] + beta * (p[q][i] - om * v[q][i]);
            z[q][i] = p[q][i] * m[q][i];
          }
      }
    }
    /* post-processing, Cg.c:376-396 / Bicgstab.c:440-455 */
    mpi_matvec(&c, x, z);
    st->xKx = mpi_dot(&c, x, z);
    st->norm_x = sqrt(mpi_dot(&c, x, x));
    for (q = 0; q < nranks; q++)
      for (i = 0; i < rk[q].nEqNov; i++) {
        r[q][i] = bb[q][i] - z[q][i];
        z[q][i] = r[q][i] * m[q][i];
      }
    st->norm_r_m = solver == 1 ? sqrt(fabs(mpi_dot(&c, r, z))) : NAN;
    st->norm_r = sqrt(mpi_dot(&c, r, r));
    st->conv = conv;
    st->iters = (int)j + 1;
    st->status = j == maxit ? 1 : 0;
    rc = st->status;
  }
done:
  for (k = 0; k < NV; k++) {
    if (w[k])
      for (q = 0; q < nranks; q++) free(w[k][q]);
    free(w[k]);
  }
  comm_free(&c);
  return rc;
}

/* ======================================================================
 * Gradient reconstruction: rcGradU (CellLoop.c:4544-4790) with
 * greenGaussCell (CellLib.c:2481-2780) or leastSquare (CellLib.c:2931-3215)
 * and the least-squares matrices of rcLeastSquare / leastSquareMatrix
 * (CellLoop.c:4830-4880, CellLib.c:3500-3590); ndm = 3.
 * ====================================================================== */

enum {
  GR_DIRICHLET = 1, GR_NEUMANN = 2, GR_ROBIN = 3, GR_SINBC = 4, GR_INLET = 6, GR_OUTLET = 7,
  GR_MOVEWALL = 8, GR_INLETSTATIC = 9, GR_OPEN = 10, GR_CONVECTIONHEAT = 11,
  GR_STATICWALL = 14, GR_FLUXPRES = 15, GR_FLUXPRESC = 16
};

/* the ch-signed ksi and |ksi| of a cell's faces */
static void cell_ksi(const orc_dif_mesh *m, int nel, int nf, double ksi[][3], double *mk)
{
  int f, j;
  for (f = 0; f < nf; f++) {
    const long q = (long)nel * m->maxviz + f;
    const int face = m->cellface[q] - 1;
    const double ch = (m->owner[2 * face] - 1 == nel) ? 1.0 : -1.0;
    mk[f] = m->mksi[face];
    for (j = 0; j < 3; j++) ksi[f][j] = ch * m->ksi[3 * face + j];
  }
}

void orc_ls_matrix(const orc_dif_mesh *m, double *lsq)
{
  const int mv = m->maxviz;
  int nel, f;
  for (nel = 0; nel < m->numel; nel++) {
    double ksi[32][3], mk[32], dx[32][3], w[32], a[6] = {0, 0, 0, 0, 0, 0}, inv[6], det;
    const int nf = m->nface[nel];
    cell_ksi(m, nel, nf, ksi, mk);
    for (f = 0; f < nf; f++) {
      w[f] = 1.e0 / pow(mk[f], 2);
      dx[f][0] = ksi[f][0] * mk[f];
      dx[f][1] = ksi[f][1] * mk[f];
      dx[f][2] = ksi[f][2] * mk[f];
      a[0] += w[f] * dx[f][0] * dx[f][0];
      a[1] += w[f] * dx[f][0] * dx[f][1];
      a[2] += w[f] * dx[f][0] * dx[f][2];
      a[3] += w[f] * dx[f][1] * dx[f][1];
      a[4] += w[f] * dx[f][1] * dx[f][2];
      a[5] += w[f] * dx[f][2] * dx[f][2];
    }
    det = a[0] * a[3] * a[5] + 2.e0 * a[1] * a[4] * a[2] -
          (a[2] * a[2] * a[3] + a[4] * a[4] * a[0] + a[1] * a[1] * a[5]);
    det = 1.e0 / det;
    inv[0] = (a[3] * a[5] - a[4] * a[4]) * det;
    inv[1] = -(a[1] * a[5] - a[2] * a[4]) * det;
    inv[2] = (a[1] * a[4] - a[2] * a[3]) * det;
    inv[3] = (a[0] * a[5] - a[2] * a[2]) * det;
    inv[4] = -(a[0] * a[4] - a[1] * a[2]) * det;
    inv[5] = (a[0] * a[3] - a[1] * a[1]) * det;
    for (f = 0; f < nf; f++) {
      double *l = lsq + (long)nel * 3 * mv;
      l[0 * mv + f] = w[f] * (dx[f][0] * inv[0] + dx[f][1] * inv[1] + dx[f][2] * inv[2]);
      l[1 * mv + f] = w[f] * (dx[f][0] * inv[1] + dx[f][1] * inv[3] + dx[f][2] * inv[4]);
      l[2 * mv + f] = w[f] * (dx[f][0] * inv[2] + dx[f][1] * inv[4] + dx[f][2] * inv[5]);
    }
  }
}

/* getLoads (Loads.c:122-169) for the types the gradient reads: -2 for a
 * function-valued load */
static int gr_par(const orc_load *ld, double *par)
{
  int i;
  if ((ld->type == GR_DIRICHLET || ld->type == GR_INLET) && ld->var != 0) return -2;
  for (i = 0; i < ORC_MAXLOADPAR; i++) par[i] = ld->par[i];
  return 0;
}

int orc_rc_grad(const orc_dif_mesh *m, const orc_load *loads, int nloads, int type, int ndf,
                const double *prop, const double *lsq, const double *u, double *gradu)
{
  const int mv = m->maxviz;
  int nel;
  if (type != ORC_RCGRADGAUSSC && type != ORC_RCLSQUARE) return -1;
  if (ndf != 1 && ndf != 3) return -1;
  if (mv < 1 || mv > 31) return -1;
  for (nel = 0; nel < m->numel; nel++) {
    const int nf = m->nface[nel];
    const short *fr = m->facer + (long)nel * (mv + 1);
    const double coefdif = prop[(m->mat[nel] - 1) * ORC_MAXPROP + 0];
    double *g = gradu + (long)nel * ndf * 3;
    double uC[3], par[ORC_MAXLOADPAR];
    int f, k, j, i;
    if (nf < 1 || nf > mv) return -1;
    for (k = 0; k < ndf; k++) uC[k] = u[(long)nel * ndf + k];
    for (f = 0; f < nf; f++)
      if (m->nelcon[(long)nel * mv + f] - 1 == -2 && fr[f] > 0) {
        const orc_load *ld;
        if (fr[f] > nloads) return -1;
        ld = &loads[fr[f] - 1];
        if (ld->type == GR_SINBC) return -2;
        if ((ld->type == GR_DIRICHLET || ld->type == GR_INLET) && ld->var != 0) return -2;
      }
    if (type == ORC_RCGRADGAUSSC) {
      double uf[32][3];
      const double invVol = 1.e0 / m->volume[nel];
      for (f = 0; f < nf; f++) {
        const long q = (long)nel * mv + f;
        const int viz = m->nelcon[q] - 1;
        const double *xmcc = m->xmcc + 3 * q;
        if (viz > -1) {
          const int face = m->cellface[q] - 1;
          const long q0 = (long)nel * mv;
          const int face0 = m->cellface[q0] - 1;
          double v[3], alpha, am1;
          /* interpolFace, INTPOLFACELINEAR (CellLib.c:7174-7200), called with
           * the cell's skew and xmcc arrays themselves (CellLib.c:2513, 2640), so
           * every face reads its first face's vSkew and xmcc; |ksi| is the
           * face's own */
          for (j = 0; j < 3; j++) v[j] = m->vskew[3 * face0 + j] + m->xmcc[3 * q0 + j];
          alpha = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]) / m->mksi[face];
          am1 = 1.0e0 - alpha;
          for (k = 0; k < ndf; k++) uf[f][k] = am1 * uC[k] + alpha * u[(long)viz * ndf + k];
        } else if (fr[f] > 0) {
          const orc_load *ld = &loads[fr[f] - 1];
          const int ty = ld->type;
          if (ndf == 1) {
            if (ty == GR_DIRICHLET || ty == GR_INLET) {
              gr_par(ld, par);
              uf[f][0] = par[0];
            } else if (ty == GR_FLUXPRES) {
              /* gradPbBuoyant without buoyancy: gradPb = 0 */
              uf[f][0] = uC[0] + (0.0 * xmcc[0] + 0.0 * xmcc[1] + 0.0 * xmcc[2]);
            } else if (ty == GR_FLUXPRESC) {
              uf[f][0] = uC[0];
            } else if (ty == GR_NEUMANN) {
              if (coefdif == 0.e0) return -1; /* uf left undefined */
              gr_par(ld, par);
              uf[f][0] = uC[0] + (par[0] / coefdif) * m->dcca[q];
            } else if (ty == GR_ROBIN || ty == GR_CONVECTIONHEAT) {
              uf[f][0] = uC[0];
              for (j = 0; j < 3; j++) uf[f][0] += g[j] * xmcc[j];
            } else if (ty == GR_OUTLET) {
              uf[f][0] = uC[0];
            } else {
              return -1; /* no branch sets the face value */
            }
          } else {
            int set = 0;
            if (ty == GR_DIRICHLET || ty == GR_MOVEWALL) {
              gr_par(ld, par);
              for (k = 0; k < 3; k++) uf[f][k] = par[k];
              set = 1;
            }
            /* a second chain: the reference's `if` here is not an `else if` */
            if (ty == GR_STATICWALL) {
              for (k = 0; k < 3; k++) uf[f][k] = 0.e0;
              set = 1;
            } else if (ty == GR_INLET) {
              gr_par(ld, par);
              for (k = 0; k < 3; k++) uf[f][k] = par[k];
              set = 1;
            } else if (ty == GR_NEUMANN) {
              if (coefdif == 0.e0) return -1;
              gr_par(ld, par);
              for (k = 0; k < 3; k++) uf[f][k] = uC[k] + (par[k] / coefdif) * m->dcca[q];
              set = 1;
            } else if (ty == GR_ROBIN || ty == GR_CONVECTIONHEAT) {
              return -1; /* the reference stops: not implemented */
            } else if (ty == GR_OUTLET || ty == GR_INLETSTATIC || ty == GR_OPEN) {
              for (k = 0; k < 3; k++) uf[f][k] = uC[k];
              set = 1;
            }
            if (!set) return -1;
          }
        } else {
          for (k = 0; k < ndf; k++) {
            uf[f][k] = uC[k];
            for (j = 0; j < 3; j++) uf[f][k] += g[3 * k + j] * xmcc[j];
          }
        }
      }
      for (k = 0; k < ndf; k++)
        for (j = 0; j < 3; j++) {
          double tmp = 0.e0;
          for (f = 0; f < nf; f++) {
            const int face = m->cellface[(long)nel * mv + f] - 1;
            const double ch = (m->owner[2 * face] - 1 == nel) ? 1.0 : -1.0;
            tmp += uf[f][k] * m->area[face] * (ch * m->normal[3 * face + j]);
          }
          g[3 * k + j] = tmp * invVol;
        }
    } else {
      const double *l = lsq + (long)nel * 3 * mv;
      double du[32][3];
      int it = 1, pass;
      for (i = 0; i < ndf * 3; i++) g[i] = 0.e0;
      for (pass = 0; pass < it; pass++) {
        for (f = 0; f < nf; f++) {
          const long q = (long)nel * mv + f;
          const int viz = m->nelcon[q] - 1;
          const double *xmcc = m->xmcc + 3 * q;
          for (k = 0; k < ndf; k++) du[f][k] = 0.e0;
          if (viz > -1) {
            for (k = 0; k < ndf; k++) du[f][k] = u[(long)viz * ndf + k] - uC[k];
          } else if (fr[f] > 0) {
            const orc_load *ld = &loads[fr[f] - 1];
            const int ty = ld->type;
            if (ndf == 1) {
              if (ty == GR_DIRICHLET || ty == GR_MOVEWALL || ty == GR_INLET) {
                gr_par(ld, par);
                du[f][0] = par[0] - uC[0];
              } else if (ty == GR_FLUXPRES) {
                du[f][0] = 0.0 * xmcc[0] + 0.0 * xmcc[1] + 0.0 * xmcc[2];
              } else if (ty == GR_NEUMANN) {
                if (coefdif != 0.e0) {
                  gr_par(ld, par);
                  du[f][0] = (par[0] / coefdif) * m->dcca[q];
                }
              } else if (ty == GR_ROBIN || ty == GR_CONVECTIONHEAT) {
                if (pass == 0) it = 2;
                du[f][0] = 0.e0;
                for (j = 0; j < 3; j++) du[f][0] += g[j] * xmcc[j];
              }
              /* FLUXPRESC, OUTLET, INLETSTAICTPRES, OPEN and the rest: 0 */
            } else {
              if (ty == GR_DIRICHLET || ty == GR_MOVEWALL) {
                gr_par(ld, par);
                for (k = 0; k < 3; k++) du[f][k] = par[k] - uC[k];
              } else if (fr[f] == GR_STATICWALL) {
                /* the reference compares the load's index, not its type,
                 * with STATICWALL (CellLib.c:3118) */
                for (k = 0; k < 3; k++) du[f][k] = -uC[k];
              } else if (ty == GR_INLET) {
                gr_par(ld, par);
                for (k = 0; k < 3; k++) du[f][k] = par[k] - uC[k];
              } else if (ty == GR_ROBIN || ty == GR_CONVECTIONHEAT) {
                return -1; /* the reference stops: not implemented */
              }
              /* the rest: 0 */
            }
          } else {
            if (pass == 0) it = 2;
            for (k = 0; k < ndf; k++) {
              du[f][k] = 0.e0;
              for (j = 0; j < 3; j++) du[f][k] += g[3 * k + j] * xmcc[j];
            }
          }
        }
        for (k = 0; k < ndf; k++)
          for (i = 0; i < 3; i++) {
            double tmp = 0.e0;
            for (f = 0; f < nf; f++) tmp += l[i * mv + f] * du[f][k];
            g[3 * k + i] = tmp;
          }
      }
    }
  }
  return 0;
}
