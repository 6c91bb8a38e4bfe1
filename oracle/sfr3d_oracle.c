/*
 * Test infrastructure, not product code: plain-C restatement of SFR3D's
 * Jacobi-PCG / Jacobi-BiCGSTAB path (the parity oracle).  Compiled with
 * -ffp-contract=off so every product and sum rounds exactly where the
 * reference's (gcc -std=c99 -O3, no FMA) does.
 */
#include "sfr3d_oracle.h"

#include <math.h>
#include <stdlib.h>

/* HccaBlas.c:393-437 (dot): one accumulator, left to right. */
double orc_dot(const double *a, const double *b, int n)
{
  double s = 0.0;
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
