/*
 * Test infrastructure, not product code: a plain-C restatement of SFR3D's
 * linear-solve path (PCG, BiCGSTAB, and the other Krylov methods behind
 * solverC: BiCGSTAB(2), GMRES, MINRES) used as the parity oracle.  Only tests/, the smoke check
 * and bench.py's CPU-baseline leg load it.  Every function cites the
 * reference lines it restates; the arithmetic is done in the same order as
 * the reference so that results are bit-identical to the reference's own
 * compiled solver (checked by tests/test_oracle.py against oracle/_ref).
 */
#ifndef SFR3D_ORACLE_H
#define SFR3D_ORACLE_H

/* storage codes, Define.h:407-410 */
#define ORC_CSRD 2
#define ORC_CSRC 3
#define ORC_ELLPACK 4

typedef struct {
  int iters;        /* j+1 as the reference reports it */
  int status;       /* 0 converged, 1 reached maxIt (the reference exits) */
  double xKx;       /* x^T A x */
  double norm_x;    /* ||x||_2 */
  double norm_r;    /* ||b - A x||_2 */
  double norm_r_m;  /* ||b - A x||_M (PCG only) */
  double conv;      /* tol * norm of b used by the stopping test */
} orc_stats;

/* y = A x for the storage/unsym pair solverC would see (setMatVec,
 * Solv.c:732-919).  For ELLPACK, ia[0] is the row width (EllPack.c:35). */
void orc_matvec(int storage, int unsym, int neq, const int *ia, const int *ja,
                const double *al, const double *ad, const double *x,
                double *y);

double orc_dot(const double *a, const double *b, int n);

/* 0: the reference's left-to-right dot (default); 1: right to left;
 * 2: pairwise.  Only for measuring the reference's sensitivity to the
 * summation order. */
void orc_set_dot_order(int order);

int orc_pcg(int storage, int unsym, int neq, const int *ia, const int *ja,
            const double *al, const double *ad, const double *b, double *x,
            double tol, unsigned maxit, int newx, orc_stats *st);

int orc_pbicgstab(int storage, int unsym, int neq, const int *ia,
                  const int *ja, const double *al, const double *ad,
                  const double *b, double *x, double tol, unsigned maxit,
                  int newx, orc_stats *st);

/* Iters.c:309-558 (pminres) */
int orc_minres(int storage, int unsym, int neq, const int *ia, const int *ja,
               const double *al, const double *ad, const double *b, double *x,
               double tol, unsigned maxit, int newx, orc_stats *st);

/* Bicgstab.c:1172-1460 (pbicgstabl2) */
int orc_pbicgstabl2(int storage, int unsym, int neq, const int *ia,
                    const int *ja, const double *al, const double *ad,
                    const double *b, double *x, double tol, unsigned maxit,
                    int newx, orc_stats *st);

/* Iters.c:587-800 (gmres), nk Krylov vectors a cycle (solverC: 15),
 * maxit cycles */
int orc_gmres(int storage, int unsym, int neq, const int *ia, const int *ja,
              const double *al, const double *ad, const double *b, double *x,
              double tol, unsigned maxit, int newx, int nk, orc_stats *st);

#endif
