/*
 * Test infrastructure: runs the reference's own program (its main, compiled
 * as sfr3d_ref_main) on a case deck with solverC wrapped at link time.  Each
 * system the program hands solverC is written to <prefix><n>.bin together
 * with the solution the reference's own solver returns, and after
 * SFR_HARVEST_CALLS calls (default 4) the program stops.  Used only by
 * tests/golden/make_cavity_golden.py to harvest real SIMPLE systems.
 *
 * File layout (little endian): int32 neq, nad, storage, solver, unsym,
 * newx, maxit; float64 tol; char name[32]; int32 ia[neq+1], ja[nad];
 * float64 al[nad], au[nad] (al[nad..2 nad) for unsym CSRC, else zeros),
 * ad[neq], b[neq],
 * x0[neq], x[neq].
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <Solv.h>

int sfr3d_ref_main(int argc, char **argv);

void __real_solverC(Memoria *m, INT const nEq, INT const nEqNov, INT const nAd,
                    INT const nAdR, INT *ia, INT *ja, DOUBLE *al, DOUBLE *ad,
                    DOUBLE *au, DOUBLE *b, DOUBLE *x, Interface *iNeq,
                    BufferOmp *bOmp, DOUBLE const tol, unsigned int maxIt,
                    short const storage, short const solver, FILE *fSolvLog,
                    bool const fLog, bool const newX, bool const unSym,
                    const char *name);

static int g_calls = 0, g_limit = 4;
static const char *g_prefix = "system";

static void put(FILE *f, const void *p, size_t sz, size_t n)
{
  if (n && fwrite(p, sz, n, f) != n) {
    fprintf(stderr, "harvest: short write\n");
    exit(3);
  }
}

void __wrap_solverC(Memoria *m, INT const nEq, INT const nEqNov, INT const nAd,
                    INT const nAdR, INT *ia, INT *ja, DOUBLE *al, DOUBLE *ad,
                    DOUBLE *au, DOUBLE *b, DOUBLE *x, Interface *iNeq,
                    BufferOmp *bOmp, DOUBLE const tol, unsigned int maxIt,
                    short const storage, short const solver, FILE *fSolvLog,
                    bool const fLog, bool const newX, bool const unSym,
                    const char *name)
{
  char path[512], nm[32];
  int32_t hdr[7];
  double t = tol;
  double *x0 = malloc(sizeof(double) * (size_t)nEq);
  double *zero = calloc((size_t)(nAd > 0 ? nAd : 1), sizeof(double));
  FILE *f;
  int i;
  memcpy(x0, x, sizeof(double) * (size_t)nEq);
  __real_solverC(m, nEq, nEqNov, nAd, nAdR, ia, ja, al, ad, au, b, x, iNeq, bOmp,
                 tol, maxIt, storage, solver, fSolvLog, fLog, newX, unSym, name);
  snprintf(path, sizeof(path), "%s%d.bin", g_prefix, g_calls);
  f = fopen(path, "wb");
  if (!f) exit(3);
  hdr[0] = nEq; hdr[1] = nAd; hdr[2] = storage; hdr[3] = solver;
  hdr[4] = unSym; hdr[5] = newX; hdr[6] = (int32_t)maxIt;
  memset(nm, 0, sizeof(nm));
  strncpy(nm, name ? name : "", sizeof(nm) - 1);
  put(f, hdr, sizeof(int32_t), 7);
  put(f, &t, sizeof(double), 1);
  put(f, nm, 1, sizeof(nm));
  put(f, ia, sizeof(INT), (size_t)nEq + 1);
  put(f, ja, sizeof(INT), (size_t)nAd);
  put(f, al, sizeof(double), (size_t)nAd);
  /* unsym CSRC: the upper part follows al (matVecCsrC, HccaBlas.c:4233-4236) */
  put(f, (unSym && storage == CSRC) ? al + nAd : zero, sizeof(double), (size_t)nAd);
  put(f, ad, sizeof(double), (size_t)nEq);
  put(f, b, sizeof(double), (size_t)nEq);
  put(f, newX ? zero : x0, sizeof(double), newX ? 0 : (size_t)nEq);
  if (newX)
    for (i = 0; i < nEq; i++) put(f, &zero[0], sizeof(double), 1);
  put(f, x, sizeof(double), (size_t)nEq);
  fclose(f);
  free(x0);
  free(zero);
  if (++g_calls >= g_limit) {
    fflush(NULL);
    exit(0);
  }
}

int main(int argc, char **argv)
{
  const char *lim = getenv("SFR_HARVEST_CALLS");
  const char *pre = getenv("SFR_HARVEST_PREFIX");
  if (lim) g_limit = atoi(lim);
  if (pre) g_prefix = pre;
  return sfr3d_ref_main(argc, argv);
}
