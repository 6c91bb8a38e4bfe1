/*
 * Test infrastructure: a thin harness around the reference's OWN compiled
 * solver (oracle/_ref/libsfr3d_ref.so).  Only tests/, the smoke check and
 * bench.py's CPU-baseline leg load it, and only as the checker or the timed
 * CPU arm -- never as the product path.
 *
 * It calls the reference's solverC (Solv.c:64-501) exactly as the SIMPLE and
 * diffusion drivers do (Simple.c:2983, Diffusion.c:145), with a Memoria arena
 * (Memoria.c:21 initMem) for its workspace and, for the OpenMP path, the
 * BufferOmp that pMatrixSolverOmp builds (HccaOpenMp.c:24-40 ->
 * partitionCsrByNonzeros, Csr.c:1827).  The iteration count, xKx and ||x||
 * are read back from the one log line the solver writes (Cg.c:201-208,
 * Bicgstab.c:235-242).  exit() is wrapped at link time so that the
 * reference's fatal non-convergence path (Cg.c:195-200, Bicgstab.c:225-231)
 * returns here with its exit code.
 */
#define _GNU_SOURCE
#include <setjmp.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <omp.h>

#include <Solv.h>
#include <CellLoop.h>
#include <Coo.h>

extern Omp ompVar;
extern Mpi mpiVar;
extern FILE *fileLogExc, *fileLogDebug;
extern iptx nmax; /* arena capacity that alloc() checks (Memoria.c:97-160) */
void partitionCsrByNonzeros(INT *ia, INT *ja, INT const neq, int nThreads,
                            INT *thBegin, INT *thEnd, INT *thSize,
                            INT *thHeight, short type);

void __real_exit(int code);

static jmp_buf g_jump;
static volatile int g_armed = 0;
static volatile int g_exit_code = 0;
static volatile double g_t0 = 0.0;

void __wrap_exit(int code)
{
  if (g_armed) {
    g_armed = 0;
    g_exit_code = code;
    longjmp(g_jump, 1);
  }
  __real_exit(code);
}

static void parse_log(const char *buf, int *iters, double *xKx, double *normx)
{
  const char *s;
  if ((s = strstr(buf, "iteration ")) != NULL) sscanf(s + 10, "%d", iters);
  if ((s = strstr(buf, "xKx ")) != NULL) sscanf(s + 4, "%le", xKx);
  if ((s = strstr(buf, "norma(x*x) ")) != NULL) sscanf(s + 11, "%le", normx);
  else if ((s = strstr(buf, "||x*x|| ")) != NULL) sscanf(s + 8, "%le", normx);
}

/*
 * Solve one system with the reference's solverC.
 *   solver : PCG=1 | PBICGSTAB=2 | PBICGSTABL2=3 | GMRES=4 | MINRES=5
 *            (Define.h:392-396)
 *   storage: CSRD=2 | CSRC=3 | ELLPACK=4 (Define.h:407-410)
 *   nthreads: 0 -> serial pcg/pbicgstab, >=1 -> pcgOmp/pbicgstabOmp
 * Returns 0 when the solver converged, otherwise the code it passed to
 * exit().  x is updated in place (newX != 0 zeroes it first).
 */
int sfr_ref_solve(int neq, int nad, int *ia, int *ja, double *al, double *ad,
                  double *au, double *b, double *x, double tol,
                  unsigned maxit, int storage, int solver, int newX,
                  int unsym, int nthreads, int *iters, double *xKx,
                  double *normx, double *seconds)
{
  Memoria mem;
  BufferOmp omp;
  char *logbuf = NULL;
  size_t loglen = 0;
  FILE *flog;
  double t0;
  int rc = 0, nvec;

  memset(&omp, 0, sizeof(omp));
  fileLogExc = stderr;
  fileLogDebug = stderr;
  mpiVar.nPrcs = 1;
  mpiVar.myId = 0;
  ompVar.fSolver = nthreads > 0;
  ompVar.nThreadsSolver = (unsigned short)(nthreads > 0 ? nthreads : 1);

  /* workspace: pc + the Krylov vectors (GMRES(15): 16 basis vectors; the
   * others: 10 at most), plus the arena's alignment */
  nvec = solver == 4 ? 20 : 12;
  nmax = (iptx)nvec * (iptx)(neq + 64) * (iptx)sizeof(double) + 65536;
  initMem(&mem, nmax, false);
  /* dalloc (Memoria.c:280) refuses to release the only vector of an arena;
   * in the application the mesh always sits below the solver workspace */
  {
    DOUBLE *base = NULL;
    HccaAlloc(DOUBLE, &mem, base, 8, "harness_base", false);
    (void)base;
  }

  flog = open_memstream(&logbuf, &loglen);
  *iters = -1;
  *xKx = 0.0;
  *normx = 0.0;
  *seconds = 0.0;

  g_t0 = 0.0;
  if (setjmp(g_jump) == 0) {
    g_armed = 1;
    if (nthreads > 0) {
      omp_set_num_threads(nthreads);
      omp.thBegin = calloc(nthreads, sizeof(INT));
      omp.thEnd = calloc(nthreads, sizeof(INT));
      omp.thSize = calloc(nthreads, sizeof(INT));
      omp.thHeight = calloc(nthreads, sizeof(INT));
      omp.thY = calloc((size_t)nthreads * (size_t)neq, sizeof(double));
      partitionCsrByNonzeros(ia, ja, neq, nthreads, omp.thBegin, omp.thEnd,
                             omp.thSize, omp.thHeight, (short)storage);
    }
    t0 = omp_get_wtime();
    g_t0 = t0;
    solverC(&mem, neq, neq, nad, 0, ia, ja, al, ad, au, b, x, NULL,
            nthreads > 0 ? &omp : NULL, tol, maxit, (short)storage,
            (short)solver, flog, true, newX != 0, unsym != 0, "oracle");
    *seconds = omp_get_wtime() - t0;
    g_armed = 0;
    rc = 0;
  } else {
    rc = g_exit_code == 0 ? -1000 : g_exit_code;
    *iters = (int)maxit;
    /* the solve ran to maxIt before exiting: its wall time is still valid */
    if (g_t0 > 0.0) *seconds = omp_get_wtime() - g_t0;
  }
  fclose(flog);
  if (rc == 0 && logbuf) parse_log(logbuf, iters, xKx, normx);
  free(logbuf);
  free(omp.thBegin);
  free(omp.thEnd);
  free(omp.thSize);
  free(omp.thHeight);
  free(omp.thY);
  finalizeMem(&mem, false);
  return rc;
}

/* Machine epsilon as the reference computes it for tol = 0 (Solv.c:614). */
double sfr_ref_smachn(void) { return smachn(); }

int sfr_ref_max_threads(void) { return omp_get_max_threads(); }

/*
 * Assemble the diffusion system with the reference's own systFormDif
 * (CellLoop.c:285-455) as diffusion() calls it (Diffusion.c:80-106), ndf = 1,
 * ndm = 3, one process.  Loads are given as parallel arrays (type, nTypeVar,
 * np, par[20] each); the scheme, residual form and time term as scalars.
 * Arrays the assembly does not read (the node incidence, node counts,
 * geometry types, face centres, eta, |vSkew|) are still passed through.
 * Returns the exit code when the reference exits (an unknown scheme).
 */
int sfr_ref_syst_form_dif(int numel, int maxviz, int *nelcon, short *nface,
                          int *cellface, int *owner, double *volume,
                          double *dcca, double *xmcc, double *mksi,
                          double *ksi, double *eta, double *area,
                          double *normal, double *xm, double *mvskew,
                          double *vskew, short *caltype, short *mat,
                          double *density, double *cdiff, int *ia, int *ja,
                          double *a, double *ad, double *b, int *id,
                          short *facer, double *u0, double *gradu0,
                          double *rcell, int nloads, const int *ltype,
                          const int *lvar, const int *lnp, const double *lpar,
                          int icod, int fres, int time_flag, int time_type,
                          double dt, double dt0, int neq, int nad, int storage,
                          int forces, int matrix, int calrcell, int unsym,
                          double *seconds)
{
  Loads *loads = calloc(nloads > 0 ? nloads : 1, sizeof(Loads));
  INT *el = calloc((size_t)numel * 8, sizeof(INT));
  short *nen = malloc((size_t)numel * sizeof(short));
  short *gtype = calloc((size_t)numel, sizeof(short));
  Diffusion diff;
  DiffModel dmodel;
  Temporal ddt;
  int i, j, rc = 0;
  double t0;

  fileLogExc = stderr;
  fileLogDebug = stderr;
  mpiVar.nPrcs = 1;
  mpiVar.myId = 0;
  for (i = 0; i < numel; i++) nen[i] = 8;
  for (i = 0; i < nloads; i++) {
    loads[i].fUse = true;
    loads[i].type = (short)ltype[i];
    loads[i].nTypeVar = (short)lvar[i];
    loads[i].np = (short)lnp[i];
    for (j = 0; j < MAXLOADPARAMETER; j++) loads[i].par[j] = lpar[i * MAXLOADPARAMETER + j];
  }
  memset(&diff, 0, sizeof(diff));
  memset(&dmodel, 0, sizeof(dmodel));
  memset(&ddt, 0, sizeof(ddt));
  diff.iCod = (short)icod;
  dmodel.fRes = fres != 0;
  ddt.flag = time_flag != 0;
  ddt.type = (short)time_type;
  ddt.dt[0] = dt;
  ddt.dt[1] = dt0;
  *seconds = 0.0;
  if (setjmp(g_jump) == 0) {
    g_armed = 1;
    t0 = omp_get_wtime();
    systFormDif(loads, &diff, &dmodel, el, nelcon, nen, nface, cellface, owner,
                volume, dcca, xmcc, mksi, ksi, eta, area, normal, xm, mvskew,
                vskew, gtype, caltype, mat, density, cdiff, ia, ja, a, ad, b,
                id, facer, u0, gradu0, rcell, &ddt, neq, neq, nad, 0,
                8, (short)maxviz, 3, numel, 1, (short)storage, forces != 0,
                matrix != 0, calrcell != 0, unsym != 0);
    *seconds = omp_get_wtime() - t0;
    g_armed = 0;
  } else {
    rc = g_exit_code == 0 ? -1000 : g_exit_code;
  }
  free(loads);
  free(el);
  free(nen);
  free(gtype);
  return rc;
}

static void fill_loads(Loads *dst, int n, const int *type, const int *var, const int *np,
                       const double *par, const double *density)
{
  int i, j;
  for (i = 0; i < n; i++) {
    memset(&dst[i], 0, sizeof(Loads));
    dst[i].fUse = true;
    dst[i].type = (short)type[i];
    dst[i].nTypeVar = (short)var[i];
    dst[i].np = (short)np[i];
    dst[i].density = density[i];
    for (j = 0; j < MAXLOADPARAMETER; j++) dst[i].par[j] = par[i * MAXLOADPARAMETER + j];
  }
}

/*
 * Assemble the SIMPLE pressure-correction system with the reference's own
 * systFormSimplePres (CellLoopInc.c:471-700), no wall model, as
 * velPresCoupling calls it; nthreads > 1 turns on its OpenMP cell loop.  cellSimplePres3D reads the velocity loads from
 * the global loadsVel table (CellPres.c, pLoadSimple call), so they are
 * copied there as well as passed.  Mesh arrays as for systFormDif; prop is
 * the nmat x MAXPROP material table.
 */
int sfr_ref_syst_form_simple_pres(int numel, int maxviz, int *nelcon, short *nface,
                                  int *cellface, int *owner, double *volume,
                                  double *dcca, double *xmcc, double *mksi,
                                  double *ksi, double *eta, double *area,
                                  double *normal, double *xm, double *mvskew,
                                  double *vskew, short *caltype, short *mat,
                                  double *prop, int *ia, int *ja, double *a,
                                  double *ad, double *b, int *id, short *facevelr,
                                  short *facepresr, double *pres, double *gradpres,
                                  double *vel, double *dfield, double *rcell,
                                  int nlvel, const int *vtype, const int *vvar,
                                  const int *vnp, const double *vpar,
                                  const double *vdens, int nlpres,
                                  const int *ptype, const int *pvar, const int *pnp,
                                  const double *ppar, const double *pdens, int icod,
                                  int neq, int nad, int storage, int forces,
                                  int matrix, int calrcell, int unsym,
                                  int nthreads, double *seconds)
{
  Loads *lp = calloc(nlpres > 0 ? nlpres : 1, sizeof(Loads));
  INT *el = calloc((size_t)numel * 8, sizeof(INT));
  short *nen = malloc((size_t)numel * sizeof(short));
  short *gtype = calloc((size_t)numel, sizeof(short));
  double *cc = calloc((size_t)numel * 3, sizeof(double));
  double *wallpar = calloc((size_t)numel * NWALLPAR, sizeof(double));
  Diffusion diff;
  Turbulence tmodel;
  Temporal ddt;
  int i, rc = 0;
  double t0;

  fileLogExc = stderr;
  fileLogDebug = stderr;
  mpiVar.nPrcs = 1;
  mpiVar.myId = 0;
  ompVar.fCell = nthreads > 1;
  ompVar.nThreadsCell = (short)(nthreads > 1 ? nthreads : 1);
  for (i = 0; i < numel; i++) nen[i] = 8;
  fill_loads(loadsVel, nlvel, vtype, vvar, vnp, vpar, vdens);
  fill_loads(lp, nlpres, ptype, pvar, pnp, ppar, pdens);
  memset(&diff, 0, sizeof(diff));
  memset(&tmodel, 0, sizeof(tmodel));
  memset(&ddt, 0, sizeof(ddt));
  diff.iCod = (short)icod;
  tmodel.fWall = false;
  *seconds = 0.0;
  if (setjmp(g_jump) == 0) {
    g_armed = 1;
    t0 = omp_get_wtime();
    systFormSimplePres(loadsVel, lp, &diff, &tmodel, el, nelcon, nen, nface, cellface,
                       owner, volume, dcca, xmcc, cc, mksi, ksi, eta, area, normal, xm,
                       mvskew, vskew, gtype, prop, caltype, mat, ia, ja, a, ad, b, id,
                       facevelr, facepresr, pres, gradpres, vel, dfield, wallpar, rcell,
                       &ddt, neq, neq, nad, 0, 8, (short)maxviz, 3, numel, 1,
                       (short)storage, forces != 0, matrix != 0, calrcell != 0,
                       unsym != 0);
    *seconds = omp_get_wtime() - t0;
    g_armed = 0;
  } else {
    rc = g_exit_code == 0 ? -1000 : g_exit_code;
  }
  free(lp);
  free(el);
  free(nen);
  free(gtype);
  free(cc);
  free(wallpar);
  return rc;
}

/*
 * The reference's Matrix Market dumps (WriteMtx.c, built with -D_MMIO_):
 * writeCoo (the "pcoo"/"pgraph" macros of Main.c:975-1010) for the matrix,
 * writeCooB for the force vector.  Returns the exit code when the reference
 * exits (a storage other than CSRD).
 */
int sfr_ref_write_coo(int neq, int nad, int *ia, int *ja, double *au, double *ad, double *al,
                      int storage, int unsym, int bin, const char *name)
{
  Memoria mem;
  char path[1024];
  int rc = 0;
  fileLogExc = stderr;
  fileLogDebug = stderr;
  nmax = (iptx)3 * (iptx)(neq + nad + 64) * (iptx)sizeof(double) + 65536;
  initMem(&mem, nmax, false);
  {
    DOUBLE *base = NULL;
    HccaAlloc(DOUBLE, &mem, base, 8, "harness_base", false);
    (void)base;
  }
  strncpy(path, name, sizeof(path) - 1);
  path[sizeof(path) - 1] = 0;
  if (setjmp(g_jump) == 0) {
    g_armed = 1;
    writeCoo(&mem, ia, ja, neq, au, ad, al, nad, (short)storage, unsym != 0, bin != 0, path);
    fflush(NULL);
    g_armed = 0;
  } else {
    rc = g_exit_code == 0 ? -1000 : g_exit_code;
  }
  finalizeMem(&mem, false);
  return rc;
}

void sfr_ref_write_coo_b(double *b, int neq, const char *name)
{
  char path[1024];
  strncpy(path, name, sizeof(path) - 1);
  path[sizeof(path) - 1] = 0;
  writeCooB(b, neq, path);
  fflush(NULL);  /* writeCooB leaves its file open */
}

/*
 * Assemble the SIMPLE momentum system with the reference's own
 * systFormSimpleVel (CellLoopInc.c:98-470) as velPresCoupling calls it
 * (Simple.c:2864-2898): ndf = 3, laminar (Turbulence all off), first-order
 * upwind, without Rhie-Chow; nthreads > 1 turns on its OpenMP cell loop.
 * dfield is updated in place.
 */
int sfr_ref_syst_form_simple_vel(int numel, int maxviz, int *nelcon, short *nface,
                                 int *cellface, int *owner, double *volume, double *dcca,
                                 double *xmcc, double *cc, double *mksi, double *ksi,
                                 double *eta, double *area, double *normal, double *xm,
                                 double *mvskew, double *vskew, short *caltype, short *mat,
                                 double *prop, int *ia, int *ja, double *a, double *ad,
                                 double *b, int *id, short *facevelr, short *facepresr,
                                 double *pres, double *gradpres, double *vel, double *gradvel,
                                 double *dfield, double *rcell, int nlvel, const int *vtype,
                                 const int *vvar, const int *vnp, const double *vpar,
                                 const double *vdens, int icod, int fso, int fvisc, int fres,
                                 int type_simple, int time_flag, int time_type, double dt,
                                 double dt0, double under, int neq, int nad, int storage,
                                 int forces, int matrix, int calrcell, int unsym,
                                 int nthreads, int advcod, int fturb, int fstruc,
                                 const double *eddy_in, const double *stress_in,
                                 double adv_beta, int adv_fn, int fwall,
                                 const double *wallpar_in, int rhie, double *seconds)
{
  INT *el = calloc((size_t)numel * 8, sizeof(INT));
  short *nen = malloc((size_t)numel * sizeof(short));
  short *gtype = calloc((size_t)numel, sizeof(short));
  double *stressr = calloc((size_t)numel * 6, sizeof(double));
  double *eddy = calloc((size_t)numel, sizeof(double));
  double *wallpar = calloc((size_t)numel * NWALLPAR, sizeof(double));
  Advection adv;
  Diffusion diff;
  Turbulence tmodel;
  MomentumModel mm;
  Temporal ddt;
  int i, rc = 0;
  double t0;

  fileLogExc = stderr;
  fileLogDebug = stderr;
  mpiVar.nPrcs = 1;
  mpiVar.myId = 0;
  /* its OpenMP cell loop only writes D here (Rhie-Chow is off), so threads
   * change nothing but the time */
  ompVar.fCell = nthreads > 1;
  ompVar.nThreadsCell = (short)(nthreads > 1 ? nthreads : 1);
  for (i = 0; i < numel; i++) nen[i] = 8;
  fill_loads(loadsVel, nlvel, vtype, vvar, vnp, vpar, vdens);
  memset(&adv, 0, sizeof(adv));
  memset(&diff, 0, sizeof(diff));
  memset(&tmodel, 0, sizeof(tmodel));
  memset(&mm, 0, sizeof(mm));
  memset(&ddt, 0, sizeof(ddt));
  adv.iCod1 = (short)(advcod > 0 ? advcod : FOUP);
  adv.par[0] = adv_beta;
  adv.iCod2 = (short)adv_fn;
  tmodel.fTurb = fturb != 0;
  tmodel.fTurbStruct = fstruc != 0;
  tmodel.fWall = fwall != 0;
  if (wallpar_in) memcpy(wallpar, wallpar_in, sizeof(double) * (size_t)numel * NWALLPAR);
  if (eddy_in) memcpy(eddy, eddy_in, sizeof(double) * (size_t)numel);
  if (stress_in) memcpy(stressr, stress_in, sizeof(double) * (size_t)numel * 6);
  diff.iCod = (short)icod;
  mm.fRes = fres != 0;
  mm.fRhieChowInt = rhie != 0;
  mm.fViscosity = fvisc != 0;
  mm.fSoPressure = fso != 0;
  ddt.flag = time_flag != 0;
  ddt.type = (short)time_type;
  ddt.dt[0] = dt;
  ddt.dt[1] = dt0;
  *seconds = 0.0;
  if (setjmp(g_jump) == 0) {
    g_armed = 1;
    t0 = omp_get_wtime();
    systFormSimpleVel(loadsVel, loadsPres, &adv, &diff, &tmodel, &mm, NULL, (short)type_simple,
                      el, nelcon, nen, nface, cellface, owner, volume, dcca, xmcc, cc, mksi,
                      ksi, eta, area, normal, xm, mvskew, vskew, gtype, prop, caltype, mat,
                      ia, ja, a, ad, b, id, facevelr, facepresr, pres, gradpres, vel, gradvel,
                      dfield, under, rcell, stressr, eddy, wallpar, &ddt, neq, neq, nad, 0, 8,
                      (short)maxviz, 3, numel, 3, 6, (short)storage, forces != 0,
                      matrix != 0, calrcell != 0, unsym != 0);
    *seconds = omp_get_wtime() - t0;
    g_armed = 0;
  } else {
    rc = g_exit_code == 0 ? -1000 : g_exit_code;
  }
  free(el);
  free(nen);
  free(gtype);
  free(stressr);
  free(eddy);
  free(wallpar);
  return rc;
}

/*
 * The reference's own gradient reconstruction: rcLeastSquare
 * (CellLoop.c:4830-4880) for the least-squares matrices, then rcGradU
 * (CellLoop.c:4544-4790) as the SIMPLE driver calls it for the velocity or
 * the pressure (Simple.c:2797-2858), with rcGrad {type, no limiter}, one
 * process, no density fields.  Every cell is a hexahedron (geomType only
 * picks the node table the Green-Gauss nodal variant would use).  gradu
 * (numel*ndf*3) is read as the previous gradient and overwritten; lsq
 * (numel*3*maxviz) receives the least-squares matrices when type is
 * RCLSQUARE.  nthreads > 1 turns on its OpenMP cell loop.
 */
int sfr_ref_rc_grad(int numel, int maxviz, int *nelcon, short *nface, int *cellface, int *owner,
                    double *volume, double *dcca, double *xmcc, double *cc, double *mksi,
                    double *ksi, double *eta, double *area, double *normal, double *xm,
                    double *mvskew, double *vskew, short *caltype, short *mat, double *prop,
                    short *facer, int nloads, const int *ltype, const int *lvar,
                    const int *lnp, const double *lpar, const double *ldens, int type, int ndf,
                    double *u, double *gradu, double *lsq, int nthreads, double *seconds)
{
  INT *el = calloc((size_t)numel * 8, sizeof(INT));
  short *nen = malloc((size_t)numel * sizeof(short));
  short *gtype = malloc((size_t)numel * sizeof(short));
  double *lsqr = calloc((size_t)numel * 6, sizeof(double));
  double *lsqm = calloc((size_t)numel * 3 * maxviz, sizeof(double));
  Loads *ld = calloc((size_t)(nloads > 0 ? nloads : 1), sizeof(Loads));
  RcGrad rc;
  int i, code = 0;
  double t0;

  fileLogExc = stderr;
  fileLogDebug = stderr;
  mpiVar.nPrcs = 1;
  mpiVar.myId = 0;
  ompVar.fGrad = nthreads > 1;
  ompVar.nThreadsGrad = (short)(nthreads > 1 ? nthreads : 1);
  for (i = 0; i < numel; i++) {
    nen[i] = 8;
    gtype[i] = HEXACELL;
  }
  fill_loads(ld, nloads, ltype, lvar, lnp, lpar, ldens);
  memset(&rc, 0, sizeof(rc));
  rc.type = (short)type;
  rc.fLimiter = false;
  if (type == RCLSQUARE || type == RCLSQUAREQR)
    rcLeastSquare(cellface, owner, mksi, ksi, lsqm, lsqr, nface, numel, (short)maxviz,
                  (short)type, 3);
  g_armed = 1;
  if (setjmp(g_jump) == 0) {
    t0 = omp_get_wtime();
    rcGradU(NULL, ld, el, nelcon, NULL, nen, nface, cellface, owner, volume, dcca, xmcc, cc,
            mksi, ksi, eta, area, normal, xm, mvskew, vskew, gtype, prop, caltype, mat, NULL,
            lsqm, lsqr, facer, u, gradu, NULL, NULL, NULL, 0.0, &rc, 8, (short)maxviz,
            (short)ndf, 3, NULL, NULL, numel, numel, 0, 0, false);
    if (seconds) *seconds = omp_get_wtime() - t0;
    g_armed = 0;
  } else {
    code = g_exit_code ? g_exit_code : -1;
  }
  if (lsq) memcpy(lsq, lsqm, sizeof(double) * (size_t)numel * 3 * maxviz);
  free(el);
  free(nen);
  free(gtype);
  free(lsqr);
  free(lsqm);
  free(ld);
  return code;
}
