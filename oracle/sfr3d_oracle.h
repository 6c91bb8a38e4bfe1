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

/* ---- diffusion system assembly (systFormDif, CellLoop.c:285-455) ------ */

#define ORC_MAXLOADPAR 20 /* MAXLOADPARAMETER, Define.h:336 */

/* The mesh arrays systFormDif reads (1-based indices as the reference
 * stores them; MAT2D/MAT3D row-major). */
typedef struct {
  int numel, maxviz;
  const int *nelcon;      /* numel*maxviz: neighbour + 1, -1 boundary */
  const short *nface;     /* numel */
  const int *cellface;    /* numel*maxviz: face + 1 */
  const int *owner;       /* nface*2 */
  const double *volume;   /* numel */
  const double *dcca;     /* numel*maxviz */
  const double *xmcc;     /* numel*maxviz*3 */
  const double *mksi;     /* per face */
  const double *ksi;      /* per face *3 */
  const double *area;     /* per face */
  const double *normal;   /* per face *3 */
  const double *vskew;    /* per face *3 */
  const short *caltype;   /* per material */
  const short *mat;       /* numel, 1-based material */
  const int *id;          /* numel: equation + 1 (0: none) */
  const short *facer;     /* numel*(maxviz+1): load + 1 per face, then the cell */
} orc_dif_mesh;

/* The fields of Loads (StructDefine.h:356-366) that pLoad reads. */
typedef struct {
  int type, var, np;
  double par[ORC_MAXLOADPAR];
  double density;        /* Loads.density (OPEN inflow) */
} orc_load;

typedef struct {
  int icod;              /* Diffusion.iCod: 1 orthogonal .. 4 over-relaxed */
  int fres;              /* DiffModel.fRes */
  int time_flag;         /* Temporal.flag */
  int time_type;         /* 0 EULER, 1 BACKWARD */
  double dt, dt0;        /* Temporal.dt[0], dt[1] */
} orc_dif_opts;

/* systFormDif with ndf = 1 and ndm = 3 on one process: writes a (al, or al
 * then au for unsym CSRC; the neq x width slots for ELLPACK), ad, b and rcell
 * as csr()/ellPack() (Csr.c:549-1022, EllPack.c:113-149) would.  Returns 0,
 * -1 for input the reference cannot take (a material whose cell library is
 * not diffusion, an unknown non-orthogonal scheme, an OUTLET load, a load
 * with too few parameters), -2 for loads given as functions or SINBC. */
int orc_dif_assemble(const orc_dif_mesh *m, const orc_load *loads, int nloads,
                     const orc_dif_opts *o, const double *density,
                     const double *cdiff, const double *u0,
                     const double *gradu0, int storage, int unsym, int neq,
                     int nad, const int *ia, const int *ja, double *a,
                     double *ad, double *b, double *rcell, int forces,
                     int matrix, int calrcell);

/* ---- pressure-correction assembly (systFormSimplePres,
 *      CellLoopInc.c:471-700 -> cellSimplePres3D, CellPres.c:903-1218) ---- */

#define ORC_MAXPROP 10 /* Define.h:349 */
#define ORC_DENSITY 1  /* Define.h:203 */

/* m->facer is facePresR (pressure loads); facevelr the velocity loads
 * (faceVelR), same shape.  prop: nmat x MAXPROP material table; pres
 * (numel), gradpres, vel and dfield (numel x 3).  icod: 1 ORTHOGONAL or
 * 4 OVERRELAXED (difusionSchemeAnisotropic leaves e and t unset for the
 * other two).  Returns 0, -1 for input the reference cannot take, -2 for
 * loads given as functions. */
int orc_pres_assemble(const orc_dif_mesh *m, const short *facevelr,
                      const orc_load *lvel, int nlvel, const orc_load *lpres,
                      int nlpres, int icod, const double *prop,
                      const double *pres, const double *gradpres,
                      const double *vel, const double *dfield, int storage,
                      int unsym, int neq, int nad, const int *ia,
                      const int *ja, double *a, double *ad, double *b,
                      double *rcell, int forces, int matrix, int calrcell);

/* ---- momentum assembly (systFormSimpleVel, CellLoopInc.c:98-470 ->
 *      cellSimpleVel3D, CellSimple.c:106-727), laminar, advection FoUp, CD
 *      or SoUp, no Rhie-Chow face velocity, no wall model -------------- */
typedef struct {
  int icod;          /* Diffusion.iCod (difusionSchemeNew) */
  int fso;           /* MomentumModel.fSoPressure: second-order face pressure */
  int fvisc;         /* MomentumModel.fViscosity: explicit viscous part */
  int fres;          /* MomentumModel.fRes */
  int type_simple;   /* 1 SIMPLE, 2 SIMPLEC (Define.h:223-224) */
  int time_flag, time_type;
  int adv;           /* Advection.iCod1: 0 or 1 FoUp, 2 CD, 3 SoUp
                        (advectiveScheme, CellLib.c:6394-6480) */
  double dt, dt0;
  double under;      /* underU (alphaVel) */
  int fturb, fstruc; /* Turbulence.fTurb / fTurbStruct */
  const double *eddy;   /* numel eddy viscosity (fturb) */
  const double *stress; /* numel*6 residual stress xx yy zz xy yz xz (fstruc) */
  double adv_beta;      /* Advection.par[0]: LUST weight (adv 6) */
  int adv_fn;           /* Advection.iCod2: NVD function 1..9 (adv 5) */
  int fwall;            /* Turbulence.fWall: the wall model's viscosity on walls */
  const double *wallpar; /* numel*NWALLPAR (yPlus, uPlus, uFri, stressW) (fwall) */
  int rhie;             /* MomentumModel.fRhieChowInt: 1 order-independent, every
                           cell's face velocity reads the D field as it was at the
                           call's start; 2 the reference's serial loop, which reads
                           the D it has already rewritten for lower-numbered
                           neighbours (CellLoopInc.c:301, 364) */
} orc_vel_opts;

/* m->facer is faceVelR (velocity loads; a cell flagged there has no
 * equation), facepresr faceRpres (read, without effect on the momentum
 * system).  cc: cell centroids (numel*3); xm: face centres (nface*3); prop
 * nmat x MAXPROP (DYNAMICVISCOSITY 0, DENSITY 1); vel, gradpres, dfield
 * numel*3; gradvel numel*9 (row i = grad u_i).  dfield is updated in place
 * cell by cell as the reference does.  a: al (al|au for unsym CSRC); ad and
 * b: 3*neq (u, v, w blocks); rcell 3*numel.  Velocity loads: MOVEWALL,
 * STATICWALL, constant INLET, OUTLET, OPEN, INLETTOTALPRES and
 * INLETSTAICTPRES (whose direction is the load's own par[0..2]: the
 * reference reads an uninitialised array there).  Returns 0, -1 for input
 * the reference cannot take, -2 for an INLET given as a function. */
int orc_vel_assemble(const orc_dif_mesh *m, const short *facepresr, const double *cc,
                     const double *xm, const orc_load *lvel, int nlvel,
                     const orc_vel_opts *o, const double *prop, const double *pres,
                     const double *gradpres, const double *vel, const double *gradvel,
                     double *dfield, int storage, int unsym, int neq, int nad,
                     const int *ia, const int *ja, double *a, double *ad, double *b,
                     double *rcell, int forces, int matrix, int calrcell);

/* ---- gradient reconstruction (rcGradU, CellLoop.c:4544-4790) ---------- */

#define ORC_RCGRADGAUSSC 1 /* Define.h:377 */
#define ORC_RCLSQUARE 3    /* Define.h:379 */

/* leastSquareMatrix with RCLSQUARE, ndm = 3 (CellLib.c:3500-3590), for
 * every cell as rcLeastSquare stores it (CellLoop.c:4830-4880):
 * lsq[(cell * 3 + i) * maxviz + face]. */
void orc_ls_matrix(const orc_dif_mesh *m, double *lsq);

/* rcGradU with rcGrad.type ORC_RCGRADGAUSSC (greenGaussCell, CellLib.c:
 * 2481-2780) or ORC_RCLSQUARE (leastSquare, CellLib.c:2931-3215), no
 * limiter, ndm = 3, ndf 1 or 3.  m->facer holds the field's face loads
 * (faceRpres, faceRvel, ...); prop nmat x MAXPROP (COEFDIF 0, read by
 * NEUMANN faces); lsq from orc_ls_matrix (least squares only); u numel*ndf;
 * gradu numel*ndf*3, row k = grad u_k: in, the previous gradient (faces
 * without a load extrapolate with it under Green-Gauss), out, the new one.
 * FLUXPRES is restated without buoyancy (gradPbBuoyant's zero branch).
 * Returns 0, -1 for input whose face value the reference leaves undefined
 * (a load type its branch does not handle, NEUMANN with zero COEFDIF under
 * Green-Gauss, ROBIN with ndf = 3), -2 for loads given as functions and
 * SINBC. */
int orc_rc_grad(const orc_dif_mesh *m, const orc_load *loads, int nloads, int type, int ndf,
                const double *prop, const double *lsq, const double *u, double *gradu);

/* ---- the MPI path: row-partitioned PCG and BiCGSTAB ------------------- */

/* One rank's layout and interface (Interface, Mesh.h:212-222; the MPI CSRD of
 * Datastruct.c:129-190): rows 0..nEqNov-1 owned, nEqNov..nEq-1 ghosts. */
typedef struct {
  int nEq, nEqNov, nAd, nAdR, unsym;
  const int *ia, *ja;
  const double *al, *ad;
  int nRcvs, nSends, nVizPart;
  const int *iaSends, *iaRcvs, *fMap;
  const short *vizPart;
  /* storage code (Define.h:407-412): 0 or 2 CSRD, 3 CSRC, 4 ELLPACK,
   * 5 CSRDCOO, 6 CSRCCOO; the layouts of Datastruct.c:115-420 */
  int storage;
} orc_rank;

/* mpiPcg (Cg.c:256-442, solver 1) or mpiPbicgstab (Bicgstab.c:298-520,
 * solver 2) with nranks ranks simulated in this process: comunicateNeq
 * (ParallelMpi.c:3346-3418) before every product, the storage's product
 * -- mpiMatVecCsrD (HccaBlas.c:4096-4130), mpiMatVecCsrDSym (:2846-2895),
 * mpiMatVecCsrC (:4394-4440), mpiMatVecCsrDcooSym (:2928-2975),
 * mpiMatVecCsrCcoo (:4611-4670) or mpiMatVecEllPack (:5094-5150) -- and
 * each dot a rank's left-to-right sum, summed over the ranks in rank order
 * (the MPI_Allreduce of dot, HccaBlas.c:393-437).  b[r][nEqNov], x[r][nEq].
 * Returns the status; -1 on a bad interface. */
int orc_mpi_solve(int solver, int nranks, const orc_rank *rk, const double *const *b,
                  double *const *x, double tol, unsigned maxit, int newx, orc_stats *st);

#endif
