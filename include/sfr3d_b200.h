/*
 * sfr3d_b200.h -- C ABI of the B200 (sm_100a) linear-solve path.
 *
 * Drop-in for SFR3D's solver entry points (include/Solv.h of the reference):
 * the Jacobi-preconditioned CG (Cg.c) and Jacobi right-preconditioned
 * BiCGSTAB (Bicgstab.c) over the CSRD, CSRC and ELLPACK layouts that
 * dataStruct (Datastruct.c:28) builds.  Plain pointers and sizes only; every
 * entry returns an int status (SFR_OK = 0) instead of calling exit() as the
 * reference does, except sfr_solverC which keeps the reference's behaviour.
 *
 * Arrays named ia/ja/al/ad/au/b/x follow the reference's meaning:
 *   CSRD  (storage 2): ia[neq+1], ja[nad] ascending per row, al[nad]
 *                      off-diagonals, ad[neq] diagonal.  unsym = 0 stores the
 *                      strict lower part only (Datastruct.c:117-335).
 *   CSRC  (storage 3): strict lower pattern; al[nad] lower values and, when
 *                      unsym, au[nad] = A(ja[k], i) (Csr.c:736-1022).  As in
 *                      solverC, au may be NULL with the upper values stored at
 *                      al + nad (HccaBlas.c:4233-4236).
 *   ELLPACK (storage 4): ia = {width, neq*width}; ja, al row-major
 *                      neq x width; padded slots have ja = i, al = 0
 *                      (EllPack.c:26-149).
 * Indices are 0-based int32 (INT, Define.h:429); values are double.
 */
#ifndef SFR3D_B200_H
#define SFR3D_B200_H

#include <stdbool.h>
#include <stdint.h>
#include <stdio.h>

#ifdef __cplusplus
extern "C" {
#endif

/* solver codes, Define.h:392-396 */
#define SFR_PCG 1
#define SFR_PBICGSTAB 2
#define SFR_PBICGSTABL2 3 /* BiCGSTAB(2), Bicgstab.c:1172 */
#define SFR_GMRES 4       /* GMRES(15), Iters.c:587; maxit counts restart cycles */
#define SFR_MINRES 5      /* MINRES, Iters.c:309 (symmetric matrices) */
/* storage codes, Define.h:407-410 */
#define SFR_CSRD 2
#define SFR_CSRC 3
#define SFR_ELLPACK 4
#define SFR_CSRDCOO 5 /* MPI: CSRD lower part, ghost columns in COO (symmetric) */
#define SFR_CSRCCOO 6 /* MPI: CSRC, ghost columns in COO */

/* status codes */
#define SFR_OK 0
#define SFR_MAXIT 1          /* maxIt reached without convergence */
#define SFR_BREAKDOWN 2      /* zero or non-finite Krylov scalar */
#define SFR_BAD_INPUT -1     /* rejected before any device work */
#define SFR_CUDA_ERROR -2    /* a CUDA call failed */
#define SFR_TIMEOUT -3       /* a bounded grid-wide wait gave up */
#define SFR_UNSUPPORTED -4   /* solver/storage pair not handled here */

/* precision modes */
#define SFR_FP64 0           /* plain FP64: the reference's arithmetic */
#define SFR_MIXED 1          /* FP32 matrix + inner Krylov, FP64 refinement */

typedef struct sfr_system sfr_system; /* one pattern resident on a device */

/* Per-solve report; the first fields are what the reference's log line and
 * post-processing report (Cg.c:155-208, Bicgstab.c:188-242). */
typedef struct {
  int32_t iters;        /* j+1 as the reference counts (sum of inner its) */
  int32_t status;       /* SFR_* */
  double xKx;           /* x^T A x */
  double norm_x;        /* ||x||_2 */
  double norm_r;        /* ||b - A x||_2 (true residual, FP64) */
  double norm_r_m;      /* ||b - A x||_M (PCG) */
  double conv;          /* stopping threshold tol*||b|| (M-norm for PCG) */
  double seconds;       /* device time of the solve (CUDA events) */
  int32_t refinements;  /* MIXED: outer FP64 refinement steps */
  int32_t inner_iters;  /* MIXED: inner FP32 iterations, all cycles */
  double relres;        /* ||b - A x||_2 / ||b||_2 at exit */
} sfr_solve_info;

/* ---- handle API ------------------------------------------------------ */

/* Upload a pattern (replaces dataStruct's product for the device; the
 * pattern is fixed for the life of the handle).  For ELLPACK, ia is the
 * two-entry header.  Replaces: the pattern half of solverC's inputs,
 * Solv.h:59-70. */
int sfr_gpu_create(int32_t neq, int32_t nad, const int32_t *ia,
                   const int32_t *ja, int32_t storage, int32_t unsym,
                   int32_t device, sfr_system **out);

/* Upload values (al/ad/au as solverC receives them, Solv.h:59-70); rewritten
 * every outer iteration in the application. */
int sfr_gpu_set_values(sfr_system *s, const double *al, const double *ad,
                       const double *au);

/* Replace only the diagonal (the u/v/w momentum solves share al/au and
 * differ in ad, Simple.c:2736-2750). */
int sfr_gpu_set_diagonal(sfr_system *s, const double *ad);

/* Solve A x = b with host b and x (copies inside).  Same semantics as
 * callCg (Solv.c:936) / callBicgStab (Solv.c:1052): newX zeroes x, tol is
 * the reference's relative tolerance.  info may be NULL.  SFR_PBICGSTABL2,
 * SFR_GMRES and SFR_MINRES (callBicgStabl2 Solv.c:1173, callGmres
 * Solv.c:1263, callMinRes Solv.c:1331) run in FP64 with one right-hand side
 * (SFR_UNSUPPORTED with SFR_MIXED); GMRES's maxit counts restart cycles of
 * 15 iterations and its iteration count is 15 x cycles + 1, as the
 * reference reports it. */
int sfr_gpu_solve(sfr_system *s, int32_t solver, const double *b, double *x,
                  double tol, uint32_t maxit, int32_t newx, int32_t precision,
                  sfr_solve_info *info);

/* Same with device-resident b and x (no host copies) on `stream`
 * (cudaStream_t, NULL = legacy default). */
int sfr_gpu_solve_device(sfr_system *s, int32_t solver, const double *d_b,
                         double *d_x, double tol, uint32_t maxit,
                         int32_t newx, int32_t precision, void *stream,
                         sfr_solve_info *info);

/* k right-hand sides sharing the matrix (the momentum u,v,w batch,
 * Simple.c:2983-3040): b and x are k*neq, RHS r at offset r*neq; ad_k is
 * NULL (shared diagonal) or k*neq per-RHS diagonals.  Solved in one
 * persistent launch.  info has k entries. */
int sfr_gpu_solve_multi(sfr_system *s, int32_t solver, int32_t k,
                        const double *ad_k, const double *b, double *x,
                        double tol, uint32_t maxit, int32_t newx,
                        int32_t precision, sfr_solve_info *info);

/* The same with device arrays (d_ad_k may be NULL) on `stream`, e.g. the
 * u, v, w systems a device momentum assembly left in d_ad3 / d_b3. */
int sfr_gpu_solve_multi_device(sfr_system *s, int32_t solver, int32_t k, const double *d_ad_k,
                               const double *d_b, double *d_x, double tol, uint32_t maxit,
                               int32_t newx, int32_t precision, void *stream,
                               sfr_solve_info *info);

/* Choose how solves run: engine 0 = automatic (by size and solve), 1 = persistent
 * (the whole solve in one cooperative launch: lowest latency, small
 * systems), 2 = graph (one full-occupancy kernel per phase inside a CUDA
 * graph whose iteration loop is a device-controlled conditional node: large
 * systems), 3 = the graph engine's kernels launched from a host loop for
 * exactly maxit iterations (for profilers, which cannot look inside graphs
 * with conditional nodes; finished solves make the remaining launches
 * no-ops), 4 = resident (mixed-precision PCG with one right-hand side: one
 * cooperative launch with a block per SM, the symmetrically scaled FP32
 * operator with 16-bit column offsets held in L2 and the inner vectors in
 * shared memory; SFR_UNSUPPORTED for other solves, for a diagonal that is
 * not positive, a matrix bandwidth above 32767 or rows that do not fit the
 * blocks' shared memory -- about 2.8 million on a B200).  The automatic
 * choice takes the resident engine for mixed PCG from 100,000 rows when it
 * applies.  threads (128 or 256) and slices_per_warp (1..64; a SELL slice is
 * 32 rows) set the graph engine's launch shape; 0 keeps the current value;
 * slices_per_warp = -1 (the default) sizes the SpMV phases to one wave of
 * the blocks resident on the GPU at once. */
int sfr_gpu_set_engine(sfr_system *s, int32_t engine, int32_t threads,
                       int32_t slices_per_warp);

/* Graph engine: in the iteration's SpMV phases each warp prefetches into
 * L2 (cp.async.bulk.prefetch.L2, one request for a slice's values and one
 * for its slot columns) the SELL slice it reaches `rounds` rounds later, so
 * that DRAM reads of the matrix overlap the current slice's gathers.  0
 * (the default) turns it off; at most 8. */
int sfr_gpu_set_prefetch(sfr_system *s, int32_t rounds);

/* Graph engine, FP64 PCG with one right-hand side: mode 1 runs each
 * iteration as one cooperative kernel (SpMV and dot, grid barrier, x/r/z
 * update and dot, grid barrier, p update) that keeps q = A p and then
 * z = M r of a block's rows in shared memory instead of HBM; mode 2 is the
 * same kernel held to 40 registers so that six blocks fit an SM; in mode 3
 * the last block to arrive at a barrier sums the partials once and
 * broadcasts the total in one epoch-tagged word that the others poll; mode
 * 4 runs mode 3's iteration in a loop inside one cooperative launch for the
 * whole solve, each block waiting after its update of p only on the blocks
 * whose p its next SpMV phase gathers.  Solves it
 * does not serve (other solvers, K > 1, mixed precision, or no co-resident
 * shape) take the three-kernel iteration.  4 is the default; 0 turns the
 * fused iteration off (three kernels an iteration); other values are
 * SFR_BAD_INPUT. */
int sfr_gpu_set_fused(sfr_system *s, int32_t mode);

/* Graph engine, BiCGSTAB: 1 stages each warp's SELL slices (slot values and
 * columns) in shared memory with bulk copies issued three slices ahead, so
 * the SpMV phases wait on memory only for their gathers; it applies when the
 * columns fit 16-bit offsets and no slice is wider than 8 slots.  0 (the
 * default) reads the slices from global memory: on the 128^3 momentum
 * systems staging measured even with FP32 values and slower with FP64 (the
 * staged FP64 phases need more registers, so fewer blocks fit an SM).  The
 * arithmetic is the same either way.  Other values are SFR_BAD_INPUT. */
int sfr_gpu_set_staging(sfr_system *s, int32_t flag);

/* Result of sfr_gpu_autotune. */
typedef struct {
  int32_t engine;           /* chosen engine: 1 persistent, 2 graph, 4 resident */
  int32_t threads;          /* graph engine block size */
  int32_t slices_per_warp;  /* graph engine SpMV phases: 0 one wave, else slices per warp */
  int32_t prefetch;         /* graph engine SpMV-phase L2 prefetch distance (rounds) */
  int32_t fused;            /* graph engine FP64 PCG: one kernel an iteration (mode) */
  double ms;                /* the choice's solve time (ms, CUDA events) */
  int32_t default_engine, default_threads, default_slices_per_warp, default_prefetch,
      default_fused;
  double default_ms;        /* the automatic choice's solve time (0 when not measured) */
  int32_t candidates;       /* candidates timed (0: taken from a cache) */
  int32_t source;           /* 0 measured, 1 this handle's table, 2 the SFR_TUNE_CACHE file */
} sfr_tune_result;

/* Autotune how this system's solves of one kind (solver, k right-hand
 * sides, own or per-RHS diagonals, precision) run: the engine (persistent,
 * graph, resident) and the graph engine's block size and SELL slices per
 * warp, each candidate timed on the caller's own right-hand sides b (k*neq
 * host doubles; ad_k NULL or k*neq per-RHS diagonals).  The automatic choice
 * is kept unless a candidate is more than 2 % faster.  The choice is kept in
 * the handle -- later solves with engine 0 (automatic) take it -- and, when
 * the environment variable SFR_TUNE_CACHE names a file, appended there and
 * read back by later tunes of the same system size, pattern, storage, kind
 * of solve and GPU, so the choice is fixed across processes.  No
 * counterpart in the reference, whose OpenMP solvers balance rows by
 * nonzeros (partitionCsrByNonzeros, Csr.c:1827-1942).  PCG and BiCGSTAB
 * only (SFR_UNSUPPORTED otherwise). */
int sfr_gpu_autotune(sfr_system *s, int32_t solver, int32_t k, const double *ad_k,
                     const double *b, double tol, uint32_t maxit, int32_t precision,
                     sfr_tune_result *out);
/* Forget this handle's autotuned choices (the automatic choice by size
 * applies again). */
int sfr_gpu_autotune_clear(sfr_system *s);

/* Solve A^T x = b (host arrays) with the same Krylov path.  The reference
 * has no transpose solve; this serves the adjoint below. */
int sfr_gpu_solve_transpose(sfr_system *s, int32_t solver, const double *b,
                            double *x, double tol, uint32_t maxit,
                            int32_t newx, int32_t precision,
                            sfr_solve_info *info);

/* Adjoint of x = A^-1 b for a scalar J with g = dJ/dx (host arrays):
 * solves A^T lam = g and returns dJ/db = lam (n) and dJ/dA_ij = -lam_i x_j
 * on the stored pattern, in the layout sfr_gpu_set_values takes: g_al like
 * al, g_ad like ad, g_au like au (CSRC unsym).  An entry stored once for two
 * mirrored positions (strict-lower storage of a symmetric matrix) gets both
 * terms.  Any gradient pointer may be NULL.  No counterpart in the
 * reference. */
int sfr_gpu_adjoint(sfr_system *s, int32_t solver, const double *x,
                    const double *g, double *lam, double *g_al, double *g_ad,
                    double *g_au, double tol, uint32_t maxit,
                    int32_t precision, sfr_solve_info *info);

int sfr_gpu_destroy(sfr_system *s);

/* ---- batches of independent systems ----------------------------------- */

typedef struct sfr_batch sfr_batch; /* many systems solved in one launch */

/* Upload nsys patterns of one storage kind (arrays of per-system pointers,
 * each system as sfr_gpu_create takes it).  The systems are concatenated
 * block-diagonally; one persistent cooperative launch (replayed from a CUDA
 * graph) solves them all, each system by its own team of thread blocks with
 * its own barrier, so each stops at its own convergence.  No counterpart in
 * the reference, which solves systems one solverC call at a time. */
int sfr_gpu_batch_create(int32_t nsys, const int32_t *neq, const int32_t *nad,
                         const int32_t *const *ia, const int32_t *const *ja,
                         int32_t storage, int32_t unsym, int32_t device,
                         sfr_batch **out);
int sfr_gpu_batch_set_values(sfr_batch *b, const double *const *al,
                             const double *const *ad,
                             const double *const *au);
/* Solve every system (b[s], x[s] host arrays of its neq); info has nsys
 * entries.  Returns the first non-OK per-system status, or an error. */
int sfr_gpu_batch_solve(sfr_batch *b, int32_t solver, const double *const *bv,
                        double *const *x, double tol, uint32_t maxit,
                        int32_t newx, int32_t precision, sfr_solve_info *info);
/* Work weights of the systems (blocks are shared out in proportion). */
int sfr_gpu_batch_set_weights(sfr_batch *b, const double *w);
/* Autotune the launch plan on bv: the batch takes as long as its slowest
 * team, so the blocks are shared out to equalise the teams' times, which
 * each team measures inside the launch.  Plans tried: the default (blocks by
 * slices x n^(1/3)), blocks by slices x measured iterations, then up to three
 * plans from a fitted model t_s(B) = f_s + w_s / B of each team's time
 * against its block count.  The fastest plan measured is kept for later
 * solves; *ms_out = its solve time.  The reference balances its OpenMP rows
 * by nonzeros (partitionCsrByNonzeros, Csr.c:1827-1942); here the balance is
 * by measured time. */
int sfr_gpu_batch_autotune(sfr_batch *b, int32_t solver,
                           const double *const *bv, double tol,
                           uint32_t maxit, int32_t precision, double *ms_out);
/* Report of the last sfr_gpu_batch_autotune. */
typedef struct {
  double default_ms;   /* blocks by the default work estimate */
  double weighted_ms;  /* blocks by slices x measured iterations */
  double tuned_ms;     /* the plan kept (fastest measured) */
  int32_t plans;       /* plans measured */
  int32_t kept;        /* 0 default, 1 weighted, 2.. a model round */
  int32_t grid;        /* blocks of the kept plan */
  int32_t max_team_blocks, min_team_blocks;
} sfr_batch_tune;
int sfr_gpu_batch_tune_report(const sfr_batch *b, sfr_batch_tune *out);
int sfr_gpu_batch_stats(const sfr_batch *b, int32_t *grid, int64_t *rows,
                        int64_t *bytes);
int sfr_gpu_batch_destroy(sfr_batch *b);

/* ---- kernels for measurement and tests (device pointers) ------------- */

/* y = A x on the device (the matVec* family, HccaBlas.c:2620-4755). */
int sfr_gpu_spmv(sfr_system *s, const double *d_x, double *d_y,
                 void *stream);
/* y = A^T x on the device (the transpose the adjoint solve uses; the
 * reference has no transpose product). */
int sfr_gpu_spmv_transpose(sfr_system *s, const double *d_x, double *d_y,
                           void *stream);
/* y = A x and returns (y, x) through *dot_out (host), the fused SpMV+dot
 * of the CG step (Cg.c:103-108). */
int sfr_gpu_spmv_dot(sfr_system *s, const double *d_x, double *d_y,
                     double *dot_out, void *stream);
/* (a, b) with the device's deterministic reduction (dot, HccaBlas.c:393). */
int sfr_gpu_dot(const double *d_a, const double *d_b, int32_t n,
                double *dot_out, void *stream);

/* (a, b) like sfr_gpu_dot, for callers that cannot let this library
 * allocate device memory (a program that reserves its GPU memory once and
 * parcels it out itself, as SFR3D does with its host arena, or one running
 * while another allocator holds the memory).  No counterpart in the
 * reference.  Never calls cudaMalloc/cudaFree: its scratch is a fixed
 * 4,752-byte device array (592 block partials, result, counter) that every
 * GPU loading the library keeps until exit.  Same launch shape as
 * sfr_gpu_dot, so the same bits.  The first call on a device looks up that
 * array's address and keeps it (cudaDeviceReset is not supported after
 * it); make it before any stream capture.  Calls share the array, so calls
 * that overlap on the GPU race.  n < 0, or a GPU with more than 148 SMs
 * (more partials than the array holds), is rejected with SFR_BAD_INPUT. */
int sfr_gpu_dot_noalloc(const double *d_a, const double *d_b, int32_t n,
                        double *dot_out, void *stream);

/* Device memory the handle holds (bytes) and its SELL slot count. */
int sfr_gpu_stats(const sfr_system *s, int64_t *bytes, int64_t *slots,
                  int32_t *bandwidth);

/* ---- device assembly of the diffusion system ------------------------- */
/* systFormDif (CellLoop.c:285-455) -> cellDif3D (CellDif.c:312-537) run on
 * the GPU and write the system's values where solverC reads them: the raw
 * al (| au) / ELLPACK slots the reference's csr()/ellPack() fill
 * (Csr.c:549-1022, EllPack.c:113-149), the diagonal and the force vector,
 * with the same rounding as the reference (ndf = 1, ndm = 3, one process).
 * The matrix never crosses PCIe: the next sfr_gpu_solve_device uses it. */

/* The mesh arrays systFormDif reads, as the reference stores them (1-based
 * indices; MAT2D/MAT3D row-major).  Arrays systFormDif passes through but
 * cellDif3D does not read (node incidence, eta, face centres, |vSkew|,
 * geometry types) are not needed. */
typedef struct {
  int32_t numel;           /* cells (mesh->numelNov) */
  int32_t maxviz;          /* face slots per cell (mesh->maxViz), 1..8 */
  int64_t nfaces;          /* length of the per-face arrays */
  int32_t nmat;            /* length of caltype */
  int32_t pad;
  const int32_t *nelcon;   /* numel*maxviz: neighbour + 1, -1 boundary (elm.adj.nelcon) */
  const int16_t *nviz;     /* numel: faces of the cell (elm.adj.nViz) */
  const int32_t *cellface; /* numel*maxviz: face + 1 (elm.cellFace) */
  const int32_t *owner;    /* nfaces*2: owner cell + 1 first (face.owner) */
  const double *volume;    /* numel (elm.geom.volume) */
  const double *dcca;      /* numel*maxviz (elm.geom.dcca) */
  const double *xmcc;      /* numel*maxviz*3 (elm.geom.xmcc) */
  const double *mksi;      /* nfaces (face.mksi) */
  const double *ksi;       /* nfaces*3 (face.ksi) */
  const double *area;      /* nfaces (face.area) */
  const double *normal;    /* nfaces*3 (face.normal) */
  const double *vskew;     /* nfaces*3 (face.vSkew) */
  const int16_t *caltype;  /* nmat: cell library of the material (1 = diffusion) */
  const int16_t *mat;      /* numel: material + 1 (elm.mat) */
  const int32_t *id;       /* numel: equation + 1 (sistEqD->id) */
  const int16_t *facer;    /* numel*(maxviz+1): load + 1 per face, then the cell's own entry */
  const double *cc;        /* numel*3 cell centroids (elm.geom.cc): momentum plans only */
  const double *xm;        /* nfaces*3 face centres (face.xm): momentum plans only */
} sfr_dif_mesh;

/* One entry of the load table (Loads, StructDefine.h:356-366). */
typedef struct {
  int32_t type;   /* DIRICHLETBC 1, NEUMANNBC 2, ROBINBC 3, INLET 6, OUTLET 7,
                   * MOVEWALL 8, INLETSTAICTPRES 9, OPEN 10, INLETTOTALPRES 13,
                   * STATICWALL 14, FLUXPRES 15 (Define.h:317-332) */
  int32_t var;    /* nTypeVar: 0 constant (1 = function: SFR_UNSUPPORTED) */
  int32_t np;     /* parameters given */
  int32_t pad;
  double par[20]; /* MAXLOADPARAMETER */
  double density; /* Loads.density (an OPEN velocity load's inflow density) */
} sfr_load;

/* The rest of what systFormDif reads (Diffusion.iCod, DiffModel.fRes,
 * Temporal). */
typedef struct {
  int32_t icod;      /* 1 ORTHOGONAL 2 MINIMAL 3 ORTHOGONALC 4 OVERRELAXED (Define.h:304-307) */
  int32_t fres;      /* b = the cell residual (1) or the force (0) */
  int32_t time_flag; /* Temporal.flag: implicit time term */
  int32_t time_type; /* 0 EULER, 1 BACKWARD */
  double dt, dt0;    /* Temporal.dt[0], dt[1] */
} sfr_dif_opts;

/* A plan is not re-entrant: calls on one plan must not overlap (they share
 * its staged load table and, for the host-array calls, its device buffers).
 * Different plans may be used from different threads. */
typedef struct sfr_dif_plan sfr_dif_plan;

/* Bind a mesh to a system (whose pattern is the one dataStruct built for
 * that mesh) and precompute on the GPU, once, what cellDif3D derives from
 * the geometry alone for scheme `icod`: the face weights, |E| and the
 * non-orthogonal split.  SFR_BAD_INPUT for a mesh the reference cannot
 * assemble (a cell library other than diffusion, an equation number out of
 * range or used twice, a neighbour index that is neither a cell nor -1, a
 * row holding a column twice), with the reason in sfr_last_error(). */
int sfr_gpu_dif_plan_create(sfr_system *s, const sfr_dif_mesh *mesh, int32_t icod,
                            sfr_dif_plan **out);

/* One systFormDif call with device arrays on `stream`: density, cdiff, u0
 * (numel) and gradu0 (numel*3, unused for ORTHOGONAL) in; b (neq) and rcell
 * (numel) out when forces / calrcell are set; the matrix into the system
 * when matrix is set.  b0 (neq, may be NULL) is added to b and to the cell
 * residuals as Diffusion.c:107-118 does after the call.  loads: nloads <= 32
 * host entries; a face may only name a load below nloads.  SINBC loads and
 * loads given as functions are SFR_UNSUPPORTED, OUTLET (which reads a
 * velocity the diffusion cell has not) SFR_BAD_INPUT. */
int sfr_gpu_dif_assemble_device(sfr_dif_plan *p, const sfr_load *loads, int32_t nloads,
                                const sfr_dif_opts *o, const double *d_density,
                                const double *d_cdiff, const double *d_u0,
                                const double *d_gradu0, const double *d_b0, double *d_b,
                                double *d_rcell, int32_t forces, int32_t matrix,
                                int32_t calrcell, void *stream);

/* The same with host arrays: the fields are copied in, b and rcell copied
 * back (either may be NULL); the matrix stays on the device. */
int sfr_gpu_dif_assemble(sfr_dif_plan *p, const sfr_load *loads, int32_t nloads,
                         const sfr_dif_opts *o, const double *density, const double *cdiff,
                         const double *u0, const double *gradu0, const double *b0, double *b,
                         double *rcell, int32_t forces, int32_t matrix, int32_t calrcell);

/* ---- device assembly of the SIMPLE pressure correction ---------------- */
/* systFormSimplePres (CellLoopInc.c:471-700) -> cellSimplePres3D
 * (CellPres.c:903-1218): face coefficients rho_f |E_f| / |ksi| from the
 * momentum D field, the Rhie-Chow face mass fluxes as the force, pressure
 * loads (pLoadSimplePres) and velocity loads (pLoadSimple, pressure part),
 * serial and without a wall model, as velPresCoupling builds it.  mesh->facer
 * is facePresR; facevelr (numel*(maxviz+1)) is faceVelR.  icod is the
 * pressure scheme: 1 ORTHOGONAL or 4 OVERRELAXED (the reference's split sets
 * nothing for the other two). */
int sfr_gpu_pres_plan_create(sfr_system *s, const sfr_dif_mesh *mesh, const int16_t *facevelr,
                             int32_t icod, sfr_dif_plan **out);

/* One systFormSimplePres call on device arrays: pres (numel), gradpres, vel
 * and dfield (numel*3) in; b and rcell (the cell mass residual) out.  prop
 * is the host material table, nmat x MAXPROP (10) doubles, density in
 * column 1.  lvel / lpres: at most 32 entries each.  INLET velocity loads
 * given as functions are SFR_UNSUPPORTED. */
int sfr_gpu_pres_assemble_device(sfr_dif_plan *p, const sfr_load *lvel, int32_t nlvel,
                                 const sfr_load *lpres, int32_t nlpres, const double *prop,
                                 const double *d_pres, const double *d_gradpres,
                                 const double *d_vel, const double *d_dfield, double *d_b,
                                 double *d_rcell, int32_t forces, int32_t matrix,
                                 int32_t calrcell, void *stream);

/* The same with host arrays (b and rcell copied back when not NULL). */
int sfr_gpu_pres_assemble(sfr_dif_plan *p, const sfr_load *lvel, int32_t nlvel,
                          const sfr_load *lpres, int32_t nlpres, const double *prop,
                          const double *pres, const double *gradpres, const double *vel,
                          const double *dfield, double *b, double *rcell, int32_t forces,
                          int32_t matrix, int32_t calrcell);

/* ---- device assembly of the SIMPLE momentum system ------------------- */
/* systFormSimpleVel (CellLoopInc.c:98-470) -> cellSimpleVel3D
 * (CellSimple.c:106-727) placed by csrSimple (Csr.c:1024): the u, v, w
 * systems share the off-diagonals and carry their own diagonals, forces and
 * residuals; the momentum D field (V / a_P, or V / (a_P - sum a_N) for
 * SIMPLEC) comes out for the pressure correction.  Restated without a wall
 * model (an eddy viscosity field and the residual stress integral are bound
 * by sfr_gpu_vel_turbulence), with the advection schemes of adv below and
 * face velocities without Rhie-Chow (with it on, the reference's serial loop
 * reads D fields it has already overwritten, so its result depends on the
 * cell order).  Velocity loads: MOVEWALL, STATICWALL, constant INLET,
 * OUTLET, OPEN, INLETTOTALPRES and INLETSTAICTPRES, whose inflow direction is
 * the load's par[0..2] (the reference's getLoads copies no parameter for
 * that type, Loads.c:148-150, and its pLoadSimple reads an uninitialised
 * array); an INLET given as a function is SFR_UNSUPPORTED.  mesh->facer is
 * faceVelR; mesh->cc and mesh->xm are required.  CSRD or CSRC. */
typedef struct {
  int32_t icod;        /* Diffusion.iCod: 1..4 */
  int32_t fso;         /* MomentumModel.fSoPressure: second-order face pressure */
  int32_t fvisc;       /* MomentumModel.fViscosity: explicit viscous part */
  int32_t fres;        /* MomentumModel.fRes */
  int32_t type_simple; /* 1 SIMPLE, 2 SIMPLEC */
  int32_t time_flag, time_type;
  int32_t adv;         /* Advection.iCod1 (advectiveScheme, CellLib.c:6394-6650): 0 or 1
                          FoUp, 2 CD (deferred central), 3 SoUp (linear upwind), 5 NVD
                          (faceBaseNvd, CellLib.c:4900, function adv_fn), 4 TVD (faceBaseTvdV1,
                          CellLib.c:4845, limiter adv_fn 1..5), 6 LUST
                          (deferredLust, CellLib.c:5162, weight adv_beta) */
  double dt, dt0;
  double under;        /* under-relaxation of the velocity (alphaVel) */
  int32_t fturb;       /* Turbulence.fTurb: effective viscosity mu + eddy viscosity
                          (fields bound by sfr_gpu_vel_turbulence) */
  int32_t fstruc;      /* Turbulence.fTurbStruct: the residual stress tensor's face
                          integral (turbStructIntegral, CellLib.c:7586) */
  double adv_beta;     /* Advection.par[0]: LUST's linear-upwind weight */
  int32_t adv_fn;      /* Advection.iCod2 for NVD: 1 BCD, 2 MUSCL, 3 SMART, 4 ModSMART,
                          5 SuperBee, 6 ModSuperBee, 7 STOIC, 8 MinMod, 9 ModBCD (nvd,
                          CellLib.c; MUSCL and STOIC weigh 0, as there) */
  int32_t fwall;       /* Turbulence.fWall: walls (MOVEWALL, STATICWALL) take the wall
                          model's viscosity mu yPlus / uPlus (mu where yPlus <= 0.01)
                          from the field bound by sfr_gpu_vel_wall (Loads.c:300-313) */
  int32_t rhie;        /* MomentumModel.fRhieChowInt: 1 Rhie-Chow face velocities
                          (interpolFaceVel, CellLib.c:6853-6960) reading the D field
                          as it was at the call's start, for every cell -- a defined,
                          order-independent form; the reference's serial loop reads
                          the D it has already rewritten for lower-numbered
                          neighbours, so its result depends on the cell order.
                          0 off; other values SFR_UNSUPPORTED */
} sfr_vel_opts;

int sfr_gpu_vel_plan_create(sfr_system *s, const sfr_dif_mesh *mesh, int32_t icod,
                            sfr_dif_plan **out);

/* The turbulence fields later momentum calls read (CellSimple.c:207-314,
 * 237-240): eddy[numel] eddy viscosity and stress[numel*6] the residual
 * stress tensor (xx, yy, zz, xy, yz, xz), either may be NULL.  on_device = 1:
 * device arrays, kept by pointer and read by every later call; 0: host
 * arrays, copied now into the plan.  Without the wall model (fwall, bound by
 * sfr_gpu_vel_wall) walls use the effective viscosity (Loads.c:300-313). */
int sfr_gpu_vel_turbulence(sfr_dif_plan *p, const double *eddy, const double *stress,
                           int32_t on_device);

/* The wall model's per-cell parameters that momentum calls with fwall read
 * (wallPar of systFormSimpleVel, CellLoopInc.c:322-324): wallpar[numel*4]
 * = yPlus, uPlus, uFri, stressW per cell (the turbulence module computes
 * them); on_device as for sfr_gpu_vel_turbulence.  NULL unbinds. */
int sfr_gpu_vel_wall(sfr_dif_plan *p, const double *wallpar, int32_t on_device);

/* One call on device arrays: pres (numel), gradpres, vel, dfield (numel*3),
 * gradvel (numel*9, row i = grad u_i) in; dfield (the new D), ad3 and b3
 * (3*neq: u, v, w blocks; ad3 may be NULL), rcell3 (3*numel) out; the shared
 * off-diagonals and the u diagonal into the system.  prop: host material
 * table nmat x 10 (viscosity column 0, density column 1). */
int sfr_gpu_vel_assemble_device(sfr_dif_plan *p, const sfr_load *lvel, int32_t nlvel,
                                const sfr_vel_opts *o, const double *prop, const double *d_pres,
                                const double *d_gradpres, const double *d_vel,
                                const double *d_gradvel, double *d_dfield, double *d_ad3,
                                double *d_b3, double *d_rcell3, int32_t forces, int32_t matrix,
                                int32_t calrcell, void *stream);

/* The same with host arrays (dfield updated in place; ad3, b3, rcell3
 * copied back when not NULL). */
int sfr_gpu_vel_assemble(sfr_dif_plan *p, const sfr_load *lvel, int32_t nlvel,
                         const sfr_vel_opts *o, const double *prop, const double *pres,
                         const double *gradpres, const double *vel, const double *gradvel,
                         double *dfield, double *ad3, double *b3, double *rcell3, int32_t forces,
                         int32_t matrix, int32_t calrcell);

/* Frees a plan (any kind); safe after the system is destroyed (the plan's
 * calls are not). */
int sfr_gpu_dif_plan_destroy(sfr_dif_plan *p);

/* ---- gradient reconstruction ------------------------------------------ */
/* rcGradU (CellLoop.c:4544-4790) on the device: the Green-Gauss cell kernel
 * (type 1, RCGRADGAUSSC: greenGaussCell, CellLib.c:2481-2780) or least
 * squares (type 3, RCLSQUARE: leastSquare, CellLib.c:2931-3215, with the
 * matrices of rcLeastSquare / leastSquareMatrix, CellLib.c:3500-3590), no
 * limiter, ndm = 3, for a scalar (ndf 1: the pressure) or the velocity
 * (ndf 3), bit-identical to the reference's.  The SIMPLE driver calls it for
 * the velocity and the pressure before each assembly (Simple.c:2797-2858);
 * here the gradient is formed where the field is.  Types 2 (Green-Gauss
 * nodal) and 4 (QR least squares) are SFR_UNSUPPORTED.
 *
 * The plan reads from mesh: nelcon, nviz, cellface, owner, volume, dcca,
 * xmcc, mksi, ksi, area, normal, vskew, mat, nmat and facer, which holds the
 * FIELD's face loads (faceRpres for the pressure, faceRvel for the
 * velocity).  Two reference behaviours are kept: greenGaussCell
 * interpolates every face with its cell's FIRST face's vSkew and xmcc
 * (CellLib.c:2513, 2640), and leastSquare with ndf 3 sets a face to -u_C
 * when its load is the 14th of the table, whatever its type, rather than
 * for STATICWALL loads (CellLib.c:3118). */
typedef struct sfr_grad_plan sfr_grad_plan;
int sfr_gpu_grad_plan_create(int32_t device, const sfr_dif_mesh *mesh, int32_t type,
                             sfr_grad_plan **out);

/* gradu (numel * ndf * 3, row k = grad u_k) is read as the previous
 * gradient and overwritten with the new one; u is numel * ndf.  prop is the
 * nmat x MAXPROP material table (COEFDIF, column 0, is read by NEUMANN
 * faces).  A face value the reference's branch leaves undefined (a load
 * type the branch has no case for, NEUMANN with COEFDIF 0 under
 * Green-Gauss, ROBIN with ndf 3) is SFR_BAD_INPUT; SINBC and loads given as
 * functions SFR_UNSUPPORTED.  FLUXPRES faces are taken without buoyancy.
 * Device arrays, on `stream` (NULL: the plan's own). */
int sfr_gpu_grad_device(sfr_grad_plan *p, const sfr_load *loads, int32_t nloads,
                        const double *prop, int32_t ndf, const double *d_u, double *d_gradu,
                        void *stream);

/* The same with host arrays (copied in and back; synchronous). */
int sfr_gpu_grad(sfr_grad_plan *p, const sfr_load *loads, int32_t nloads, const double *prop,
                 int32_t ndf, const double *u, double *gradu);

int sfr_gpu_grad_plan_destroy(sfr_grad_plan *p);

/* Copy the system's values back in the reference's layout: al (nad, or the
 * neq*width ELLPACK slots), ad (neq) and, for unsym CSRC, au (nad).  Any
 * pointer may be NULL. */
int sfr_gpu_get_values(sfr_system *s, double *al, double *ad, double *au);

/* Matrix Market dumps in the reference's own format (writeCoo and writeCooB,
 * WriteMtx.c:26-179, as the "pcoo" macro writes the assembled system,
 * Main.c:995-1020): CSRD only; bin writes 1.0 for every entry (the "pgraph"
 * macro).  sfr_gpu_write_coo dumps a device system (its values as
 * sfr_gpu_get_values reads them) with the host's pattern. */
int sfr_write_coo(const char *path, int32_t neq, const int32_t *ia, const int32_t *ja,
                  const double *au, const double *ad, const double *al, int32_t nad,
                  int32_t storage, int32_t unsym, int32_t bin);
int sfr_write_coo_b(const char *path, const double *b, int32_t neq);
int sfr_gpu_write_coo(sfr_system *s, const char *path, const int32_t *ia, const int32_t *ja,
                      int32_t bin);

/* x -> u as updateCellValue does after the solve (CellLoop.c:4023-4057,
 * ndf = 1): u[cell] = x[id[cell] - 1] (add = 0) or += (add = 1) for every
 * cell with id > 0, on device arrays. */
int sfr_gpu_dif_update_cells(sfr_dif_plan *p, const double *d_x, double *d_u, int32_t add,
                             void *stream);


const char *sfr_status_string(int status);
/* Text of the last failure on the calling thread (validation or CUDA). */
const char *sfr_last_error(void);
/* Compute capability of the GPU this library was built for and of `device`;
 * returns SFR_OK when the device can run it. */
int sfr_gpu_check_device(int32_t device, int32_t *major, int32_t *minor);

/* Self-test of the bounded device-side waits that replace the reference's
 * blocking MPI collectives inside the solvers (no counterpart in the
 * reference, whose MPI_Allreduce waits without a limit).  Four co-resident
 * blocks meet once at one of the waits the engines use: kind 0 the grid
 * barrier (persistent engine, fused iteration modes 1-2), kind 1 the
 * fused iteration's tagged exchange (modes 3-6), kind 2 the resident
 * engine's exchange.  The last `absent` blocks (0-3) leave before the wait.
 * Returns SFR_OK when the wait completed (absent = 0) and SFR_TIMEOUT when
 * it gave up after `spin_limit` polls because a participant never arrived;
 * either way every block has left and the context stays usable.  Allocates
 * 64 bytes (768 for kind 2) of device memory for the call. */
int sfr_gpu_wait_selftest(int32_t kind, int32_t absent, uint32_t spin_limit, void *stream);

/* ---- row partition over several GPUs (the reference's MPI path) ------ */

/* The reference's interface map (Interface, include/Mesh.h:212-222), with
 * the same field order and types, so a pointer to the reference's struct can
 * be passed as is.  Local equations 0..nEqNov-1 are this rank's rows, nEqNov..
 * nEq-1 its ghosts.  xb[0..nRcvs) receives and xb[nRcvs..nRcvs+nSends) sends;
 * neighbour n = vizPart[n] sends xb[iaRcvs[n]..iaRcvs[n+1]) to this rank and
 * receives xb[iaSends[n]..iaSends[n+1]) from it; fMap[i] is the local
 * equation of xb[i] (comunicateNeq, ParallelMpi.c:3346-3418).  xb is unused
 * here (the device keeps its own buffers) and may be NULL. */
typedef struct {
  int32_t nRcvs;
  int32_t nSends;
  int32_t *iaSends;
  int32_t *iaRcvs;
  int32_t *fMap;
  double *xb;
  uint16_t nVizPart;
  int16_t *vizPart;
} sfr_interface;

/* A row partition of one global CSRD system into the reference's per-rank
 * layouts (the preprocessor's product that dataStruct turns into the MPI
 * CSRD, Datastruct.c:129-190).  Built on the host. */
typedef struct sfr_part sfr_part;

/* Sizes of rank `rank`'s layout. */
typedef struct {
  int32_t nEq;      /* owned + ghost equations */
  int32_t nEqNov;   /* owned equations */
  int32_t nAd;      /* entries of the square part */
  int32_t nAdR;     /* entries of the rectangular (ghost-column) part; 0 unsym */
  int32_t nRcvs, nSends;
  int32_t nVizPart;
  int32_t ia_len;   /* nEqNov+1 (unsym) or 2*(nEqNov+1) (sym) */
} sfr_part_sizes;

/* Partition the rows of a global CSRD system (unsym = 1: full off-diagonal
 * rows; 0: strict lower part, the symmetric storage).  part[i] is the rank
 * of row i, or part = NULL for contiguous row blocks balanced by entries.
 * Each rank numbers its rows in global order, then its ghosts by neighbour
 * rank and, within a neighbour, by global number; rows are sorted by local
 * column (sortGraphCsr, Graph.c:114).  unsym: ia[nEqNov+1], ja[nAd] full
 * rows (mpiMatVecCsrD, HccaBlas.c:4096-4130).  sym: ia[0..nEqNov] the strict
 * lower square part and ia[nEqNov+1..] the ghost columns of the full row,
 * indexing ja + nAd (mpiMatVecCsrDSym, HccaBlas.c:2846-2895). */
int sfr_part_create(int32_t neq, const int32_t *ia, const int32_t *ja, int32_t unsym,
                    int32_t nparts, const int32_t *part, sfr_part **out);
int sfr_part_sizes_of(const sfr_part *p, int32_t rank, sfr_part_sizes *sz);
/* Fill rank `rank`'s arrays (sizes from sfr_part_sizes_of): ia, ja; src[k]
 * = index in the global al of local entry k (nAd + nAdR entries); l2g[nEq]
 * = global equation of each local one; the interface arrays iaSends and
 * iaRcvs (nVizPart+1), fMap (nRcvs+nSends), vizPart (nVizPart).  Any
 * output may be NULL. */
int sfr_part_fill(const sfr_part *p, int32_t rank, int32_t *ia, int32_t *ja, int32_t *src,
                  int32_t *l2g, int32_t *iaSends, int32_t *iaRcvs, int32_t *fMap,
                  int16_t *vizPart);
int sfr_part_destroy(sfr_part *p);

/* A set of ranks that solve together.  A local group holds all nparts ranks
 * in this process on one device (the halo is a device gather, the sums are
 * taken in rank order); an NCCL group is one rank per process, the halo
 * exchanged with ncclSend/ncclRecv and the sums with ncclAllReduce.  NCCL is
 * loaded at run time (libnccl.so.2, or the file named by SFR_NCCL_LIBRARY). */
typedef struct sfr_dist_group sfr_dist_group;
/* One rank's partition resident on a device. */
typedef struct sfr_dist sfr_dist;

int sfr_dist_group_local(int32_t nparts, int32_t device, sfr_dist_group **out);
/* 128-byte NCCL unique id, made on one rank and given to every rank. */
int sfr_dist_nccl_id(uint8_t id[128]);
int sfr_dist_group_nccl(int32_t nranks, int32_t rank, const uint8_t id[128], int32_t device,
                        sfr_dist_group **out);
int sfr_dist_group_destroy(sfr_dist_group *g);
/* kind (0 local, 1 NCCL), rank count and, for NCCL, this process's rank. */
int sfr_dist_group_info(const sfr_dist_group *g, int32_t *kind, int32_t *nranks, int32_t *rank);

/* Upload rank `rank`'s layout (as sfr_part_fill writes it, or as the
 * reference's dataStruct builds it under MPI) and interface.  Storage is
 * CSRD.  In a local group every rank is created in this process before the
 * first solve. */
int sfr_gpu_dist_create(sfr_dist_group *g, int32_t rank, int32_t nEq, int32_t nEqNov,
                        int32_t nAd, int32_t nAdR, const int32_t *ia, const int32_t *ja,
                        int32_t unsym, const sfr_interface *iNeq, sfr_dist **out);
/* The same for every MPI storage the reference's dataStruct builds
 * (Datastruct.c:115-420) and setMatVec multiplies (Solv.c:749-897):
 *   SFR_CSRD     unsym: full rows over local columns (mpiMatVecCsrD);
 *                sym: strict-lower square part, ghost columns in CSR at
 *                ia + nEqNov + 1 (mpiMatVecCsrDSym);
 *   SFR_CSRC     the CSRD-sym pattern; unsym values al | au | ghost values
 *                (mpiMatVecCsrC, HccaBlas.c:4394), sym as CSRD sym;
 *   SFR_CSRDCOO  symmetric: the square part as CSRD sym, the ghost columns
 *                in COO (rows at ia + 2 (nEqNov + 1), CSR pointers at
 *                ia + nEqNov + 1) added after the rest of the row
 *                (mpiMatVecCsrDcooSym, HccaBlas.c:2928);
 *   SFR_CSRCCOO  the same with CSRC values (mpiMatVecCsrCcoo, :4611);
 *   SFR_ELLPACK  ia = {width, nEqNov * width}, every row `width` slots over
 *                local columns (mpiMatVecEllPack, :5094).
 * Each row keeps the reference's summation order.  SFR_UNSUPPORTED for
 * CSRDCOO unsym and other storages. */
int sfr_gpu_dist_create_storage(sfr_dist_group *g, int32_t rank, int32_t storage, int32_t nEq,
                                int32_t nEqNov, int32_t nAd, int32_t nAdR, const int32_t *ia,
                                const int32_t *ja, int32_t unsym, const sfr_interface *iNeq,
                                sfr_dist **out);
/* al (every value the storage holds: nAd + nAdR, 2 nAd + nAdR for CSRC /
 * CSRCCOO unsym, nEqNov * width for ELLPACK), ad[nEqNov] (host). */
int sfr_gpu_dist_set_values(sfr_dist *d, const double *al, const double *ad);
/* mpiPcg (Cg.c:256-442) or mpiPbicgstab (Bicgstab.c:298-520) over every
 * rank this process holds: parts[nlocal] in rank order (all ranks for a
 * local group, the one rank for NCCL), b[r][nEqNov] and x[r][nEq] on the
 * host (x's ghost entries are written too).  info (may be NULL) is
 * identical on every rank. */
int sfr_gpu_dist_solve(sfr_dist_group *g, int32_t nlocal, sfr_dist *const *parts,
                       int32_t solver, const double *const *b, double *const *x,
                       double tol, uint32_t maxIt, int32_t newX, sfr_solve_info *info);
int sfr_gpu_dist_destroy(sfr_dist *d);

/* ---- drop-in for the reference entry point --------------------------- */

/* Same arguments and meaning as solverC (Solv.h:59-70, Solv.c:64-501).
 * Memoria*, Interface* and BufferOmp* are accepted as opaque pointers and
 * unused.  PCG and PBICGSTAB over CSRD/CSRC/ELLPACK run on the GPU; the
 * pattern is cached per (ia, ja, storage) so a repeated call uploads only
 * al/ad/au/b.  Writes the reference's log line to fSolvLog when fLog is
 * set.  On non-convergence prints the reference's message and calls
 * exit(EXIT_FAILURE) for PCG, GMRES and BiCGSTAB(2) and exit(-2) for
 * BiCGSTAB (Cg.c:195-200, Bicgstab.c:225-231, Iters.c:773-777,
 * Bicgstab.c:1428-1432) unless sfr_set_exit_on_failure(0) was called, in
 * which case it returns the status; MINRES only prints its warning, as the
 * reference does (Iters.c:525-529). */
int sfr_solverC(void *m, int32_t nEq, int32_t nEqNov, int32_t nAd,
                int32_t nAdR, int32_t *ia, int32_t *ja, double *al,
                double *ad, double *au, double *b, double *x, void *iNeq,
                void *bOmp, double tol, uint32_t maxIt, int16_t storage,
                int16_t solver, FILE *fSolvLog, bool fLog, bool newX,
                bool unSym, const char *name);
/* The MPI branch of solverC (Solv.c:952-977, 1070-1093: mpiPcg and
 * mpiPbicgstab when nPrcs > 1).  With an NCCL group set, every sfr_solverC
 * call of this process is one rank's share: iNeq is the reference's
 * Interface (sfr_interface has its layout), storage must be CSRD, al holds
 * nAd + nAdR values, x holds nEq entries (ghosts are written too), and
 * solver PCG or PBICGSTAB.  Rank 0 writes the MPIPCG / MPIPBICGSTAB log line
 * and the non-convergence messages; failure exits with EXIT_SOLVER (-2) as
 * the reference does (Cg.c:409-420, Bicgstab.c:478-488).  The partition is
 * cached per (ia, ja); g = NULL returns to the single-GPU path. */
int sfr_solverC_set_group(sfr_dist_group *g);
void sfr_set_exit_on_failure(int32_t flag);
/* SFR_MIXED: the inner FP32 residual must fall by this factor (0 < delta
 * < 1) before the FP64 solution is refreshed and the true residual
 * recomputed.  Sets the factor of both solvers on every engine (defaults:
 * PCG 0.1, 0.02 on the resident engine; BiCGSTAB 1e-4). */
void sfr_set_reliable_delta(double delta);
/* The same for one solver (SFR_PCG or SFR_PBICGSTAB). */
int sfr_set_solver_reliable_delta(int32_t solver, double delta);
/* Precision used by sfr_solverC (SFR_FP64 default). */
void sfr_set_precision(int32_t precision);
/* flag != 0: sfr_solverC autotunes (sfr_gpu_autotune) the first PCG or
 * BiCGSTAB solve of each pattern it caches, on that call's own right-hand
 * side, and every later call takes the choice.  Off by default. */
void sfr_set_autotune(int32_t flag);
/* Release every pattern sfr_solverC cached. */
void sfr_solverC_release(void);

#ifdef __cplusplus
}
#endif
#endif
