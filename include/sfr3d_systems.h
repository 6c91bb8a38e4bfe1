/*
 * sfr3d_systems.h -- seeded finite-volume test systems in SFR3D's own sparse
 * layouts (host library libsfr3d_systems.so; no GPU code).
 *
 * The reference assembles its systems from a mesh deck (systFormDif,
 * CellLoop.c:285 -> cellDif3D, CellDif.c:312; systFormSimpleVel,
 * CellLoopInc.c:98 -> cellSimpleVel3D, CellSimple.c:106) and stores them with
 * dataStruct (Datastruct.c:28).  This library builds the same kind of system
 * directly on a hexahedral box mesh, with the same coefficient conventions:
 *   - off-diagonal A(P,N) = -a_N, diagonal A(P,P) = sP + sum_N a_N
 *     (CellDif.c:500-523, CellSimple.c:557);
 *   - diffusion a_N = k_f |S_f| / |xi|, xi = c_N - c_P, with the harmonic
 *     face diffusivity k_f = 1 / (alpha/k_P + (1-alpha)/k_N)
 *     (CellDif.c:415-423; orthogonal part);
 *   - Dirichlet face: sP += k_P |S_f| / d_Pf (Loads.c:894-903); Neumann-zero
 *     adds nothing;
 *   - first-order upwind: a_N = D_f + max(-F_f, 0), sP += F_f
 *     (CellSimple.c:405-406), F_f the outward face flux;
 *   - implicit Euler time term sP += rho V / dt (CellDif.c:485-497).
 * Equations are numbered by reverse Cuthill-McKee (the reference calls genrcm,
 * Rcm.c:56, from reord, Reord.c:18), optionally after a seeded random
 * permutation of the cells.
 *
 * Layouts returned (all int32 indices, 0-based, as the reference stores them):
 *   CSRD  (storage 2, Datastruct.c:117-335): ia[neq+1], ja[] ascending per
 *         row, al[] off-diagonal values, ad[neq] diagonal.  "full" = every
 *         off-diagonal (unsym); "lower" = strict lower part only (sym).
 *   CSRC  (storage 3, Datastruct.c:338-570, Csr.c:736-1022): strict lower
 *         pattern; al[k] = A(i, ja[k]) and, for unsym, au[k] = A(ja[k], i).
 *   ELLPACK (storage 4, EllPack.c:26-149): row-major neq x width slots in
 *         cell-face order; a boundary slot has ja = i and a = 0.
 */
#ifndef SFR3D_SYSTEMS_H
#define SFR3D_SYSTEMS_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Kind of physics on the box. */
#define SFR_SYS_DIFFUSION 1   /* symmetric Poisson / diffusion */
#define SFR_SYS_CONVDIFF  2   /* nonsymmetric momentum convection-diffusion */

/* Face bits for Dirichlet boundaries. */
#define SFR_FACE_XMIN 1
#define SFR_FACE_XMAX 2
#define SFR_FACE_YMIN 4
#define SFR_FACE_YMAX 8
#define SFR_FACE_ZMIN 16
#define SFR_FACE_ZMAX 32

typedef struct {
  int32_t kind;            /* SFR_SYS_DIFFUSION | SFR_SYS_CONVDIFF */
  int32_t nx, ny, nz;      /* cells per axis */
  double lx, ly, lz;       /* box extents */
  double jitter;           /* node jitter, fraction of the local spacing */
  double log10k_lo;        /* per-cell diffusivity 10^U(lo,hi) */
  double log10k_hi;        /*   (lo == hi: constant 10^lo)     */
  int32_t dirichlet_faces; /* SFR_FACE_* bits */
  int32_t permute;         /* random cell permutation before numbering */
  int32_t rcm;             /* reverse Cuthill-McKee numbering */
  int32_t nrhs;            /* right-hand sides to draw */
  int32_t rhs_normal;      /* 0: iid U[-1,1], 1: iid N(0,1) */
  double peclet;           /* CONVDIFF: max cell Peclet |F_f| / D_f */
  double nu;               /* CONVDIFF: kinematic viscosity */
  double dt;               /* CONVDIFF: implicit time step (rho = 1) */
  uint64_t seed;
} sfr_sys_params;

typedef struct {
  int32_t neq;        /* rows */
  int32_t nnz_full;   /* off-diagonal nonzeros (CSRD full) */
  int32_t nnz_lower;  /* strict-lower nonzeros (CSRC / CSRD sym) */
  int32_t width;      /* ELLPACK slots per row (faces per cell) */
  int32_t nrhs;
  int32_t unsym;      /* 1 when A != A^T */
  int32_t bandwidth;  /* max |i - j| over the nonzeros */
  int32_t pad;
  double velocity_scale; /* CONVDIFF: U that gives the requested Peclet */
} sfr_sys_info_t;

/* Build a system; returns an opaque handle or NULL on bad parameters. */
void *sfr_sys_build(const sfr_sys_params *p);
void sfr_sys_free(void *h);
int sfr_sys_info(const void *h, sfr_sys_info_t *out);

/* CSRD full: ia[neq+1], ja[nnz_full], al[nnz_full], ad[neq]. */
int sfr_sys_csrd_full(const void *h, int32_t *ia, int32_t *ja, double *al,
                      double *ad);
/* CSRD symmetric storage (strict lower): ia[neq+1], ja/al[nnz_lower]. */
int sfr_sys_csrd_lower(const void *h, int32_t *ia, int32_t *ja, double *al);
/* CSRC: ia[neq+1], ja[nnz_lower], a[2*nnz_lower] = al then au (the layout
 * solverC receives for unsym CSRC, HccaBlas.c:4233-4236). */
int sfr_sys_csrc(const void *h, int32_t *ia, int32_t *ja, double *a);
/* ELLPACK: ja[neq*width], a[neq*width] row-major. */
int sfr_sys_ell(const void *h, int32_t *ja, double *a);
/* Right-hand sides: b[nrhs*neq], RHS r at b + r*neq. */
int sfr_sys_rhs(const void *h, double *b);
/* new equation number of each natural cell id (i + nx*(j + ny*k)). */
int sfr_sys_numbering(const void *h, int32_t *eq_of_cell);

/* The box as the reference's mesh arrays: the geometry inputs of systFormDif
 * (CellLoop.c:285-311) with maxViz = 6 face slots per cell in the order
 * x-, x+, y-, y+, z-, z+ (the ELLPACK slot order above).  Cell arrays are
 * indexed by natural cell id; every index is 1-based as the reference stores
 * it.  Faces are oriented out of their owner (fOwner[2f], the minus-side
 * cell; the plus-side cell on a minus boundary).  Geometry:
 *   cell centre = mean of the 8 vertices; volume by 6 tetrahedra;
 *   face centre xm = mean of the 4 vertices; area vector
 *   0.5 (v2 - v0) x (v3 - v1); normal its unit vector;
 *   ksi = unit vector from the owner's centre to the neighbour's (to xm on
 *   the boundary), mksi its length; vSkew = (point where the centre line
 *   crosses the face plane) - xm, zero on the boundary; eta = unit first
 *   edge of the face; per cell slot xmcc = xm - centre and
 *   dcca = |xmcc . normal|. */
typedef struct {
  int32_t *nelcon;   /* numel*6: neighbour cell + 1, -1 on the boundary */
  int16_t *nviz;     /* numel: faces of the cell (6) */
  int32_t *cellface; /* numel*6: face id + 1 */
  double *volume;    /* numel */
  double *dcca;      /* numel*6 */
  double *xmcc;      /* numel*6*3 */
  double *cdiff;     /* numel: the cell diffusivity of the system */
  int32_t *id;       /* numel: equation + 1 */
  int32_t *owner;    /* nface*2: owner cell + 1, neighbour cell + 1 or -1 */
  double *mksi;      /* nface */
  double *ksi;       /* nface*3 */
  double *eta;       /* nface*3 */
  double *area;      /* nface */
  double *normal;    /* nface*3 */
  double *xm;        /* nface*3 */
  double *mvskew;    /* nface */
  double *vskew;     /* nface*3 */
} sfr_sys_mesh_t;

int sfr_sys_mesh_sizes(const void *h, int32_t *numel, int64_t *nface);
int sfr_sys_mesh(const void *h, const sfr_sys_mesh_t *m);

/* Reverse Cuthill-McKee of a symmetric graph given as CSR adjacency
 * (xadj[n+1], adj[]): perm[new] = old.  Returns 0 on success. */
int sfr_rcm(int32_t n, const int32_t *xadj, const int32_t *adj, int32_t *perm);

/* Draw the parameters of `count` uneven Poisson boxes: each axis
 * n = round(exp(U(ln nmin, ln nmax))), one random axis stretched by U(1,10),
 * constant diffusivity 10^U(-1,1), Dirichlet on one random face, RHS
 * U[-1,1], RCM numbering.  Seeds of the boxes derive from `seed`. */
int sfr_sys_batch_params(int32_t count, int32_t nmin, int32_t nmax,
                         uint64_t seed, sfr_sys_params *out);

#ifdef __cplusplus
}
#endif
#endif
