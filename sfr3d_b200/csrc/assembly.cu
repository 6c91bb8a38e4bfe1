// Device assembly: systFormDif (CellLoop.c:285-455) -> cellDif3D
// (CellDif.c:312-537) and systFormSimplePres (CellLoopInc.c:471-700) ->
// cellSimplePres3D (CellPres.c:903-1218), placing values as csr()/ellPack()
// do (Csr.c:549-1022, EllPack.c:113-149); ndf = 1, ndm = 3, one process.
//
// Every cell writes exactly one row (its own), so the assembly is one thread
// per equation with no atomics.  A plan binds the mesh to a system once, on
// the device:
//   - cells are put in equation order, so that the per-call reads of the
//     plan are coalesced and row r's outputs land at r;
//   - what the cell routines derive from the geometry alone (the
//     owner-signed ksi and normal, interpolFace's alpha, and for diffusion
//     |E| and the explicit part t of difusionSchemeNew) is computed once by
//     the same IEEE operations in the same order, so that the per-call
//     arithmetic starts from bit-identical values;
//   - the destination of each coefficient in the reference's raw value array
//     (al, al|au, or the ELLPACK slots) and in the solver's SELL copy is
//     resolved from the system's own pattern.
// A call then reads the plan (face-major, row-contiguous) and the per-cell
// fields, and writes al|au, ad and b where solverC reads them, plus the
// solver's SELL copy on full-row layouts.  All products, sums, divisions and
// square roots use explicitly rounded intrinsics (no contraction), in the
// reference's C evaluation order.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "common.cuh"
#include "internal.h"

namespace sfr {
namespace {

constexpr int kMaxViz = 8;        // face slots per cell handled
constexpr int kGeo = 9;           // geometry fields per (face, row): diffusion, pressure
constexpr int kGeoVel = 22;       // momentum
constexpr int kMaxLoads = 32;     // entries of the load table
constexpr int32_t kFlagP = 0x40000000;  // neighbour whose equation id is -1

// plan-time error codes (first one wins)
enum PlanError : int {
  kErrNone = 0,
  kErrNface = 1,
  kErrLibrary = 2,
  kErrId = 3,
  kErrIdTwice = 4,
  kErrFace = 5,
  kErrNeighbour = 6,
  kErrColumnTwice = 7,
  kErrLoad = 8,
  kErrWidth = 9,
};

const char *plan_error_text(int e) {
  switch (e) {
    case kErrNface: return "a cell's face count is outside 1..maxviz";
    case kErrLibrary: return "a cell's material does not use the diffusion cell library (calType 1)";
    case kErrId: return "an equation number is outside 1..neq";
    case kErrIdTwice: return "two cells carry the same equation number";
    case kErrFace: return "a cellFace entry or its owner is out of range";
    case kErrNeighbour: return "a neighbour index is neither a cell nor -1 (boundary)";
    case kErrColumnTwice: return "a row of the pattern holds the same column twice";
    case kErrLoad: return "a boundary face names a load outside 1..32";
    case kErrWidth: return "a cell has more faces than the ELLPACK row has slots";
  }
  return "unknown plan error";
}

struct MeshDev {
  int32_t numel, maxviz, nmat;
  int64_t nfaces;
  const int32_t *nelcon, *cellface, *owner, *id;
  const int16_t *nviz, *caltype, *mat, *facer;
  const int16_t *facevelr;  // pressure plans: the velocity loads of each face
  const double *volume, *dcca, *xmcc, *mksi, *ksi, *area, *normal, *vskew;
  const double *cc, *xm;    // momentum plans: cell centroids, face centres
};

struct PatternDev {
  const int32_t *sptr, *col, *src;
  int32_t n, storage, unsym, width;  // width: ELLPACK slots per row
};

struct PlanDev {
  int32_t n, maxviz;
  size_t fstride;       // maxviz * n: distance between geometry fields
  int32_t *cell;        // [n] cell assembling row r, -1 none
  int16_t *nface;       // [n]
  int32_t *nb;          // [maxviz][n] neighbour cell (| kFlagP), -1 bare boundary, -(load+2)
  int32_t *dst;         // [maxviz][n] raw value index, -1 none
  int32_t *sslot;       // [maxviz][n] slot of the value in row r of the SELL copy, -1 none
  double *geo;          // [kGeo][maxviz][n]
  double *vol;          // [n]
};

// The system's SELL copy, written directly when every stored value of a row
// comes from that row's own cell (full-row layouts): the assembly then also
// does what the value refresh would (the FP32 copy, the row compensation and
// the FP32 diagonal), in the same slot order.
struct FuseDev {
  double *val;
  float *val32;
  const int32_t *sptr;
  double *comp;
  float *diag32;
};

__device__ __forceinline__ double dot3(const double a[3], const double b[3]) {
  return xadd(xadd(xmul(a[0], b[0]), xmul(a[1], b[1])), xmul(a[2], b[2]));
}

__device__ __forceinline__ void flag_error(int *err, int code) { atomicCAS(err, 0, code); }

// difusionSchemeNew, ndm = 3 (CellLib.c:5824-6000)
__device__ void dif_scheme(int icod, const double s[3], const double k[3], double e[3],
                           double t[3]) {
  if (icod == 1) {  // ORTHOGONAL
    const double ss = xsqrt(dot3(s, s));
    for (int j = 0; j < 3; ++j) {
      e[j] = xmul(ss, k[j]);
      t[j] = 0.0;
    }
    return;
  }
  double tmp;
  if (icod == 2) {  // MINIMAL
    tmp = dot3(s, k);
  } else if (icod == 3) {  // ORTHOGONALC
    tmp = xsqrt(dot3(s, s));
  } else {  // OVERRELAXED
    tmp = xdiv(dot3(s, s), dot3(s, k));
  }
  for (int j = 0; j < 3; ++j) e[j] = xmul(tmp, k[j]);
  for (int j = 0; j < 3; ++j) t[j] = xsub(s[j], e[j]);
}

// column c of row r in the system's SELL copy -> index in the raw values
// (and the slot, in *slot); -1 absent, -3 present twice
__device__ int raw_index(const PatternDev &P, int r, int c, int *slot) {
  const int slice = r >> 5, lane = r & 31;
  const int beg = P.sptr[slice];
  const int w = (P.sptr[slice + 1] - beg) >> 5;
  int found = -1, hits = 0;
  *slot = -1;
  for (int j = 0; j < w; ++j) {
    const int e = beg + j * 32 + lane;
    if (P.col[e] == c && P.src[e] >= 0) {
      found = P.src[e];
      *slot = e;
      ++hits;
    }
  }
  return hits > 1 ? -3 : found;
}

// stored (non-padding) slots of row r
__device__ int real_slots(const PatternDev &P, int r) {
  const int slice = r >> 5, lane = r & 31;
  const int beg = P.sptr[slice];
  const int w = (P.sptr[slice + 1] - beg) >> 5;
  int k = 0;
  for (int j = 0; j < w; ++j) k += P.src[beg + j * 32 + lane] >= 0;
  return k;
}

// kind 0: diffusion (systFormDif) geometry [alpha, |E|, |ksi|, ksi, t];
// kind 1: pressure correction (systFormSimplePres) [alpha, area, |ksi|, ksi,
// normal], the anisotropic split being per call (it scales S by the face D).
// Boundary slots: [area, dcca, 0, normal, 0] (kind 0), [area, dcca, 0, ksi,
// normal] (kind 1).
__global__ void plan_kernel(MeshDev m, PatternDev P, PlanDev p, int icod, int kind, int *err,
                            unsigned *used_loads, int *free_cells, int *partial_rows,
                            unsigned *used_vel_loads) {
  const int nel = blockIdx.x * blockDim.x + threadIdx.x;
  if (nel >= m.numel) return;
  const int mv = m.maxviz;
  const int nf = m.nviz[nel];
  if (nf < 1 || nf > mv) return flag_error(err, kErrNface);
  const int16_t *fr = m.facer + static_cast<size_t>(nel) * (mv + 1);
  if (fr[nf] >= 1) {  // the cell's value is prescribed: no equation
    atomicAdd(free_cells, 1);
    return;
  }
  const int lm = m.mat[nel] - 1;
  if (lm < 0 || lm >= m.nmat || m.caltype[lm] != 1) return flag_error(err, kErrLibrary);
  const int row = m.id[nel] - 1;
  if (row < 0 || row >= P.n) return flag_error(err, kErrId);
  if (P.storage == SFR_ELLPACK && nf > P.width) return flag_error(err, kErrWidth);
  if (atomicCAS(p.cell + row, -1, nel) != -1) return flag_error(err, kErrIdTwice);
  p.nface[row] = static_cast<int16_t>(nf);
  p.vol[row] = m.volume[nel];
  const bool sym_lower = !P.unsym && P.storage != SFR_ELLPACK;
  int written = 0;  // SELL slots of row r this cell writes
  for (int f = 0; f < nf; ++f) {
    const size_t q = static_cast<size_t>(nel) * mv + f;
    const size_t o = static_cast<size_t>(f) * P.n + row;
    const int64_t face = static_cast<int64_t>(m.cellface[q]) - 1;
    if (face < 0 || face >= m.nfaces) return flag_error(err, kErrFace);
    const double ch = (m.owner[2 * face] - 1 == nel) ? 1.0 : -1.0;
    double ksi[3], nrm[3], g[kGeoVel];
    const int nfield = kind == 2 ? kGeoVel : kGeo;
    for (int k = kGeo; k < kGeoVel; ++k) g[k] = 0.0;
    for (int j = 0; j < 3; ++j) {
      ksi[j] = xmul(ch, m.ksi[3 * face + j]);
      nrm[j] = xmul(ch, m.normal[3 * face + j]);
    }
    const int viz = m.nelcon[q] - 1;
    int32_t nbv, dst = -1;
    int slot = -1;
    if (viz > -1) {
      if (viz >= m.numel) return flag_error(err, kErrNeighbour);
      const double area = m.area[face], mk = m.mksi[face];
      double v[3];
      // interpolFace, INTPOLFACELINEAR (CellLib.c:7174-7200)
      for (int j = 0; j < 3; ++j) v[j] = xadd(m.vskew[3 * face + j], m.xmcc[3 * q + j]);
      g[0] = xdiv(xsqrt(dot3(v, v)), mk);  // alpha
      g[2] = mk;
      if (kind != 1) {
        double s[3], e[3], t[3];
        for (int j = 0; j < 3; ++j) s[j] = xmul(area, nrm[j]);
        dif_scheme(icod, s, ksi, e, t);
        g[1] = xsqrt(dot3(e, e));  // |E|
        for (int j = 0; j < 3; ++j) {
          g[3 + j] = ksi[j];
          g[6 + j] = t[j];
        }
        if (kind == 2) {  // [9..11] normal, 12 area, [13..15] xmcc, [16..18] xm - c_V,
                          // [19..21] the face's skew vector (TVD)
          for (int j = 0; j < 3; ++j) {
            g[9 + j] = nrm[j];
            g[13 + j] = m.xmcc[3 * q + j];
            g[16 + j] = xsub(m.xm[3 * face + j], m.cc[3 * static_cast<size_t>(viz) + j]);
            g[19 + j] = m.vskew[3 * face + j];
          }
          g[12] = area;
        }
      } else {
        g[1] = area;
        for (int j = 0; j < 3; ++j) {
          g[3 + j] = ksi[j];
          g[6 + j] = nrm[j];
        }
      }
      const int lid = m.id[viz] - 1;
      nbv = viz | (lid == -2 ? kFlagP : 0);
      if (P.storage == SFR_ELLPACK) {
        dst = row * P.width + f;
        slot = P.sptr[row >> 5] + f * 32 + (row & 31);
      } else if (lid > -1 && !(sym_lower && lid > row)) {
        dst = raw_index(P, row, lid, &slot);
        if (dst == -3) return flag_error(err, kErrColumnTwice);
      }
    } else {
      if (viz != -2) return flag_error(err, kErrNeighbour);
      const int ld = fr[f];
      if (ld < 0 || ld > kMaxLoads) return flag_error(err, kErrLoad);
      if (ld > 0) atomicOr(used_loads, 1u << (ld - 1));
      g[0] = m.area[face];
      g[1] = m.dcca[q];
      g[2] = 0.0;
      if (kind == 0) {
        nbv = ld > 0 ? -(ld - 1) - 2 : -1;
        for (int j = 0; j < 3; ++j) {
          g[3 + j] = nrm[j];
          g[6 + j] = 0.0;
        }
      } else if (kind == 2) {  // faceVelR's load; [9..11] normal, 12 area, [13..15] xmcc
        nbv = ld > 0 ? -(ld - 1) - 2 : -1;
        for (int j = 0; j < 3; ++j) {
          g[3 + j] = ksi[j];
          g[6 + j] = 0.0;
          g[9 + j] = nrm[j];
          g[13 + j] = m.xmcc[3 * q + j];
        }
        g[12] = m.area[face];
      } else {
        const int lv = m.facevelr[static_cast<size_t>(nel) * (mv + 1) + f];
        if (lv < 0 || lv > kMaxLoads) return flag_error(err, kErrLoad);
        if (lv > 0) atomicOr(used_vel_loads, 1u << (lv - 1));
        nbv = -2 - (ld | (lv << 6));  // both loads of the face, 0 = none
        for (int j = 0; j < 3; ++j) {
          g[3 + j] = ksi[j];
          g[6 + j] = nrm[j];
        }
      }
      if (P.storage == SFR_ELLPACK) {
        dst = row * P.width + f;
        slot = P.sptr[row >> 5] + f * 32 + (row & 31);
      }
    }
    if (sym_lower) slot = -1;  // the row's mirrored slots come from other cells
    written += slot >= 0;
    p.nb[o] = nbv;
    p.dst[o] = dst;
    p.sslot[o] = slot;
    for (int k = 0; k < nfield; ++k) p.geo[k * p.fstride + o] = g[k];
  }
  if (sym_lower || written != real_slots(P, row)) atomicAdd(partial_rows, 1);
}

struct DevLoad {
  int32_t type;
  int32_t pad;
  double par[5];
  double par_last;  // par[np - 1]
  double density;   // Loads.density
};

struct CallOpts {
  int fres, time_flag, time_type, forces, matrix, calrcell;
  double dt, dt0;
};

// pLoad for constant loads (Loads.c:881-990)
__device__ __forceinline__ void apply_load(const DevLoad &L, double kc, double area, double dcca,
                                           const double n[3], double &sP, double &pp) {
  switch (L.type) {
    case 1: {  // DIRICHLETBC
      const double aP = xdiv(xmul(kc, area), dcca);
      sP = xadd(sP, aP);
      pp = xadd(pp, xmul(aP, L.par[0]));
      break;
    }
    case 3: {  // ROBINBC
      const double h = L.par[0];
      const double aP = xmul(xdiv(xmul(kc, h), xadd(kc, xmul(h, dcca))), area);
      sP = xadd(sP, aP);
      pp = xadd(pp, xmul(aP, L.par[1]));
      break;
    }
    case 2:  // NEUMANNBC
      pp = xadd(pp, xmul(area, L.par[0]));
      break;
    case 6: {  // INLET
      const double tA = L.par[0];
      double wfn = xadd(xmul(L.par[1], n[0]), xmul(L.par[2], n[1]));
      wfn = xadd(wfn, xmul(L.par[3], n[2]));
      pp = xsub(pp, xmul(xmul(xmul(wfn, L.par[4]), area), tA));
      const double aP = xdiv(xmul(kc, area), dcca);
      sP = xadd(sP, aP);
      pp = xadd(pp, xmul(aP, tA));
      break;
    }
    default:
      break;  // codes pLoad does not test add nothing
  }
}

// The row's coefficients (off-diagonals -la, diagonal d) where the reference's
// csr()/ellPack() put them, and, fused, the value refresh for the row: SELL
// values, their FP32 copy, the FP32 diagonal and the compensation summed in
// slot order as the refresh sums it.
template <int kMV, bool kFused>
__device__ __forceinline__ void write_row(const FuseDev &fu, int r, int nf, const double (&la)[kMV],
                                          double d, const int32_t (&dsts)[kMV],
                                          const int32_t (&slots)[kMV], double *stage,
                                          double *diag) {
  diag[r] = d;
#pragma unroll
  for (int f = 0; f < kMV; ++f)
    if (f < nf && dsts[f] >= 0) stage[dsts[f]] = xmul(la[f], -1.0);
  if (kFused) {
    fu.diag32[r] = __double2float_rn(d);
    const int base = fu.sptr[r >> 5] + (r & 31);
    double acc = 0.0;
#pragma unroll
    for (int k = 0; k < kMV; ++k)
#pragma unroll
      for (int f = 0; f < kMV; ++f)
        if (f < nf && slots[f] == base + 32 * k) {
          const double v = xmul(la[f], -1.0);
          const float v32 = __double2float_rn(v);
          fu.val[slots[f]] = v;
          fu.val32[slots[f]] = v32;
          acc = xadd(acc, xsub(static_cast<double>(v32), v));
        }
    fu.comp[r] = -acc;
  }
}

// One row of cellDif3D.  kOrth: ORTHOGONAL scheme, whose explicit part t is
// zero, so the non-orthogonal correction adds coef * (+-0) to a force that
// can never be -0: it changes nothing for finite fields and is skipped
// (gradu0 is not read).  kMV: face slots of the plan (maxviz rounded up to
// 6 or 8); every slot is read, unused ones hold a bare-boundary marker, so
// that all of a row's loads are issued before the first is used.
template <bool kOrth, int kMV, bool kFused>
__global__ void __launch_bounds__(256)
    dif_assemble_kernel(PlanDev p, FuseDev fu, const DevLoad *__restrict__ loads, CallOpts o,
                        const double *__restrict__ density, const double *__restrict__ cdiff,
                        const double *__restrict__ u0, const double *__restrict__ gradu0,
                        const double *__restrict__ b0, double *__restrict__ stage,
                        double *__restrict__ diag, double *__restrict__ b,
                        double *__restrict__ rcell) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= p.n) return;
  const int cell = __ldcs(p.cell + r);
  if (cell < 0) return;
  const int nf = __ldcs(p.nface + r);
  const size_t fs = p.fstride;
  int32_t nbs[kMV], dsts[kMV];
  double alpha[kMV], modE[kMV], mk[kMV], kn[kMV], un[kMV];
#pragma unroll
  for (int f = 0; f < kMV; ++f) {
    const size_t q = static_cast<size_t>(f) * p.n + r;
    nbs[f] = __ldcs(p.nb + q);
    alpha[f] = __ldcs(p.geo + q);
    modE[f] = __ldcs(p.geo + fs + q);
    mk[f] = __ldcs(p.geo + 2 * fs + q);
  }
  const double kc = cdiff[cell], uc = u0[cell];
#pragma unroll
  for (int f = 0; f < kMV; ++f) {
    const int c = nbs[f] >= 0 ? (nbs[f] & (kFlagP - 1)) : cell;
    kn[f] = cdiff[c];
    un[f] = u0[c];
  }
  int32_t slots[kMV];
  if (o.matrix) {
#pragma unroll
    for (int f = 0; f < kMV; ++f) {
      dsts[f] = __ldcs(p.dst + static_cast<size_t>(f) * p.n + r);
      slots[f] = kFused ? __ldcs(p.sslot + static_cast<size_t>(f) * p.n + r) : -1;
    }
  }
  double gp[3] = {0.0, 0.0, 0.0};
  if (!kOrth)
    for (int j = 0; j < 3; ++j) gp[j] = gradu0[3 * static_cast<size_t>(cell) + j];
  double la[kMV];
  double pp = 0.0, sP = 0.0;
#pragma unroll
  for (int f = 0; f < kMV; ++f) {
    la[f] = 0.0;
    if (f >= nf) continue;
    const int32_t nb = nbs[f];
    if (nb >= 0) {
      const double am1 = xsub(1.0, alpha[f]);
      double coef = xadd(xdiv(alpha[f], kc), xdiv(am1, kn[f]));
      coef = xdiv(1.0, coef);
      la[f] = xdiv(xmul(coef, modE[f]), mk[f]);
      if (!kOrth) {
        const size_t q = static_cast<size_t>(f) * p.n + r;
        const int c = nb & (kFlagP - 1);
        const double duDksi = xdiv(xsub(un[f], uc), mk[f]);
        double k[3], t[3], gf[3], gc[3];
        for (int j = 0; j < 3; ++j) {
          k[j] = __ldcs(p.geo + (3 + j) * fs + q);
          t[j] = __ldcs(p.geo + (6 + j) * fs + q);
          gf[j] = xadd(xmul(am1, gp[j]),
                       xmul(alpha[f], gradu0[3 * static_cast<size_t>(c) + j]));
        }
        const double du = xsub(duDksi, dot3(gf, k));
        for (int j = 0; j < 3; ++j) gc[j] = xadd(gf[j], xmul(du, k[j]));
        pp = xadd(pp, xmul(coef, dot3(gc, t)));
      }
    } else if (nb <= -2) {
      // boundary slot: alpha holds the area, modE the centre-face distance
      const size_t q = static_cast<size_t>(f) * p.n + r;
      double n[3] = {0.0, 0.0, 0.0};
      const DevLoad &L = loads[-nb - 2];
      if (L.type == 6)
        for (int j = 0; j < 3; ++j) n[j] = __ldcs(p.geo + (3 + j) * fs + q);
      apply_load(L, kc, alpha[f], modE[f], n, sP, pp);
    }
  }
  // implicit time term, CellDif.c:485-497
  if (o.time_flag) {
    const double rho = density[cell], vol = p.vol[r];
    if (o.time_type == 0) {
      sP = xadd(sP, xdiv(xmul(rho, vol), o.dt));
    } else if (o.time_type == 1) {
      const double tmp = xadd(xdiv(1.0, o.dt), xdiv(1.0, xadd(o.dt, o.dt0)));
      sP = xadd(sP, xmul(xmul(tmp, rho), vol));
    }
  }
  double d = sP;
#pragma unroll
  for (int f = 0; f < kMV; ++f)
    if (f < nf) d = xadd(d, la[f]);
  double rr = 0.0;
#pragma unroll
  for (int f = 0; f < kMV; ++f)
    if (f < nf && nbs[f] >= 0) {
      if (nbs[f] & kFlagP)
        pp = xadd(pp, xmul(la[f], un[f]));
      else
        rr = xadd(rr, xmul(la[f], un[f]));
    }
  rr = xadd(rr, xsub(pp, xmul(d, uc)));
  const double bb = b0 ? b0[r] : 0.0;
  if (o.forces) {
    const double lb = o.fres ? rr : pp;
    b[r] = b0 ? xadd(lb, bb) : lb;
  }
  if (o.calrcell) rcell[cell] = b0 ? xadd(rr, bb) : rr;
  if (o.matrix) write_row<kMV, kFused>(fu, r, nf, la, d, dsts, slots, stage, diag);
}

// difusionSchemeAnisotropic, ndm = 3 (CellLib.c:6054-6170): ORTHOGONAL or
// OVERRELAXED (the only two that set e and t)
template <bool kOver>
__device__ __forceinline__ void pres_split(const double s[3], const double k[3], double e[3],
                                           double t[3]) {
  if (!kOver) {
    const double ss = xsqrt(dot3(s, s));
    for (int j = 0; j < 3; ++j) {
      e[j] = xmul(ss, k[j]);
      t[j] = 0.0;
    }
  } else {
    const double tmp = xdiv(dot3(s, s), dot3(s, k));
    for (int j = 0; j < 3; ++j) e[j] = xmul(tmp, k[j]);
    for (int j = 0; j < 3; ++j) t[j] = xsub(s[j], e[j]);
  }
}

// pLoadSimplePres with fCal and no buoyancy (Loads.c:728-845): a pressure
// load's share of the diagonal
__device__ __forceinline__ void pres_load(const DevLoad &L, const double e[3], const double n[3],
                                          const double vc[3], double rhoC, double area,
                                          double dd, double &sP) {
  const double modE = xsqrt(dot3(e, e));
  if (L.type == 1) {  // DIRICHLETBC
    sP = xadd(sP, xdiv(xmul(rhoC, modE), dd));
  } else if (L.type == 13) {  // INLETTOTALPRES
    const double rhoEnv = L.par[0];
    const double dc = xdiv(modE, dd);
    const double ev[3] = {L.par[2], L.par[3], L.par[4]};
    double tmp0 = dot3(vc, n);
    double tmp1 = xmul(dot3(ev, n), area);
    const double m = xmul(xmul(rhoEnv, tmp0), area);
    const double modVel = xdiv(m, xmul(rhoEnv, tmp1));
    tmp0 = xmul(rhoEnv, modVel);
    tmp1 = xsub(m, xmul(xmul(dc, tmp0), tmp0));
    sP = xadd(sP, xdiv(xmul(xmul(rhoEnv, m), dc), tmp1));
  } else if (L.type == 10) {  // OPEN: outflow only, added twice as the reference does
    if (dot3(vc, n) > 0.0) {
      const double a = xdiv(xmul(rhoC, modE), dd);
      sP = xadd(sP, a);
      sP = xadd(sP, a);
    }
  }
}

// pLoadSimple with fCalVel = false, fCalPres = true (Loads.c:265-720): a
// velocity load's mass flux in the pressure equation
__device__ __forceinline__ void vel_load(const DevLoad &L, const double n[3], const double vc[3],
                                         double rhoC, double area, double &pp) {
  double m;
  switch (L.type) {
    case 7:   // OUTLET
    case 9:   // INLETSTAICTPRES
      m = xmul(xmul(rhoC, dot3(vc, n)), area);
      break;
    case 6: {  // INLET: prescribed velocity par[0..2], density par[np - 1]
      const double t[3] = {L.par[0], L.par[1], L.par[2]};
      m = xmul(xmul(L.par_last, dot3(t, n)), area);
      break;
    }
    case 10: {  // OPEN
      const double wfn = dot3(vc, n);
      m = xmul(xmul(wfn >= 0.0 ? rhoC : L.density, wfn), area);
      break;
    }
    case 13:  // INLETTOTALPRES
      m = xmul(xmul(L.par[0], dot3(vc, n)), area);
      break;
    default:
      return;  // walls and the rest: nothing in the pressure equation
  }
  pp = xsub(pp, m);
}

struct PresOpts {
  int forces, matrix, calrcell;
};

// One row of cellSimplePres3D (CellPres.c:903-1218).  kOver: the
// OVERRELAXED anisotropic split (else ORTHOGONAL).  loads: [0, 32) pressure
// loads, [32, 64) velocity loads; dens: density of each material.
template <bool kOver, int kMV, bool kFused>
__global__ void __launch_bounds__(256, 2)
    pres_assemble_kernel(PlanDev p, FuseDev fu, const DevLoad *__restrict__ loads, PresOpts o,
                         const int16_t *__restrict__ mat, const double *__restrict__ dens,
                         const double *__restrict__ pres, const double *__restrict__ gradp,
                         const double *__restrict__ vel, const double *__restrict__ dfield,
                         double *__restrict__ stage, double *__restrict__ diag,
                         double *__restrict__ b, double *__restrict__ rcell) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= p.n) return;
  const int cell = __ldcs(p.cell + r);
  if (cell < 0) return;
  const int nf = __ldcs(p.nface + r);
  const size_t fs = p.fstride;
  int32_t nbs[kMV], dsts[kMV], slots[kMV];
  double alpha[kMV], area[kMV], mk[kMV];
#pragma unroll
  for (int f = 0; f < kMV; ++f) {
    const size_t q = static_cast<size_t>(f) * p.n + r;
    nbs[f] = __ldcs(p.nb + q);
    alpha[f] = __ldcs(p.geo + q);
    area[f] = __ldcs(p.geo + fs + q);
    mk[f] = __ldcs(p.geo + 2 * fs + q);
  }
  const size_t c3 = 3 * static_cast<size_t>(cell);
  const double rhoC = dens[mat[cell] - 1], presC = pres[cell];
  const double vc[3] = {vel[c3], vel[c3 + 1], vel[c3 + 2]};
  const double gpc[3] = {gradp[c3], gradp[c3 + 1], gradp[c3 + 2]};
  const double dc[3] = {dfield[c3], dfield[c3 + 1], dfield[c3 + 2]};
  double la[kMV];
  double pp = 0.0, sP = 0.0;
#pragma unroll
  for (int f = 0; f < kMV; ++f) {
    la[f] = 0.0;
    if (f >= nf) continue;
    const int32_t nb = nbs[f];
    const size_t q = static_cast<size_t>(f) * p.n + r;
    double k[3], n[3], s[3], e[3], t[3];
    for (int j = 0; j < 3; ++j) {
      k[j] = __ldcs(p.geo + (3 + j) * fs + q);
      n[j] = __ldcs(p.geo + (6 + j) * fs + q);
    }
    if (nb >= 0) {
      const size_t v3 = 3 * static_cast<size_t>(nb & (kFlagP - 1));
      const int c = nb & (kFlagP - 1);
      const double a = alpha[f], am1 = xsub(1.0, a);
      const double rho = xadd(xmul(am1, rhoC), xmul(a, dens[mat[c] - 1]));
      double dF[3], wf[3], gf[3];
      for (int j = 0; j < 3; ++j) {
        dF[j] = xadd(xmul(am1, dc[j]), xmul(a, dfield[v3 + j]));
        s[j] = xmul(xmul(dF[j], area[f]), n[j]);
        wf[j] = xadd(xmul(am1, vc[j]), xmul(a, vel[v3 + j]));
        gf[j] = xadd(xmul(am1, gpc[j]), xmul(a, gradp[v3 + j]));
      }
      pres_split<kOver>(s, k, e, t);
      la[f] = xdiv(xmul(rho, xsqrt(dot3(e, e))), mk[f]);
      // interpolFaceVel, ndm = 3 (CellLib.c:6853-6960): Rhie-Chow face velocity
      double wfn = dot3(wf, n);
      const double g0 = xdiv(xsub(pres[c], presC), mk[f]);
      const double nk = xadd(xadd(xmul(xmul(dF[0], k[0]), n[0]), xmul(xmul(dF[1], k[1]), n[1])),
                             xmul(xmul(dF[2], k[2]), n[2]));
      const double g1 = xmul(xsub(dot3(gf, k), g0), nk);
      wfn = xadd(wfn, g1);
      pp = xsub(pp, xmul(xmul(rho, wfn), area[f]));
    } else {
      const int code = -nb - 2;
      const int lp = code & 63, lv = code >> 6;
      if (lp) {
        for (int j = 0; j < 3; ++j) s[j] = xmul(xmul(dc[j], alpha[f]), n[j]);
        pres_split<kOver>(s, k, e, t);
        pres_load(loads[lp - 1], e, n, vc, rhoC, alpha[f], area[f], sP);
      }
      if (lv) vel_load(loads[kMaxLoads + lv - 1], n, vc, rhoC, alpha[f], pp);
    }
  }
  double d = sP;
#pragma unroll
  for (int f = 0; f < kMV; ++f)
    if (f < nf) d = xadd(d, la[f]);
  if (o.forces) b[r] = pp;
  if (o.calrcell) rcell[cell] = pp;
  if (!o.matrix) return;
#pragma unroll
  for (int f = 0; f < kMV; ++f) {  // loaded late: fewer live registers in the face loop
    dsts[f] = __ldcs(p.dst + static_cast<size_t>(f) * p.n + r);
    slots[f] = kFused ? __ldcs(p.sslot + static_cast<size_t>(f) * p.n + r) : -1;
  }
  write_row<kMV, kFused>(fu, r, nf, la, d, dsts, slots, stage, diag);
}

struct VelOpts {
  int fso, fvisc, fres, simplec, time_flag, time_type, forces, matrix, calrcell;
  double dt, dt0, under;
  int adv;  // 1 FoUp, 2 CD, 3 SoUp, 6 LUST
  int fturb, fstruc;
  const double *eddy, *stress;  // numel, numel*6 (device)
  double beta;  // LUST weight
  int nvd;      // NVD function
  int fwall;    // the wall model's viscosity on walls
  const double *wall;  // numel*4: yPlus, uPlus, uFri, stressW (device)
  int rhie;     // Rhie-Chow face velocity, D from the call's start
  const double *dold;  // numel*3: that D (a copy made before the launch)
};

// nvd (CellLib.c): the two weights of an NVD function at phi~; the
// reference's table, MUSCL and STOIC left at (0, 0) as it leaves them
__host__ __device__ inline void nvd_weights(double ph, int fn, double *p0, double *p1) {
  constexpr double k13 = 3.33333333333333333333E-1, k23 = 6.66666666666666666666E-1;
  double a = 1.0, b = 0.0;
  switch (fn) {
    case 1: if (ph >= 0 && ph <= 1.0) { a = 0.5; b = 0.5; } break;
    case 3:
      if (ph >= 0 && ph <= 5.0 / 6.0) { a = 3.0 / 4.0; b = 3.0 / 8.0; }
      else if (ph > 5.0 / 6.0 && ph <= 1.0) { a = 0.0; b = 1.0; }
      break;
    case 4:
      if (ph >= 0 && ph <= 1.0 / 6.0) { a = 3.0; b = 0.0; }
      else if (ph > 1.0 / 6.0 && ph <= 0.7) { a = 3.0 / 4.0; b = 3.0 / 8.0; }
      else if (ph > 0.7 && ph <= 1.0) { a = k13; b = k23; }
      break;
    case 5:
      if (ph >= 0 && ph <= 0.5) { a = 0.5; b = 0.5; }
      else if (ph > 0.5 && ph <= k23) { a = 1.5; b = 0.0; }
      else if (ph > k23 && ph <= 1.0) { a = 0.0; b = 1.0; }
      break;
    case 6:
      if (ph >= 0 && ph <= k13) { a = 2.0; b = 0.0; }
      else if (ph > k13 && ph <= 0.5) { a = 0.5; b = 0.5; }
      else if (ph > 0.5 && ph <= k23) { a = 1.5; b = 0.0; }
      else if (ph > k23 && ph <= 1.0) { a = 0.0; b = 1.0; }
      break;
    case 8:
      if (ph >= 0 && ph <= 0.5) { a = 1.5; b = 0.0; }
      else if (ph > 0.5 && ph <= 1.0) { a = 0.5; b = 0.5; }
      break;
    case 9:
      if (ph >= 0 && ph <= 0.25) { a = 2.5; b = 0.0; }
      else if (ph > 0.25 && ph <= 1.0) { a = 0.5; b = 0.5; }
      break;
    default: a = 0.0; b = 0.0; break;  // 2 MUSCL, 7 STOIC
  }
  *p0 = a;
  *p1 = b;
}


// turbStructIntegral (CellLib.c:7586-7626): p -= area (s n), s the face's
// residual stress without its trace (interior: g1 Rc + g2 Rv)
__device__ __noinline__ void struct_integral(const double *rc, const double *rv,
                                                const double n[3], double p[3], double area,
                                                double g1, double g2) {
  constexpr double kThird = 3.33333333333333333333E-1;
  double s[6];
  if (!rv) {
    const double tmp = xmul(kThird, xadd(xadd(rc[0], rc[1]), rc[2]));
    for (int k = 0; k < 3; ++k) s[k] = xsub(rc[k], tmp);
    for (int k = 3; k < 6; ++k) s[k] = rc[k];
  } else {
    for (int k = 0; k < 6; ++k) s[k] = xadd(xmul(g1, rc[k]), xmul(g2, rv[k]));
    const double tmp = xmul(kThird, xadd(xadd(s[0], s[1]), s[2]));
    for (int k = 0; k < 3; ++k) s[k] = xsub(s[k], tmp);
  }
  const double r0[3] = {s[0], s[3], s[5]}, r1[3] = {s[3], s[1], s[4]}, r2[3] = {s[5], s[4], s[2]};
  p[0] = xsub(p[0], xmul(area, dot3(r0, n)));
  p[1] = xsub(p[1], xmul(area, dot3(r1, n)));
  p[2] = xsub(p[2], xmul(area, dot3(r2, n)));
}

// moveWall, not Dirichlet (CellLib.c:7715-7770)
__device__ __forceinline__ void move_wall(const double vC[3], const double vB[3],
                                          const double n[3], double sPc[3], double p[3],
                                          double dcca, double visc, double area) {
  const double aP = xdiv(xmul(visc, area), dcca);
  double w[3];
  for (int k = 0; k < 3; ++k) {
    w[k] = xsub(1.0, xmul(n[k], n[k]));
    sPc[k] = xadd(sPc[k], xmul(aP, w[k]));
  }
  // p_k += aP (vB_k (1 - n_k n_k) + (vC_a - vB_a) n_a n_k + (vC_b - vB_b) n_b n_k),
  // a < b the two other components in increasing order
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const int a = k == 0 ? 1 : 0, b = k == 2 ? 1 : 2;
    const double t1 = xmul(vB[k], w[k]);
    const double t2 = xmul(xmul(xsub(vC[a], vB[a]), n[a]), n[k]);
    const double t3 = xmul(xmul(xsub(vC[b], vB[b]), n[b]), n[k]);
    p[k] = xadd(p[k], xmul(aP, xadd(xadd(t1, t2), t3)));
  }
}

// One row of cellSimpleVel3D (CellSimple.c:106-727), laminar, first-order
// upwind, face velocity without Rhie-Chow; three diagonals and forces.
// mtab: density then viscosity of each material.
// The deferred correction of advectiveScheme (CellLib.c:6394-6480) with cv
// in the place of wfn: CD deferredCd (CellLib.c:5113); SoUp upwindLinearV1
// (CellLib.c:5072) from the upwind cell's gradient, r = xm - cc (plan words
// 13-15 for this cell, 16-18 for the neighbour).  Out of line: the main
// path keeps its registers.
__device__ __noinline__ void advection_correction(int adv, double cv, double am1, double alpha,
                                                  double beta, int nvd, const double velC[3],
                                                  const double velV[3], const double gvC[9],
                                                  const double *gvV, const double *g, size_t fs,
                                                  double cvc[3]) {
  if (adv == 2) {
    for (int i = 0; i < 3; ++i)
      cvc[i] = xsub(xadd(xmul(am1, velC[i]), xmul(alpha, velV[i])), cv < 0.0 ? velV[i] : velC[i]);
  } else if (adv == 3) {
    double rr[3];
    const bool down = cv < 0.0;
    for (int j = 0; j < 3; ++j) rr[j] = __ldcs(g + ((down ? 16 : 13) + j) * fs);
    for (int i = 0; i < 3; ++i) {
      double gu[3];
      for (int j = 0; j < 3; ++j) gu[j] = down ? gvV[3 * i + j] : gvC[3 * i + j];
      cvc[i] = dot3(gu, rr);
    }
  } else if (adv == 4) {  // faceBaseTvdV1 (CellLib.c:4845-4875) with limitFaceBase
    double ksi[3];
    for (int j = 0; j < 3; ++j) ksi[j] = __ldcs(g + (3 + j) * fs);
    const double mk = __ldcs(g + 2 * fs);
    const bool down = cv < 0.0;
    for (int i = 0; i < 3; ++i) {
      const double du = xadd(down ? xsub(velC[i], velV[i]) : xsub(velV[i], velC[i]), 1.e-14);
      const double gf0 = dot3(down ? gvV + 3 * i : gvC + 3 * i, ksi);
      const double gf = xmul(xmul(down ? -2.0 : 2.0, gf0), mk);
      const double r = xsub(xdiv(gf, du), 1.0);
      double lim = 0.0;  // limitFaceBase (CellLib.c:4482-4530); min/max as Define.h:455-456
      if (nvd == 1) {
        const double a = fabs(r);
        lim = xdiv(xadd(r, a), xadd(1.0, a));
      } else if (nvd == 2) {
        if (r > 0.0) {
          const double a = xmul(r, r);
          lim = xdiv(xadd(r, a), xadd(1.0, a));
        }
      } else if (nvd == 3 || nvd == 4) {
        const double cap = nvd == 3 ? 1.0 : 2.0, mn = r < cap ? r : cap;
        lim = 0.0 > mn ? 0.0 : mn;
      } else if (nvd == 5) {
        const double r2 = xmul(2.0, r);
        const double a = r2 < 1.0 ? r2 : 1.0, b = r < 2.0 ? r : 2.0, c = a > b ? a : b;
        lim = 0.0 > c ? 0.0 : c;
      }
      cvc[i] = xmul(xmul(0.5, lim), du);
    }
  } else if (adv == 5) {  // faceBaseNvd (CellLib.c:4900-4937), the cell as uP
    double ksi[3];
    for (int j = 0; j < 3; ++j) ksi[j] = __ldcs(g + (3 + j) * fs);
    const double mk = __ldcs(g + 2 * fs);
    const bool down = cv < 0.0;
    for (int i = 0; i < 3; ++i) {
      const double uP = velC[i], uV = velV[i];
      const double gf0 = dot3(down ? gvV + 3 * i : gvC + 3 * i, ksi);
      const double gf = xadd(xmul(xmul(down ? -2.0 : 2.0, gf0), mk), 1.e-32);
      const double phi = xadd(xdiv(down ? xsub(uV, uP) : xsub(uP, uV), gf), 1.0);
      double p0, p1;
      nvd_weights(phi, nvd, &p0, &p1);
      const double a = down ? uV : uP, b = down ? uP : uV;
      cvc[i] = xadd(xadd(xmul(xsub(p0, 1.0), a), xmul(p1, b)),
                    xmul(xsub(xsub(1.0, p0), p1), xsub(b, gf)));
    }
  } else if (adv == 6) {  // deferredLust (CellLib.c:5162-5198)
    double rC[3], rV[3];
    for (int j = 0; j < 3; ++j) {
      rC[j] = __ldcs(g + (13 + j) * fs);
      rV[j] = __ldcs(g + (16 + j) * fs);
    }
    const bool down = cv < 0.0;
    for (int i = 0; i < 3; ++i) {
      const double *gc = gvC + 3 * i, *gv = gvV + 3 * i;
      const double up = down ? velV[i] : velC[i];
      const double ul = xadd(up, down ? dot3(gv, rV) : dot3(gc, rC));
      double uf1 = xadd(xadd(velC[i], xmul(gc[0], rC[0])), xmul(gc[1], rC[1]));
      double uf2 = xadd(xadd(velV[i], xmul(gv[0], rV[0])), xmul(gv[1], rV[1]));
      uf1 = xadd(uf1, xmul(gc[2], rC[2]));
      uf2 = xadd(uf2, xmul(gv[2], rV[2]));
      const double cd = xadd(xmul(am1, uf1), xmul(alpha, uf2));
      cvc[i] = xsub(xadd(xmul(beta, ul), xmul(xsub(1.0, beta), cd)), up);
    }
  }
}

// kExt: the deferred advection corrections and the turbulence fields; the
// laminar first-order-upwind instantiation carries none of that code.
template <int kMV, bool kExt>
__global__ void __launch_bounds__(256, 2)
    vel_assemble_kernel(PlanDev p, const DevLoad *__restrict__ loads, VelOpts o,
                        const int16_t *__restrict__ mat, const double *__restrict__ mtab, int nmat,
                        const double *__restrict__ pres, const double *__restrict__ gradp,
                        const double *__restrict__ vel, const double *__restrict__ gradvel,
                        double *__restrict__ dfield, double *__restrict__ stage,
                        double *__restrict__ diag, double *__restrict__ ad3,
                        double *__restrict__ b3, double *__restrict__ rcell3, int numel) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= p.n) return;
  const int cell = __ldcs(p.cell + r);
  if (cell < 0) return;
  const int nf = __ldcs(p.nface + r);
  const size_t fs = p.fstride;
  const int mc = mat[cell] - 1;
  const double rhoC = mtab[mc], muC = mtab[nmat + mc];
  const double effC = xadd(muC, kExt && o.fturb ? o.eddy[cell] : 0.0);
  const size_t c3 = 3 * static_cast<size_t>(cell), c9 = 9 * static_cast<size_t>(cell);
  const double presC = pres[cell];
  double velC[3], gpC[3], gvC[9];
  for (int k = 0; k < 3; ++k) {
    velC[k] = vel[c3 + k];
    gpC[k] = gradp[c3 + k];
  }
  for (int k = 0; k < 9; ++k) gvC[k] = gradvel[c9 + k];
  double pp[3] = {0.0, 0.0, 0.0}, pf[3] = {0.0, 0.0, 0.0}, sPc[3] = {0.0, 0.0, 0.0};
  double sP = 0.0, la[kMV];
#pragma unroll
  for (int f = 0; f < kMV; ++f) {
    la[f] = 0.0;
    if (f >= nf) continue;
    const size_t q = static_cast<size_t>(f) * p.n + r;
    const int32_t nb = __ldcs(p.nb + q);
    const double *g = p.geo + q;
    double n[3];
    for (int j = 0; j < 3; ++j) n[j] = __ldcs(g + (9 + j) * fs);
    const double area = __ldcs(g + 12 * fs);
    if (nb >= 0) {
      const int c = nb & (kFlagP - 1);
      const size_t v3 = 3 * static_cast<size_t>(c), v9 = 9 * static_cast<size_t>(c);
      const int mv = mat[c] - 1;
      const double rhoV = mtab[mv],
                   effV = xadd(mtab[nmat + mv], kExt && o.fturb ? o.eddy[c] : 0.0);
      const double alpha = __ldcs(g), modE = __ldcs(g + fs), mk = __ldcs(g + 2 * fs);
      const double am1 = xsub(1.0, alpha);
      double ksi[3], t[3], velV[3], wf[3];
      for (int j = 0; j < 3; ++j) {
        ksi[j] = __ldcs(g + (3 + j) * fs);
        t[j] = __ldcs(g + (6 + j) * fs);
        velV[j] = vel[v3 + j];
        wf[j] = xadd(xmul(am1, velC[j]), xmul(alpha, velV[j]));
      }
      // mediaHarmonica (CellLib.c:7879)
      const double visc = (effC == 0.0 || effV == 0.0)
                              ? 0.0
                              : xdiv(1.0, xadd(xdiv(alpha, effC), xdiv(am1, effV)));
      const double dfd = xdiv(xmul(visc, modE), mk);
      const double density = xadd(xmul(am1, rhoC), xmul(alpha, rhoV));
      double wfn = dot3(wf, n);
      if (kExt && o.rhie) {
        // interpolFaceVel, ndm = 3 (CellLib.c:6853-6960) with the face D of
        // CellSimple.c:339-350, both D values as they were at the call's start
        double dF[3], gp[3];
        for (int j = 0; j < 3; ++j) {
          dF[j] = xadd(xmul(am1, o.dold[c3 + j]), xmul(alpha, o.dold[v3 + j]));
          gp[j] = xadd(xmul(am1, gpC[j]), xmul(alpha, gradp[v3 + j]));
        }
        const double g0 = xdiv(xsub(pres[c], presC), mk);
        const double nk = xadd(xadd(xmul(xmul(dF[0], ksi[0]), n[0]), xmul(xmul(dF[1], ksi[1]), n[1])),
                               xmul(xmul(dF[2], ksi[2]), n[2]));
        wfn = xadd(wfn, xmul(xsub(dot3(gp, ksi), g0), nk));
      }
      const double cv = xmul(xmul(density, wfn), area);
      la[f] = xsub(dfd, cv < 0.0 ? cv : 0.0);
      sP = xadd(sP, cv);
      // advectiveScheme (CellLib.c:6394-6480) with cv in the place of wfn:
      // FoUp cvc = 0; CD deferredCd (CellLib.c:5113); SoUp upwindLinearV1
      // (CellLib.c:5072) from the upwind cell's gradient, r = xm - cc
      double cvc[3] = {0.0, 0.0, 0.0};
      if (kExt && o.adv != 1)
        advection_correction(o.adv, cv, am1, alpha, o.beta, o.nvd, velC, velV, gvC, gradvel + v9,
                             g, fs, cvc);
      double gvc[9];
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        double gf[3];
        for (int j = 0; j < 3; ++j)
          gf[j] = xadd(xmul(am1, gvC[3 * i + j]), xmul(alpha, gradvel[v9 + 3 * i + j]));
        const double du = xsub(xdiv(xsub(velV[i], velC[i]), mk), dot3(gf, ksi));
        for (int j = 0; j < 3; ++j) gvc[3 * i + j] = xadd(gf[j], xmul(du, ksi[j]));
        const double dfdc = xmul(visc, dot3(gvc + 3 * i, t));
        if (kExt && o.adv == 4) {  // TVD: minus the compact gradient along the skew vector
          const double vs[3] = {__ldcs(g + 19 * fs), __ldcs(g + 20 * fs), __ldcs(g + 21 * fs)};
          cvc[i] = xsub(cvc[i], dot3(gvc + 3 * i, vs));
        }
        pp[i] = xadd(pp[i], xsub(dfdc, xmul(cv, cvc[i])));  // p += dfdc - cv cvc
      }
      // facePressure (CellLib.c:7499), interior
      double pFace;
      if (o.fso) {
        double xmcc[3], vv[3], gpV[3];
        for (int j = 0; j < 3; ++j) {
          xmcc[j] = __ldcs(g + (13 + j) * fs);
          vv[j] = __ldcs(g + (16 + j) * fs);
          gpV[j] = gradp[v3 + j];
        }
        double p1 = xadd(presC, xmul(gpC[0], xmcc[0]));
        p1 = xadd(p1, xmul(gpC[1], xmcc[1]));
        p1 = xadd(p1, xmul(gpC[2], xmcc[2]));
        double p2 = xadd(pres[c], xmul(gpV[0], vv[0]));
        p2 = xadd(p2, xmul(gpV[1], vv[1]));
        p2 = xadd(p2, xmul(gpV[2], vv[2]));
        pFace = xmul(0.5, xadd(p1, p2));
      } else {
        pFace = xadd(xmul(am1, presC), xmul(alpha, pres[c]));
      }
      const double tmp = xmul(pFace, area);
      for (int j = 0; j < 3; ++j) pf[j] = xadd(pf[j], xmul(tmp, n[j]));
      // viscosityPartExp (CellLib.c:7439), fDiv false
      if (o.fvisc) {
        const double aP = xmul(muC, area);
        for (int i = 0; i < 3; ++i) {
          const double col[3] = {gvc[i], gvc[3 + i], gvc[6 + i]};
          pp[i] = xadd(pp[i], xmul(aP, dot3(col, n)));
        }
      }
      if (kExt && o.fstruc)
        struct_integral(o.stress + 6 * static_cast<size_t>(cell),
                        o.stress + 6 * static_cast<size_t>(c), n, pp, area, am1, alpha);
    } else {
      const double dcca = __ldcs(g + fs);
      const double tmp = xmul(presC, area);
      for (int j = 0; j < 3; ++j) pf[j] = xadd(pf[j], xmul(tmp, n[j]));
      if (kExt && o.fstruc)
        struct_integral(o.stress + 6 * static_cast<size_t>(cell), nullptr, n, pp, area, 0.0,
                        0.0);
      if (nb <= -2) {
        const DevLoad &L = loads[-nb - 2];
        if (L.type == 8 || L.type == 14) {  // MOVEWALL, STATICWALL
          const double vB[3] = {L.type == 8 ? L.par[0] : 0.0, L.type == 8 ? L.par[1] : 0.0,
                                L.type == 8 ? L.par[2] : 0.0};
          double visc = effC;
          if (kExt && o.fwall) {  // the wall model's viscosity (Loads.c:300-313)
            const double yp = o.wall[4 * static_cast<size_t>(cell)];
            const double up = o.wall[4 * static_cast<size_t>(cell) + 1];
            visc = yp > 0.01e0 ? xdiv(xmul(muC, yp), up) : muC;
          }
          move_wall(velC, vB, n, sPc, pp, dcca, visc, area);
        } else if (L.type == 6) {  // INLET
          const double tA[3] = {L.par[0], L.par[1], L.par[2]};
          double wfn = xadd(xmul(tA[0], n[0]), xmul(tA[1], n[1]));
          wfn = xadd(wfn, xmul(tA[2], n[2]));
          const double mflux = xmul(xmul(L.par_last, wfn), area);
          // stress (CellLib.c:7013), lambda = 0
          const double tr = xadd(xadd(gvC[0], gvC[4]), gvC[8]);
          const double nu2 = xmul(2.0, muC), z = xmul(0.0, tr);
          const double ss[6] = {xadd(xmul(nu2, gvC[0]), z), xadd(xmul(nu2, gvC[4]), z),
                                xadd(xmul(nu2, gvC[8]), z), xmul(muC, xadd(gvC[3], gvC[1])),
                                xmul(muC, xadd(gvC[7], gvC[5])), xmul(muC, xadd(gvC[6], gvC[2]))};
          const double sa[3] = {xmul(area, n[0]), xmul(area, n[1]), xmul(area, n[2])};
          const double r0[3] = {ss[0], ss[3], ss[5]}, r1[3] = {ss[3], ss[1], ss[4]},
                       r2[3] = {ss[5], ss[4], ss[2]};
          pp[0] = xadd(pp[0], dot3(r0, sa));
          pp[1] = xadd(pp[1], dot3(r1, sa));
          pp[2] = xadd(pp[2], dot3(r2, sa));
          for (int k = 0; k < 3; ++k) pp[k] = xsub(pp[k], xmul(mflux, tA[k]));
        } else if (L.type == 7 || L.type == 10) {  // OUTLET, OPEN
          const double wfn = dot3(velC, n);
          if (L.type == 10 && wfn < 0.0) {
            // OPEN inflow (Loads.c:604-627): along the cell's own velocity
            const double mflux = xmul(xmul(L.density, wfn), area);
            const double aP = xmul(xmul(mflux, wfn), xdiv(1.0, xsqrt(dot3(velC, velC))));
            for (int k = 0; k < 3; ++k) pp[k] = xsub(pp[k], xmul(aP, velC[k]));
          } else {
            // OUTLET (Loads.c:436-518), OPEN outflow (Loads.c:531-600)
            const double mflux = xmul(xmul(rhoC, wfn), area);
            if (L.type == 7) {  // stress (CellLib.c:7013), lambda = 0
              const double tr = xadd(xadd(gvC[0], gvC[4]), gvC[8]);
              const double nu2 = xmul(2.0, muC), z = xmul(0.0, tr);
              const double ss[6] = {xadd(xmul(nu2, gvC[0]), z), xadd(xmul(nu2, gvC[4]), z),
                                    xadd(xmul(nu2, gvC[8]), z), xmul(muC, xadd(gvC[3], gvC[1])),
                                    xmul(muC, xadd(gvC[7], gvC[5])),
                                    xmul(muC, xadd(gvC[6], gvC[2]))};
              const double sa[3] = {xmul(area, n[0]), xmul(area, n[1]), xmul(area, n[2])};
              const double r0[3] = {ss[0], ss[3], ss[5]}, r1[3] = {ss[3], ss[1], ss[4]},
                           r2[3] = {ss[5], ss[4], ss[2]};
              pp[0] = xadd(pp[0], dot3(r0, sa));
              pp[1] = xadd(pp[1], dot3(r1, sa));
              pp[2] = xadd(pp[2], dot3(r2, sa));
            }
            // gradFaceNull (CellLib.c:5477-5600): the cell gradient less its
            // part along the centroid-to-face direction, applied to xmcc
            const double xc[3] = {__ldcs(g + 13 * fs), __ldcs(g + 14 * fs), __ldcs(g + 15 * fs)};
            const double mod = xsqrt(dot3(xc, xc));
            const double ef[3] = {xdiv(xc[0], mod), xdiv(xc[1], mod), xdiv(xc[2], mod)};
            for (int i = 0; i < 3; ++i) {
              const double prod = dot3(gvC + 3 * i, ef);
              double gf[3];
              for (int j = 0; j < 3; ++j) gf[j] = xsub(gvC[3 * i + j], xmul(prod, ef[j]));
              pp[i] = xsub(pp[i], xmul(mflux, dot3(gf, xc)));
              sPc[i] = xadd(sPc[i], mflux);
            }
          }
        } else if (L.type == 9) {
          // INLETSTAICTPRES (Loads.c:364-392), the load's par[0..2] as the
          // inflow direction (the reference's getLoads copies none for it)
          const double wfn = dot3(velC, n);
          const double dir[3] = {L.par[0], L.par[1], L.par[2]};
          const double t3 = xdiv(wfn, dot3(dir, n));
          const double mflux = xmul(xmul(rhoC, wfn), area);
          for (int k = 0; k < 3; ++k) pp[k] = xsub(pp[k], xmul(xmul(mflux, dir[k]), t3));
        } else if (L.type == 13) {
          // INLETTOTALPRES (Loads.c:634-672): density par[0], direction par[2..4]
          const double ev[3] = {L.par[2], L.par[3], L.par[4]};
          const double t1 = xmul(dot3(ev, n), area);
          const double mflux = xmul(xmul(L.par[0], dot3(velC, n)), area);
          const double tm = xmul(mflux, xdiv(mflux, xmul(L.par[0], t1)));
          for (int k = 0; k < 3; ++k) pp[k] = xsub(pp[k], xmul(tm, ev[k]));
        }
      }
    }
  }
  // implicit time term, CellSimple.c:606-617
  if (o.time_flag) {
    const double vol = p.vol[r];
    if (o.time_type == 0) {
      sP = xadd(sP, xdiv(xmul(rhoC, vol), o.dt));
    } else if (o.time_type == 1) {
      const double tmp = xadd(xdiv(1.0, o.dt), xdiv(1.0, xadd(o.dt, o.dt0)));
      sP = xadd(sP, xmul(xmul(tmp, rhoC), vol));
    }
  }
  double lAn = 0.0;
#pragma unroll
  for (int f = 0; f < kMV; ++f)
    if (f < nf) lAn = xadd(lAn, la[f]);
  double dk[3], rc[3];
  const double relax = xsub(1.0, o.under);
  for (int k = 0; k < 3; ++k) {
    dk[k] = xdiv(xadd(xadd(sP, sPc[k]), lAn), o.under);
    pp[k] = xadd(pp[k], xmul(xmul(relax, dk[k]), velC[k]));
    pp[k] = xsub(pp[k], pf[k]);
    rc[k] = 0.0;
  }
#pragma unroll
  for (int f = 0; f < kMV; ++f) {
    if (f >= nf) continue;
    const int32_t nb = __ldcs(p.nb + static_cast<size_t>(f) * p.n + r);
    if (nb < 0) continue;
    const size_t v3 = 3 * static_cast<size_t>(nb & (kFlagP - 1));
    for (int k = 0; k < 3; ++k) {
      const double t = xmul(la[f], vel[v3 + k]);
      if (nb & kFlagP)
        pp[k] = xadd(pp[k], t);
      else
        rc[k] = xadd(rc[k], t);
    }
  }
  const double vol = p.vol[r];
  for (int k = 0; k < 3; ++k) {
    rc[k] = xadd(rc[k], xsub(pp[k], xmul(dk[k], velC[k])));
    dfield[c3 + k] = o.simplec ? xdiv(vol, xsub(dk[k], lAn)) : xdiv(vol, dk[k]);
    if (o.forces) b3[static_cast<size_t>(k) * p.n + r] = o.fres ? rc[k] : pp[k];
    if (o.calrcell) rcell3[static_cast<size_t>(k) * numel + cell] = rc[k];
  }
  if (!o.matrix) return;
  diag[r] = dk[0];
  if (ad3)
    for (int k = 0; k < 3; ++k) ad3[static_cast<size_t>(k) * p.n + r] = dk[k];
#pragma unroll
  for (int f = 0; f < kMV; ++f)
    if (f < nf) {
      const int32_t t = __ldcs(p.dst + static_cast<size_t>(f) * p.n + r);
      if (t >= 0) stage[t] = xmul(la[f], -1.0);
    }
}

__global__ void update_cells_kernel(const int32_t *id, int numel, int n, const double *x,
                                    double *u, int add) {
  const int nel = blockIdx.x * blockDim.x + threadIdx.x;
  if (nel >= numel) return;
  const int row = id[nel] - 1;
  if (row > -1 && row < n) u[nel] = add ? xadd(u[nel], x[row]) : x[row];
}

template <typename T>
cudaError_t upload(T **dst, const T *src, size_t count) {
  *dst = nullptr;
  if (count == 0) return cudaSuccess;
  cudaError_t e = cudaMalloc(dst, sizeof(T) * count);
  if (e != cudaSuccess) return e;
  return cudaMemcpy(*dst, src, sizeof(T) * count, cudaMemcpyHostToDevice);
}

}  // namespace
}  // namespace sfr

struct sfr_dif_plan {
  sfr_system *s = nullptr;       // the system written; must outlive the plan's calls
  int32_t device = 0;            // destroy needs no live system
  int32_t kind = 0;              // 0 diffusion (systFormDif), 1 pressure (systFormSimplePres),
                                 // 2 momentum (systFormSimpleVel)
  int32_t numel = 0, maxviz = 0, icod = 0, nmat = 0;
  int free_cells = 0;            // cells without an equation (their rcell is zeroed)
  unsigned used_loads = 0;       // bit l: some boundary face names load l (pressure loads)
  unsigned used_vel_loads = 0;   // the same for the velocity loads (pressure plans)
  sfr::PlanDev d{};
  bool fused = false;            // the assembly also refreshes the SELL copy
  int32_t *d_id = nullptr;       // per cell: equation + 1 (updateCellValue)
  int16_t *d_mat = nullptr;      // per cell: material + 1 (pressure plans)
  // the load tables ([0, 32) loads, [32, 64) velocity loads) then the density
  // of each material (pressure plans)
  unsigned char *d_table = nullptr;
  std::vector<unsigned char> table_host;  // what d_table holds
  // host-array calls: device copies of the fields and results
  double *h_fields = nullptr;    // diffusion: density | cdiff | u0 | gradu0; pressure:
                                 // pres | gradpres | vel | dfield
  double *h_b0 = nullptr, *h_b = nullptr, *h_rcell = nullptr;
  // momentum plans: the turbulence fields (bound device arrays, or the plan's
  // own copies of host arrays)
  const double *t_eddy = nullptr, *t_stress = nullptr;
  double *own_eddy = nullptr, *own_stress = nullptr;
  const double *t_wall = nullptr;  // the wall model's per-cell parameters
  double *own_wall = nullptr;
  double *dsnap = nullptr;         // Rhie-Chow: the D field at a call's start
};

namespace {

#define SFR_CUA(expr)                                     \
  do {                                                    \
    cudaError_t e_ = (expr);                              \
    if (e_ != cudaSuccess) {                              \
      sfr::set_last_error(cudaGetErrorString(e_));        \
      return SFR_CUDA_ERROR;                              \
    }                                                     \
  } while (0)

int bad(const char *why) {
  sfr::set_last_error(why);
  return SFR_BAD_INPUT;
}

int unsupported(const char *why) {
  sfr::set_last_error(why);
  return SFR_UNSUPPORTED;
}

constexpr size_t kTableLoads = 2 * sfr::kMaxLoads;

// the load tables, then density and viscosity of each material
size_t table_bytes(const sfr_dif_plan *p) {
  return sizeof(sfr::DevLoad) * kTableLoads + 2 * sizeof(double) * std::max(p->nmat, 1);
}

void free_plan_buffers(sfr_dif_plan *p) {
  cudaFree(p->d.cell);
  cudaFree(p->d.nface);
  cudaFree(p->d.nb);
  cudaFree(p->d.dst);
  cudaFree(p->d.sslot);
  cudaFree(p->d.geo);
  cudaFree(p->d.vol);
  cudaFree(p->d_id);
  cudaFree(p->d_mat);
  cudaFree(p->d_table);
  cudaFree(p->h_fields);
  cudaFree(p->h_b0);
  cudaFree(p->h_b);
  cudaFree(p->h_rcell);
  cudaFree(p->own_eddy);
  cudaFree(p->own_stress);
  cudaFree(p->own_wall);
  cudaFree(p->dsnap);
}

void fill_load(sfr::DevLoad *d, const sfr_load &L) {
  d->type = L.type;
  for (int j = 0; j < 5; ++j) d->par[j] = L.par[j];
  d->par_last = L.np >= 1 && L.np <= 20 ? L.par[L.np - 1] : 0.0;
  d->density = L.density;
}

// Copy the host table to the device when it changed since the last call.
int stage_table(sfr_dif_plan *p, const std::vector<unsigned char> &h, cudaStream_t st) {
  if (h != p->table_host) {
    SFR_CUA(cudaMemcpyAsync(p->d_table, h.data(), h.size(), cudaMemcpyHostToDevice, st));
    SFR_CUA(cudaStreamSynchronize(st));  // h is the caller's local
    p->table_host = h;
  }
  return SFR_OK;
}

// Diffusion: the loads the mesh uses against what pLoad accepts
// (Loads.c:881-990, getLoads Loads.c:122-169).
int stage_dif_loads(sfr_dif_plan *p, const sfr_load *loads, int32_t nloads, cudaStream_t st) {
  if (nloads < 0 || nloads > sfr::kMaxLoads || (nloads > 0 && !loads))
    return bad("nloads must be 0..32");
  for (int l = 0; l < sfr::kMaxLoads; ++l) {
    if (!(p->used_loads & (1u << l))) continue;
    if (l >= nloads) return bad("a boundary face names a load beyond nloads");
    const sfr_load &L = loads[l];
    const bool needs_value = L.type == 1 || L.type == 2 || L.type == 6;
    if ((L.type == 1 || L.type == 6) && L.var != 0)
      return unsupported("loads given as functions (nTypeVar 1) are not assembled on the device");
    if (L.type == 4) return unsupported("SINBC loads are not assembled on the device");
    if (L.type == 7) return bad("an OUTLET load reads a cell velocity the diffusion cell has not");
    if (needs_value && L.np < 1) return bad("a load has no parameters");
    if (L.type == 6 && L.np < 5) return bad("an INLET load needs 5 parameters");
  }
  std::vector<unsigned char> h(table_bytes(p), 0);
  auto *t = reinterpret_cast<sfr::DevLoad *>(h.data());
  for (int l = 0; l < nloads; ++l) fill_load(t + l, loads[l]);
  return stage_table(p, h, st);
}

// Pressure correction: pLoadSimplePres (Loads.c:728-845) reads pressure
// loads' parameters directly; of the velocity loads (pLoadSimple,
// Loads.c:265-720) only INLET reads a parameter list (getLoads copies np of
// them, then par[0..2] and par[np - 1] are read).  prop: nmat x MAXPROP.
int stage_pres_tables(sfr_dif_plan *p, const sfr_load *lvel, int32_t nlvel,
                      const sfr_load *lpres, int32_t nlpres, const double *prop,
                      cudaStream_t st) {
  if (nlvel < 0 || nlvel > sfr::kMaxLoads || (nlvel > 0 && !lvel) || nlpres < 0 ||
      nlpres > sfr::kMaxLoads || (nlpres > 0 && !lpres))
    return bad("nlvel and nlpres must be 0..32");
  if (!prop) return bad("prop is NULL");
  for (int l = 0; l < sfr::kMaxLoads; ++l) {
    if ((p->used_loads & (1u << l)) && l >= nlpres)
      return bad("a boundary face names a pressure load beyond nlpres");
    if (!(p->used_vel_loads & (1u << l))) continue;
    if (l >= nlvel) return bad("a boundary face names a velocity load beyond nlvel");
    const sfr_load &L = lvel[l];
    if (L.type == 6 && L.var != 0)
      return unsupported("loads given as functions (nTypeVar 1) are not assembled on the device");
    if (L.type == 6 && (L.np < 3 || L.np > 20)) return bad("an INLET load needs 3..20 parameters");
  }
  std::vector<unsigned char> h(table_bytes(p), 0);
  auto *t = reinterpret_cast<sfr::DevLoad *>(h.data());
  for (int l = 0; l < nlpres; ++l) fill_load(t + l, lpres[l]);
  for (int l = 0; l < nlvel; ++l) fill_load(t + sfr::kMaxLoads + l, lvel[l]);
  auto *dens = reinterpret_cast<double *>(h.data() + sizeof(sfr::DevLoad) * kTableLoads);
  for (int k = 0; k < p->nmat; ++k) dens[k] = prop[k * 10 + 1];  // MAXPROP 10, DENSITY 1
  return stage_table(p, h, st);
}

// Momentum: pLoadSimple with fCalVel (Loads.c:265-720): MOVEWALL,
// STATICWALL, constant INLET, OUTLET, OPEN, INLETSTAICTPRES and
// INLETTOTALPRES (getLoads copies par[0..4] of the last two, Loads.c:148-155,
// and OPEN reads Loads.density); prop: nmat x MAXPROP (DYNAMICVISCOSITY 0,
// DENSITY 1).
int stage_vel_tables(sfr_dif_plan *p, const sfr_load *lvel, int32_t nlvel, const double *prop,
                     cudaStream_t st) {
  if (nlvel < 0 || nlvel > sfr::kMaxLoads || (nlvel > 0 && !lvel))
    return bad("nlvel must be 0..32");
  if (!prop) return bad("prop is NULL");
  for (int l = 0; l < sfr::kMaxLoads; ++l) {
    if (!(p->used_loads & (1u << l))) continue;
    if (l >= nlvel) return bad("a boundary face names a velocity load beyond nlvel");
    const sfr_load &L = lvel[l];
    if (L.type == 6 && L.var != 0)
      return unsupported("loads given as functions (nTypeVar 1) are not assembled on the device");
    if (L.type == 6 && (L.np < 3 || L.np > 20)) return bad("an INLET load needs 3..20 parameters");
  }
  std::vector<unsigned char> h(table_bytes(p), 0);
  auto *t = reinterpret_cast<sfr::DevLoad *>(h.data());
  for (int l = 0; l < nlvel; ++l) fill_load(t + l, lvel[l]);
  auto *mt = reinterpret_cast<double *>(h.data() + sizeof(sfr::DevLoad) * kTableLoads);
  for (int k = 0; k < p->nmat; ++k) {
    mt[k] = prop[k * 10 + 1];            // DENSITY
    mt[p->nmat + k] = prop[k * 10 + 0];  // DYNAMICVISCOSITY
  }
  return stage_table(p, h, st);
}

int create_plan(sfr_system *s, const sfr_dif_mesh *mesh, const int16_t *facevelr, int32_t icod,
                int32_t kind, sfr_dif_plan **out) {
  if (!s || !mesh || !out) return bad("NULL argument");
  *out = nullptr;
  const sfr_dif_mesh &m = *mesh;
  if (kind == 0 && (icod < 1 || icod > 4)) return bad("icod must be 1..4 (Define.h:304-307)");
  if (kind == 2 && (icod < 1 || icod > 4)) return bad("icod must be 1..4 (Define.h:304-307)");
  if (kind == 2 && (!m.cc || !m.xm)) return bad("the momentum plan needs cc and xm");
  if (kind == 2 && s->storage == SFR_ELLPACK)
    return bad("csrSimple refuses ELLPACK for ndf > 1 (EllPack.c:143-147)");
  if (kind == 1 && icod != 1 && icod != 4)
    return bad("the pressure split (difusionSchemeAnisotropic) sets e and t only for "
               "ORTHOGONAL (1) and OVERRELAXED (4)");
  if (kind == 1 && !facevelr) return bad("facevelr is NULL");
  if (m.numel < 1 || m.maxviz < 1 || m.maxviz > sfr::kMaxViz || m.nfaces < 1 || m.nmat < 1)
    return bad("mesh sizes out of range (maxviz 1..8)");
  const void *need[] = {m.nelcon, m.nviz, m.cellface, m.owner, m.volume, m.dcca, m.xmcc,
                        m.mksi, m.ksi, m.area, m.normal, m.vskew, m.caltype, m.mat,
                        m.id, m.facer};
  for (const void *q : need)
    if (!q) return bad("a mesh array is NULL");
  if (static_cast<int64_t>(s->n) * m.maxviz > INT32_MAX) return bad("system too large");
  for (int64_t f = 0; f < m.nfaces; ++f)
    if (m.owner[2 * f] < 1 || m.owner[2 * f] > m.numel) return bad("a face owner is out of range");
  if (kind != 0)
    for (int32_t c = 0; c < m.numel; ++c)  // the density lookup of every cell
      if (m.mat[c] < 1 || m.mat[c] > m.nmat) return bad("a cell's material is out of range");
  SFR_CUA(cudaSetDevice(s->device));
  auto *p = new sfr_dif_plan;
  p->s = s;
  p->device = s->device;
  p->kind = kind;
  p->numel = m.numel;
  p->maxviz = m.maxviz;
  p->icod = icod;
  p->nmat = m.nmat;
  p->table_host.assign(table_bytes(p), 0);
  const int n = s->n;
  const int mvpad = m.maxviz <= 6 ? 6 : sfr::kMaxViz;  // slots the assembly kernels read
  const size_t slots = static_cast<size_t>(mvpad) * n;
  sfr::MeshDev md{};
  md.numel = m.numel;
  md.maxviz = m.maxviz;
  md.nmat = m.nmat;
  md.nfaces = m.nfaces;
  const size_t ne = m.numel, nv = ne * m.maxviz, nf = m.nfaces;
  int rc = SFR_OK;
  int *d_err = nullptr;
  auto release_mesh = [&]() {
    cudaFree(const_cast<int32_t *>(md.nelcon));
    cudaFree(const_cast<int32_t *>(md.cellface));
    cudaFree(const_cast<int32_t *>(md.owner));
    cudaFree(const_cast<int16_t *>(md.nviz));
    cudaFree(const_cast<int16_t *>(md.caltype));
    cudaFree(const_cast<int16_t *>(md.facer));
    cudaFree(const_cast<int16_t *>(md.facevelr));
    cudaFree(const_cast<double *>(md.volume));
    cudaFree(const_cast<double *>(md.dcca));
    cudaFree(const_cast<double *>(md.xmcc));
    cudaFree(const_cast<double *>(md.mksi));
    cudaFree(const_cast<double *>(md.ksi));
    cudaFree(const_cast<double *>(md.area));
    cudaFree(const_cast<double *>(md.normal));
    cudaFree(const_cast<double *>(md.vskew));
    cudaFree(const_cast<double *>(md.cc));
    cudaFree(const_cast<double *>(md.xm));
    cudaFree(d_err);
  };
  auto up = [&](cudaError_t e) {
    if (e != cudaSuccess && rc == SFR_OK) {
      sfr::set_last_error(cudaGetErrorString(e));
      rc = SFR_CUDA_ERROR;
    }
  };
  {
    int32_t *t32;
    int16_t *t16;
    double *t64;
    up(sfr::upload(&t32, m.nelcon, nv)); md.nelcon = t32;
    up(sfr::upload(&t32, m.cellface, nv)); md.cellface = t32;
    up(sfr::upload(&t32, m.owner, 2 * nf)); md.owner = t32;
    up(sfr::upload(&t32, m.id, ne)); md.id = t32;
    p->d_id = t32;  // kept by the plan for updateCellValue
    up(sfr::upload(&t16, m.nviz, ne)); md.nviz = t16;
    up(sfr::upload(&t16, m.caltype, static_cast<size_t>(m.nmat))); md.caltype = t16;
    up(sfr::upload(&t16, m.mat, ne)); md.mat = t16;
    p->d_mat = t16;  // kept by the plan for the density lookup
    up(sfr::upload(&t16, m.facer, ne * (m.maxviz + 1))); md.facer = t16;
    if (kind == 1) {
      up(sfr::upload(&t16, facevelr, ne * (m.maxviz + 1)));
      md.facevelr = t16;
    }
    up(sfr::upload(&t64, m.volume, ne)); md.volume = t64;
    up(sfr::upload(&t64, m.dcca, nv)); md.dcca = t64;
    up(sfr::upload(&t64, m.xmcc, 3 * nv)); md.xmcc = t64;
    up(sfr::upload(&t64, m.mksi, nf)); md.mksi = t64;
    up(sfr::upload(&t64, m.ksi, 3 * nf)); md.ksi = t64;
    up(sfr::upload(&t64, m.area, nf)); md.area = t64;
    up(sfr::upload(&t64, m.normal, 3 * nf)); md.normal = t64;
    up(sfr::upload(&t64, m.vskew, 3 * nf)); md.vskew = t64;
    if (kind == 2) {
      up(sfr::upload(&t64, m.cc, 3 * ne)); md.cc = t64;
      up(sfr::upload(&t64, m.xm, 3 * nf)); md.xm = t64;
    }
  }
  sfr::PlanDev &d = p->d;
  d.n = n;
  d.maxviz = mvpad;
  d.fstride = slots;
  up(cudaMalloc(&d.cell, sizeof(int32_t) * n));
  up(cudaMalloc(&d.nface, sizeof(int16_t) * n));
  up(cudaMalloc(&d.nb, sizeof(int32_t) * slots));
  up(cudaMalloc(&d.dst, sizeof(int32_t) * slots));
  up(cudaMalloc(&d.sslot, sizeof(int32_t) * slots));
  const int nfield = kind == 2 ? sfr::kGeoVel : sfr::kGeo;
  up(cudaMalloc(&d.geo, sizeof(double) * slots * nfield));
  up(cudaMalloc(&d.vol, sizeof(double) * n));
  up(cudaMalloc(&p->d_table, table_bytes(p)));
  up(cudaMalloc(&d_err, sizeof(int) * 5));
  if (rc == SFR_OK) {
    up(cudaMemset(d.cell, 0xFF, sizeof(int32_t) * n));
    up(cudaMemset(d.nface, 0, sizeof(int16_t) * n));
    up(cudaMemset(d.nb, 0xFF, sizeof(int32_t) * slots));
    up(cudaMemset(d.dst, 0xFF, sizeof(int32_t) * slots));
    up(cudaMemset(d.sslot, 0xFF, sizeof(int32_t) * slots));
    up(cudaMemset(d.geo, 0, sizeof(double) * slots * nfield));
    up(cudaMemset(p->d_table, 0, table_bytes(p)));
    up(cudaMemset(d_err, 0, sizeof(int) * 5));
  }
  if (rc == SFR_OK) {
    sfr::PatternDev P{s->A.sptr, s->A.col, s->A.src, n, s->storage, s->unsym,
                      s->storage == SFR_ELLPACK ? s->nsrc / std::max(n, 1) : 0};
    const int blocks = (m.numel + 255) / 256;
    sfr::plan_kernel<<<blocks, 256>>>(md, P, d, icod, kind, d_err,
                                      reinterpret_cast<unsigned *>(d_err + 1), d_err + 2,
                                      d_err + 3, reinterpret_cast<unsigned *>(d_err + 4));
    up(cudaGetLastError());
    int h[5] = {0, 0, 0, 0, 0};
    up(cudaMemcpy(h, d_err, sizeof(h), cudaMemcpyDeviceToHost));
    if (rc == SFR_OK && h[0] != sfr::kErrNone) rc = bad(sfr::plan_error_text(h[0]));
    p->used_loads = static_cast<unsigned>(h[1]);
    p->free_cells = h[2];
    p->used_vel_loads = static_cast<unsigned>(h[4]);
    // every stored value of every row written by the row's own cell (the
    // momentum kernel leaves the refresh to the usual gather)
    p->fused = kind != 2 && h[3] == 0 && s->A.val32 != nullptr;
  }
  if (rc == SFR_OK && p->fused) {
    if (!s->d_comp) {
      up(cudaMalloc(&s->d_comp, sizeof(double) * std::max(n, 1)));
      if (rc == SFR_OK) s->bytes += static_cast<int64_t>(sizeof(double)) * n;
    }
    if (!s->values_set) {  // padding slots hold zeros, as the refresh leaves them
      up(cudaMemset(s->A.val, 0, sizeof(double) * std::max<int64_t>(s->A.nslots, 1)));
      up(cudaMemset(s->A.val32, 0, sizeof(float) * std::max<int64_t>(s->A.nslots, 1)));
    }
  }
  md.id = nullptr;   // the plan's (freed with it)
  md.mat = nullptr;  // likewise
  release_mesh();
  if (rc != SFR_OK) {
    free_plan_buffers(p);
    delete p;
    return rc;
  }
  *out = p;
  return SFR_OK;
}

// device copies for the host-array calls, allocated together on first use
// (all or none, so that a failed allocation leaves the plan as it was)
// fields a cell: diffusion density, cdiff, u0, gradu0 (6); pressure pres,
// gradpres, vel, dfield (10); momentum pres, gradpres, vel, gradvel, dfield
// (19).  Momentum calls keep their three-block ad and b in h_b0 and h_b.
int ensure_host_buffers(sfr_dif_plan *p) {
  if (p->h_fields) return SFR_OK;
  const size_t ne = p->numel, n = p->s->n, k = p->kind == 2 ? 3 : 1;
  const size_t per_cell = p->kind == 2 ? 19 : 10;
  double *f = nullptr, *b0 = nullptr, *b = nullptr, *rc = nullptr;
  cudaError_t e = cudaMalloc(&f, sizeof(double) * ne * per_cell);
  if (e == cudaSuccess) e = cudaMalloc(&b0, sizeof(double) * n * k);
  if (e == cudaSuccess) e = cudaMalloc(&b, sizeof(double) * n * k);
  if (e == cudaSuccess) e = cudaMalloc(&rc, sizeof(double) * ne * k);
  if (e != cudaSuccess) {
    cudaFree(f);
    cudaFree(b0);
    cudaFree(b);
    cudaFree(rc);
    sfr::set_last_error(cudaGetErrorString(e));
    return SFR_CUDA_ERROR;
  }
  p->h_fields = f;
  p->h_b0 = b0;
  p->h_b = b;
  p->h_rcell = rc;
  return SFR_OK;
}

int copy_back(sfr_dif_plan *p, double *b, double *rcell, int32_t forces, int32_t calrcell,
              cudaStream_t st) {
  if (forces && b)
    SFR_CUA(cudaMemcpyAsync(b, p->h_b, sizeof(double) * p->s->n, cudaMemcpyDeviceToHost, st));
  if (calrcell && rcell)
    SFR_CUA(cudaMemcpyAsync(rcell, p->h_rcell, sizeof(double) * p->numel, cudaMemcpyDeviceToHost,
                            st));
  SFR_CUA(cudaStreamSynchronize(st));
  return SFR_OK;
}

}  // namespace

extern "C" {

int sfr_gpu_dif_plan_create(sfr_system *s, const sfr_dif_mesh *mesh, int32_t icod,
                            sfr_dif_plan **out) {
  return create_plan(s, mesh, nullptr, icod, 0, out);
}

int sfr_gpu_pres_plan_create(sfr_system *s, const sfr_dif_mesh *mesh, const int16_t *facevelr,
                             int32_t icod, sfr_dif_plan **out) {
  return create_plan(s, mesh, facevelr, icod, 1, out);
}

int sfr_gpu_dif_assemble_device(sfr_dif_plan *p, const sfr_load *loads, int32_t nloads,
                                const sfr_dif_opts *o, const double *d_density,
                                const double *d_cdiff, const double *d_u0,
                                const double *d_gradu0, const double *d_b0, double *d_b,
                                double *d_rcell, int32_t forces, int32_t matrix,
                                int32_t calrcell, void *stream) {
  if (!p || !o) return bad("NULL argument");
  if (p->kind != 0) return bad("not a diffusion plan");
  if (o->icod != p->icod) return bad("opts.icod differs from the scheme the plan was built for");
  if (!d_cdiff || !d_u0) return bad("cdiff and u0 are required");
  if (o->icod != 1 && !d_gradu0) return bad("gradu0 is required by non-orthogonal schemes");
  if (o->time_flag && !d_density) return bad("density is required by the time term");
  if (forces && !d_b) return bad("forces set without b");
  if (calrcell && !d_rcell) return bad("calrcell set without rcell");
  sfr_system *s = p->s;
  SFR_CUA(cudaSetDevice(s->device));
  cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : s->stream;
  int rc = stage_dif_loads(p, loads, nloads, st);
  if (rc != SFR_OK) return rc;
  if (calrcell && p->free_cells > 0)
    SFR_CUA(cudaMemsetAsync(d_rcell, 0, sizeof(double) * p->numel, st));
  sfr::CallOpts co{o->fres != 0, o->time_flag != 0, o->time_type, forces != 0, matrix != 0,
                   calrcell != 0, o->dt, o->dt0};
  const int blocks = (s->n + 255) / 256;
  const bool fuse = p->fused && matrix;
  sfr::FuseDev fu{s->A.val, s->A.val32, s->A.sptr, s->d_comp, s->d_diag32};
  const auto *loads_d = reinterpret_cast<const sfr::DevLoad *>(p->d_table);
  auto launch = [&](auto kernel) {
    kernel<<<blocks, 256, 0, st>>>(p->d, fu, loads_d, co, d_density, d_cdiff, d_u0, d_gradu0,
                                   d_b0, s->d_stage, s->d_diag, d_b, d_rcell);
  };
  const bool orth = p->icod == 1, six = p->d.maxviz == 6;
  constexpr int k8 = sfr::kMaxViz;
  if (fuse) {
    if (six)
      orth ? launch(sfr::dif_assemble_kernel<true, 6, true>)
           : launch(sfr::dif_assemble_kernel<false, 6, true>);
    else
      orth ? launch(sfr::dif_assemble_kernel<true, k8, true>)
           : launch(sfr::dif_assemble_kernel<false, k8, true>);
  } else {
    if (six)
      orth ? launch(sfr::dif_assemble_kernel<true, 6, false>)
           : launch(sfr::dif_assemble_kernel<false, 6, false>);
    else
      orth ? launch(sfr::dif_assemble_kernel<true, k8, false>)
           : launch(sfr::dif_assemble_kernel<false, k8, false>);
  }
  SFR_CUA(cudaGetLastError());
  if (matrix) return sfr::values_refreshed(s, st, fuse);
  return SFR_OK;
}

int sfr_gpu_dif_assemble(sfr_dif_plan *p, const sfr_load *loads, int32_t nloads,
                         const sfr_dif_opts *o, const double *density, const double *cdiff,
                         const double *u0, const double *gradu0, const double *b0, double *b,
                         double *rcell, int32_t forces, int32_t matrix, int32_t calrcell) {
  if (!p || !o) return bad("NULL argument");
  if (!cdiff || !u0) return bad("cdiff and u0 are required");
  sfr_system *s = p->s;
  SFR_CUA(cudaSetDevice(s->device));
  int rc = ensure_host_buffers(p);
  if (rc != SFR_OK) return rc;
  const size_t ne = p->numel;
  cudaStream_t st = s->stream;
  double *fd = p->h_fields;
  double *d_density = fd, *d_cdiff = fd + ne, *d_u0 = fd + 2 * ne, *d_grad = fd + 3 * ne;
  if (density)
    SFR_CUA(cudaMemcpyAsync(d_density, density, sizeof(double) * ne, cudaMemcpyHostToDevice, st));
  SFR_CUA(cudaMemcpyAsync(d_cdiff, cdiff, sizeof(double) * ne, cudaMemcpyHostToDevice, st));
  SFR_CUA(cudaMemcpyAsync(d_u0, u0, sizeof(double) * ne, cudaMemcpyHostToDevice, st));
  if (gradu0)
    SFR_CUA(cudaMemcpyAsync(d_grad, gradu0, sizeof(double) * ne * 3, cudaMemcpyHostToDevice, st));
  if (b0)
    SFR_CUA(cudaMemcpyAsync(p->h_b0, b0, sizeof(double) * s->n, cudaMemcpyHostToDevice, st));
  rc = sfr_gpu_dif_assemble_device(p, loads, nloads, o, density ? d_density : nullptr, d_cdiff,
                                   d_u0, gradu0 ? d_grad : nullptr, b0 ? p->h_b0 : nullptr,
                                   p->h_b, p->h_rcell, forces, matrix, calrcell, st);
  if (rc != SFR_OK) return rc;
  return copy_back(p, b, rcell, forces, calrcell, st);
}

int sfr_gpu_pres_assemble_device(sfr_dif_plan *p, const sfr_load *lvel, int32_t nlvel,
                                 const sfr_load *lpres, int32_t nlpres, const double *prop,
                                 const double *d_pres, const double *d_gradpres,
                                 const double *d_vel, const double *d_dfield, double *d_b,
                                 double *d_rcell, int32_t forces, int32_t matrix,
                                 int32_t calrcell, void *stream) {
  if (!p) return bad("NULL argument");
  if (p->kind != 1) return bad("not a pressure-correction plan");
  if (!d_pres || !d_gradpres || !d_vel || !d_dfield)
    return bad("pres, gradpres, vel and dfield are required");
  if (forces && !d_b) return bad("forces set without b");
  if (calrcell && !d_rcell) return bad("calrcell set without rcell");
  sfr_system *s = p->s;
  SFR_CUA(cudaSetDevice(s->device));
  cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : s->stream;
  int rc = stage_pres_tables(p, lvel, nlvel, lpres, nlpres, prop, st);
  if (rc != SFR_OK) return rc;
  if (calrcell && p->free_cells > 0)
    SFR_CUA(cudaMemsetAsync(d_rcell, 0, sizeof(double) * p->numel, st));
  sfr::PresOpts po{forces != 0, matrix != 0, calrcell != 0};
  const int blocks = (s->n + 255) / 256;
  const bool fuse = p->fused && matrix;
  sfr::FuseDev fu{s->A.val, s->A.val32, s->A.sptr, s->d_comp, s->d_diag32};
  const auto *loads_d = reinterpret_cast<const sfr::DevLoad *>(p->d_table);
  const auto *dens =
      reinterpret_cast<const double *>(p->d_table + sizeof(sfr::DevLoad) * kTableLoads);
  auto launch = [&](auto kernel) {
    kernel<<<blocks, 256, 0, st>>>(p->d, fu, loads_d, po, p->d_mat, dens, d_pres, d_gradpres,
                                   d_vel, d_dfield, s->d_stage, s->d_diag, d_b, d_rcell);
  };
  const bool over = p->icod == 4, six = p->d.maxviz == 6;
  constexpr int k8 = sfr::kMaxViz;
  if (fuse) {
    if (six)
      over ? launch(sfr::pres_assemble_kernel<true, 6, true>)
           : launch(sfr::pres_assemble_kernel<false, 6, true>);
    else
      over ? launch(sfr::pres_assemble_kernel<true, k8, true>)
           : launch(sfr::pres_assemble_kernel<false, k8, true>);
  } else {
    if (six)
      over ? launch(sfr::pres_assemble_kernel<true, 6, false>)
           : launch(sfr::pres_assemble_kernel<false, 6, false>);
    else
      over ? launch(sfr::pres_assemble_kernel<true, k8, false>)
           : launch(sfr::pres_assemble_kernel<false, k8, false>);
  }
  SFR_CUA(cudaGetLastError());
  if (matrix) return sfr::values_refreshed(s, st, fuse);
  return SFR_OK;
}

int sfr_gpu_pres_assemble(sfr_dif_plan *p, const sfr_load *lvel, int32_t nlvel,
                          const sfr_load *lpres, int32_t nlpres, const double *prop,
                          const double *pres, const double *gradpres, const double *vel,
                          const double *dfield, double *b, double *rcell, int32_t forces,
                          int32_t matrix, int32_t calrcell) {
  if (!p) return bad("NULL argument");
  if (!pres || !gradpres || !vel || !dfield) return bad("pres, gradpres, vel and dfield are required");
  sfr_system *s = p->s;
  SFR_CUA(cudaSetDevice(s->device));
  int rc = ensure_host_buffers(p);
  if (rc != SFR_OK) return rc;
  const size_t ne = p->numel;
  cudaStream_t st = s->stream;
  double *fd = p->h_fields;
  double *d_pres = fd, *d_gp = fd + ne, *d_vel = fd + 4 * ne, *d_df = fd + 7 * ne;
  SFR_CUA(cudaMemcpyAsync(d_pres, pres, sizeof(double) * ne, cudaMemcpyHostToDevice, st));
  SFR_CUA(cudaMemcpyAsync(d_gp, gradpres, sizeof(double) * ne * 3, cudaMemcpyHostToDevice, st));
  SFR_CUA(cudaMemcpyAsync(d_vel, vel, sizeof(double) * ne * 3, cudaMemcpyHostToDevice, st));
  SFR_CUA(cudaMemcpyAsync(d_df, dfield, sizeof(double) * ne * 3, cudaMemcpyHostToDevice, st));
  rc = sfr_gpu_pres_assemble_device(p, lvel, nlvel, lpres, nlpres, prop, d_pres, d_gp, d_vel,
                                    d_df, p->h_b, p->h_rcell, forces, matrix, calrcell, st);
  if (rc != SFR_OK) return rc;
  return copy_back(p, b, rcell, forces, calrcell, st);
}

int sfr_gpu_vel_plan_create(sfr_system *s, const sfr_dif_mesh *mesh, int32_t icod,
                            sfr_dif_plan **out) {
  return create_plan(s, mesh, nullptr, icod, 2, out);
}

int sfr_gpu_vel_assemble_device(sfr_dif_plan *p, const sfr_load *lvel, int32_t nlvel,
                                const sfr_vel_opts *o, const double *prop, const double *d_pres,
                                const double *d_gradpres, const double *d_vel,
                                const double *d_gradvel, double *d_dfield, double *d_ad3,
                                double *d_b3, double *d_rcell3, int32_t forces, int32_t matrix,
                                int32_t calrcell, void *stream) {
  if (!p || !o) return bad("NULL argument");
  if (p->kind != 2) return bad("not a momentum plan");
  if (o->icod != p->icod) return bad("opts.icod differs from the scheme the plan was built for");
  if (o->type_simple != 1 && o->type_simple != 2)
    return bad("type_simple must be SIMPLE (1) or SIMPLEC (2)");
  if (!d_pres || !d_gradpres || !d_vel || !d_gradvel || !d_dfield)
    return bad("pres, gradpres, vel, gradvel and dfield are required");
  if (forces && !d_b3) return bad("forces set without b");
  if (calrcell && !d_rcell3) return bad("calrcell set without rcell");
  sfr_system *s = p->s;
  SFR_CUA(cudaSetDevice(s->device));
  cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : s->stream;
  int rc = stage_vel_tables(p, lvel, nlvel, prop, st);
  if (rc != SFR_OK) return rc;
  if (calrcell && p->free_cells > 0)
    SFR_CUA(cudaMemsetAsync(d_rcell3, 0, sizeof(double) * 3 * p->numel, st));
  if (o->adv < 0 || o->adv > 6)
    return bad("adv: FoUp (0 or 1), CD (2), SoUp (3), TVD (4), NVD (5) or LUST (6)");
  if (o->adv == 5 && (o->adv_fn < 1 || o->adv_fn > 9)) return bad("adv_fn: NVD function 1..9");
  if (o->adv == 4 && (o->adv_fn < 1 || o->adv_fn > 5)) return bad("adv_fn: TVD limiter 1..5");
  if ((o->fturb && !p->t_eddy) || (o->fstruc && !p->t_stress))
    return bad("fturb / fstruc set without the field bound by sfr_gpu_vel_turbulence");
  if (o->fwall && !p->t_wall) return bad("fwall set without the field bound by sfr_gpu_vel_wall");
  if (o->rhie < 0 || o->rhie > 1)
    return unsupported("rhie: 0 off, 1 D from the call's start (the reference's serial order, in "
                       "which a cell reads its lower-numbered neighbours' new D, is not restated "
                       "on the device)");
  if (o->rhie) {  // every face velocity reads D as it was before this call
    if (!p->dsnap) SFR_CUA(cudaMalloc(&p->dsnap, sizeof(double) * 3 * p->numel));
    SFR_CUA(cudaMemcpyAsync(p->dsnap, d_dfield, sizeof(double) * 3 * p->numel,
                            cudaMemcpyDeviceToDevice, st));
  }
  sfr::VelOpts vo{o->fso != 0, o->fvisc != 0, o->fres != 0, o->type_simple == 2,
                  o->time_flag != 0, o->time_type, forces != 0, matrix != 0, calrcell != 0,
                  o->dt, o->dt0, o->under, o->adv == 0 ? 1 : o->adv, o->fturb != 0,
                  o->fstruc != 0, p->t_eddy, p->t_stress, o->adv_beta, o->adv_fn,
                  o->fwall != 0, p->t_wall, o->rhie != 0, p->dsnap};
  const int blocks = (s->n + 255) / 256;
  const auto *loads_d = reinterpret_cast<const sfr::DevLoad *>(p->d_table);
  const auto *mtab =
      reinterpret_cast<const double *>(p->d_table + sizeof(sfr::DevLoad) * kTableLoads);
  auto launch = [&](auto kernel) {
    kernel<<<blocks, 256, 0, st>>>(p->d, loads_d, vo, p->d_mat, mtab, p->nmat, d_pres,
                                   d_gradpres, d_vel, d_gradvel, d_dfield, s->d_stage,
                                   s->d_diag, d_ad3, d_b3, d_rcell3, p->numel);
  };
  const bool ext = vo.adv != 1 || vo.fturb || vo.fstruc || vo.fwall || vo.rhie;
  if (p->d.maxviz == 6)
    ext ? launch(sfr::vel_assemble_kernel<6, true>) : launch(sfr::vel_assemble_kernel<6, false>);
  else
    ext ? launch(sfr::vel_assemble_kernel<sfr::kMaxViz, true>)
        : launch(sfr::vel_assemble_kernel<sfr::kMaxViz, false>);
  SFR_CUA(cudaGetLastError());
  if (matrix) return sfr::values_refreshed(s, st, false);
  return SFR_OK;
}

int sfr_gpu_vel_assemble(sfr_dif_plan *p, const sfr_load *lvel, int32_t nlvel,
                         const sfr_vel_opts *o, const double *prop, const double *pres,
                         const double *gradpres, const double *vel, const double *gradvel,
                         double *dfield, double *ad3, double *b3, double *rcell3, int32_t forces,
                         int32_t matrix, int32_t calrcell) {
  if (!p || !o) return bad("NULL argument");
  if (!pres || !gradpres || !vel || !gradvel || !dfield)
    return bad("pres, gradpres, vel, gradvel and dfield are required");
  if (p->kind != 2) return bad("not a momentum plan");
  sfr_system *s = p->s;
  SFR_CUA(cudaSetDevice(s->device));
  int rc = ensure_host_buffers(p);
  if (rc != SFR_OK) return rc;
  const size_t ne = p->numel, n = s->n;
  cudaStream_t st = s->stream;
  double *f = p->h_fields;
  double *d_pres = f, *d_gp = f + ne, *d_vel = f + 4 * ne, *d_gv = f + 7 * ne,
         *d_df = f + 16 * ne, *d_rc = p->h_rcell, *d_ad3 = p->h_b0, *d_b3 = p->h_b;
  auto cp = [&](void *dst, const void *src, size_t bytes, cudaMemcpyKind k) {
    if (rc == SFR_OK && cudaMemcpyAsync(dst, src, bytes, k, st) != cudaSuccess) {
      sfr::set_last_error("a copy of the host-array call failed");
      rc = SFR_CUDA_ERROR;
    }
  };
  cp(d_pres, pres, sizeof(double) * ne, cudaMemcpyHostToDevice);
  cp(d_gp, gradpres, sizeof(double) * ne * 3, cudaMemcpyHostToDevice);
  cp(d_vel, vel, sizeof(double) * ne * 3, cudaMemcpyHostToDevice);
  cp(d_gv, gradvel, sizeof(double) * ne * 9, cudaMemcpyHostToDevice);
  cp(d_df, dfield, sizeof(double) * ne * 3, cudaMemcpyHostToDevice);
  if (rc == SFR_OK)
    rc = sfr_gpu_vel_assemble_device(p, lvel, nlvel, o, prop, d_pres, d_gp, d_vel, d_gv, d_df,
                                     d_ad3, d_b3, d_rc, forces, matrix, calrcell, st);
  if (rc == SFR_OK) {
    cp(dfield, d_df, sizeof(double) * ne * 3, cudaMemcpyDeviceToHost);
    if (matrix && ad3) cp(ad3, d_ad3, sizeof(double) * n * 3, cudaMemcpyDeviceToHost);
    if (forces && b3) cp(b3, d_b3, sizeof(double) * n * 3, cudaMemcpyDeviceToHost);
    if (calrcell && rcell3) cp(rcell3, d_rc, sizeof(double) * ne * 3, cudaMemcpyDeviceToHost);
    if (rc == SFR_OK && cudaStreamSynchronize(st) != cudaSuccess) rc = SFR_CUDA_ERROR;
  }
  cudaStreamSynchronize(st);
  return rc;
}

int sfr_gpu_dif_update_cells(sfr_dif_plan *p, const double *d_x, double *d_u, int32_t add,
                             void *stream) {
  if (!p || !d_x || !d_u) return bad("NULL argument");
  SFR_CUA(cudaSetDevice(p->device));
  cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : p->s->stream;
  sfr::update_cells_kernel<<<(p->numel + 255) / 256, 256, 0, st>>>(p->d_id, p->numel, p->s->n,
                                                                     d_x, d_u, add != 0);
  SFR_CUA(cudaGetLastError());
  return SFR_OK;
}

int sfr_gpu_vel_turbulence(sfr_dif_plan *p, const double *eddy, const double *stress,
                           int32_t on_device) {
  if (!p) return bad("NULL argument");
  if (p->kind != 2) return bad("not a momentum plan");
  SFR_CUA(cudaSetDevice(p->device));
  if (on_device) {
    p->t_eddy = eddy;
    p->t_stress = stress;
    return SFR_OK;
  }
  const size_t ne = p->numel;
  p->t_eddy = p->t_stress = nullptr;
  if (eddy) {
    if (!p->own_eddy) SFR_CUA(cudaMalloc(&p->own_eddy, sizeof(double) * ne));
    SFR_CUA(cudaMemcpy(p->own_eddy, eddy, sizeof(double) * ne, cudaMemcpyHostToDevice));
    p->t_eddy = p->own_eddy;
  }
  if (stress) {
    if (!p->own_stress) SFR_CUA(cudaMalloc(&p->own_stress, sizeof(double) * ne * 6));
    SFR_CUA(cudaMemcpy(p->own_stress, stress, sizeof(double) * ne * 6, cudaMemcpyHostToDevice));
    p->t_stress = p->own_stress;
  }
  return SFR_OK;
}

int sfr_gpu_vel_wall(sfr_dif_plan *p, const double *wallpar, int32_t on_device) {
  if (!p) return bad("NULL argument");
  if (p->kind != 2) return bad("not a momentum plan");
  SFR_CUA(cudaSetDevice(p->device));
  if (on_device || !wallpar) {
    p->t_wall = wallpar;
    return SFR_OK;
  }
  const size_t bytes = sizeof(double) * 4 * static_cast<size_t>(p->numel);
  if (!p->own_wall) SFR_CUA(cudaMalloc(&p->own_wall, bytes));
  SFR_CUA(cudaMemcpy(p->own_wall, wallpar, bytes, cudaMemcpyHostToDevice));
  p->t_wall = p->own_wall;
  return SFR_OK;
}

int sfr_gpu_dif_plan_destroy(sfr_dif_plan *p) {
  if (!p) return SFR_OK;
  cudaSetDevice(p->device);
  free_plan_buffers(p);
  delete p;
  return SFR_OK;
}

}  // extern "C"
