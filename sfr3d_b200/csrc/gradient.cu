// Gradient reconstruction on the device: rcGradU (CellLoop.c:4544-4790)
// with the Green-Gauss cell kernel (greenGaussCell, CellLib.c:2481-2780) or
// least squares (leastSquare, CellLib.c:2931-3215), no limiter, ndm = 3,
// ndf 1 (pressure, a scalar) or 3 (velocity).
//
// The SIMPLE driver reconstructs the velocity and pressure gradients before
// each assembly (Simple.c:2797-2858); with this kernel they are formed where
// the fields already are, and the assembly kernels read them from HBM.
//
// Layout.  The plan holds, per (face slot f, cell c) with stride numel, the
// face's neighbour (or its load, encoded -(load index) - 2; -1 a boundary
// face without a load), and the words the cell kernel reads for that face:
//   Green-Gauss: the interpolation weight alpha, the area, the outward
//                normal (3), xmcc (3), dcca;
//   least squares: the three entries of the cell's matrix for the face,
//                xmcc (3), dcca.
// Per cell: the face count, the material, 1/volume (Green-Gauss).  Both
// alpha and the least-squares matrix depend on the mesh alone; the plan
// computes them once on the host with the reference's own expressions (one
// IEEE rounding per operation: the host build has no FMA contraction, and
// pow is the same libm call), as the reference computes its matrices once
// (rcLeastSquare, Main.c:736).
//
// One thread per cell; the cell reads only its own previous gradient, so the
// update is in place, as in the reference.  Every face sum runs in face order
// with one rounding per multiply and per add (xmul/xadd), so the result is
// bit-identical to rcGradU's.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "internal.h"

struct sfr_grad_plan {
  int device = 0;
  int type = 0;
  int32_t numel = 0, maxviz = 0, nmat = 0;
  uint64_t used_loads = 0;              // loads some boundary face names (index bits)
  std::vector<uint64_t> load_mats;      // per load: materials of the cells naming it
  int32_t *nb = nullptr;                // [maxviz][numel]
  double *geo = nullptr;                // [nwords][maxviz][numel]
  int16_t *nface = nullptr, *mat = nullptr;
  double *inv_vol = nullptr;            // Green-Gauss
  void *table = nullptr;                // loads, then the COEFDIF of each material
  std::vector<unsigned char> table_host;
  double *d_u = nullptr, *d_g = nullptr;  // host-buffer calls: staging
  cudaStream_t stream = nullptr;
  int64_t bytes = 0;
};

namespace sfr {
namespace {

constexpr int kGradMaxViz = 8;
constexpr int kGradMaxLoads = 32;
constexpr int kGaussWords = 10;  // alpha, area, normal (3), xmcc (3), dcca
constexpr int kLsqWords = 7;     // L (3), xmcc (3), dcca

enum {
  kDirichlet = 1, kNeumann = 2, kRobin = 3, kSinbc = 4, kInlet = 6, kOutlet = 7, kMoveWall = 8,
  kInletStatic = 9, kOpen = 10, kConvectionHeat = 11, kStaticWall = 14, kFluxPres = 15,
  kFluxPresC = 16
};

struct GradLoad {
  int32_t type, pad;
  double par[3];
};

struct GradDev {
  int numel;
  size_t fs;  // maxviz * numel: distance between geometry words
  const int32_t *nb;
  const double *geo;
  const int16_t *nface, *mat;
  const double *inv_vol;
};

// uC + sum_j g_j x_j in the reference's order (a running sum from uC)
__device__ __forceinline__ double extrap(double uc, const double g[3], const double x[3]) {
  double v = uc;
#pragma unroll
  for (int j = 0; j < 3; ++j) v = xadd(v, xmul(g[j], x[j]));
  return v;
}

// A cell's neighbours and their values, loaded for every face before any
// face is computed (kMV face slots unrolled), so the gathers of all faces are
// in flight together.  Taken for the velocity (ndf 3: at 128^3 least squares
// 0.256 -> 0.222 ms, Green-Gauss 0.285 -> 0.253 ms); for a scalar the extra
// registers cost more than they save (least squares 0.151 -> 0.384 ms), and
// the face loop reads each value where it needs it.
template <int NDF, int kMV>
__device__ __forceinline__ void neighbour_values(const GradDev &d, const double *__restrict__ u,
                                                 int c, int nf, int (&nbs)[kMV],
                                                 double (&un)[kMV][NDF]) {
#pragma unroll
  for (int f = 0; f < kMV; ++f) nbs[f] = f < nf ? d.nb[static_cast<size_t>(f) * d.numel + c] : -1;
#pragma unroll
  for (int f = 0; f < kMV; ++f)
#pragma unroll
    for (int k = 0; k < NDF; ++k)
      un[f][k] = nbs[f] >= 0 ? u[static_cast<size_t>(nbs[f]) * NDF + k] : 0.0;
}

// greenGaussCell (CellLib.c:2481-2780) for one cell
template <int NDF, int kMV>
__global__ void __launch_bounds__(256) gauss_cell_kernel(GradDev d, const GradLoad *__restrict__ ld,
                                                         const double *__restrict__ coefdif,
                                                         const double *__restrict__ u,
                                                         double *__restrict__ gradu) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= d.numel) return;
  const int nf = d.nface[c];
  const double coef = coefdif[d.mat[c] - 1];
  constexpr bool kPre = NDF > 1;
  int nbs[kPre ? kMV : 1];
  double un[kPre ? kMV : 1][NDF];
  if constexpr (kPre) neighbour_values<NDF, kMV>(d, u, c, nf, nbs, un);
  double uC[NDF], gold[NDF][3], acc[NDF][3];
#pragma unroll
  for (int k = 0; k < NDF; ++k) {
    uC[k] = u[static_cast<size_t>(c) * NDF + k];
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      gold[k][j] = gradu[(static_cast<size_t>(c) * NDF + k) * 3 + j];
      acc[k][j] = 0.0;
    }
  }
  const size_t fs = d.fs;
  auto face = [&](int f) {
    const size_t o = static_cast<size_t>(f) * d.numel + c;
    const int nb = kPre ? nbs[kPre ? f : 0] : d.nb[o];
    const double *g = d.geo + o;
    const double area = g[fs];
    const double n[3] = {g[2 * fs], g[3 * fs], g[4 * fs]};
    double uf[NDF];
    if (nb >= 0) {
      const double alpha = g[0];
      const double am1 = xsub(1.0e0, alpha);
#pragma unroll
      for (int k = 0; k < NDF; ++k)
        uf[k] = xadd(xmul(am1, uC[k]),
                     xmul(alpha, kPre ? un[kPre ? f : 0][k] : u[static_cast<size_t>(nb) * NDF + k]));
    } else {
      const double x[3] = {g[5 * fs], g[6 * fs], g[7 * fs]};
      if (nb == -1) {
#pragma unroll
        for (int k = 0; k < NDF; ++k) uf[k] = extrap(uC[k], gold[k], x);
      } else {
        const GradLoad &L = ld[-nb - 2];
        const double dcca = g[8 * fs];
        if (NDF == 1) {
          if (L.type == kDirichlet || L.type == kInlet) {
            uf[0] = L.par[0];
          } else if (L.type == kFluxPres) {  // gradPbBuoyant without buoyancy: 0
            uf[0] = xadd(uC[0], xadd(xadd(xmul(0.0, x[0]), xmul(0.0, x[1])), xmul(0.0, x[2])));
          } else if (L.type == kNeumann) {
            uf[0] = xadd(uC[0], xmul(xdiv(L.par[0], coef), dcca));
          } else if (L.type == kRobin || L.type == kConvectionHeat) {
            uf[0] = extrap(uC[0], gold[0], x);
          } else {  // FLUXPRESC, OUTLET (the host rejects the rest)
            uf[0] = uC[0];
          }
        } else {
          if (L.type == kDirichlet || L.type == kMoveWall || L.type == kInlet) {
#pragma unroll
            for (int k = 0; k < NDF; ++k) uf[k] = L.par[k];
          } else if (L.type == kStaticWall) {
#pragma unroll
            for (int k = 0; k < NDF; ++k) uf[k] = 0.e0;
          } else if (L.type == kNeumann) {
#pragma unroll
            for (int k = 0; k < NDF; ++k) uf[k] = xadd(uC[k], xmul(xdiv(L.par[k], coef), dcca));
          } else {  // OUTLET, INLETSTAICTPRES, OPEN
#pragma unroll
            for (int k = 0; k < NDF; ++k) uf[k] = uC[k];
          }
        }
      }
    }
#pragma unroll
    for (int k = 0; k < NDF; ++k)
#pragma unroll
      for (int j = 0; j < 3; ++j) acc[k][j] = xadd(acc[k][j], xmul(xmul(uf[k], area), n[j]));
  };
  if constexpr (kPre) {
#pragma unroll
    for (int f = 0; f < kMV; ++f)
      if (f < nf) face(f);
  } else {
    for (int f = 0; f < nf; ++f) face(f);
  }
  const double iv = d.inv_vol[c];
#pragma unroll
  for (int k = 0; k < NDF; ++k)
#pragma unroll
    for (int j = 0; j < 3; ++j)
      gradu[(static_cast<size_t>(c) * NDF + k) * 3 + j] = xmul(acc[k][j], iv);
}

// leastSquare (CellLib.c:2931-3215) for one cell: gradU = L du, twice when a
// face extrapolates with the gradient (the second pass with the first's)
template <int NDF, int kMV>
__global__ void __launch_bounds__(256) least_squares_kernel(GradDev d,
                                                            const GradLoad *__restrict__ ld,
                                                            const double *__restrict__ coefdif,
                                                            const double *__restrict__ u,
                                                            double *__restrict__ gradu) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= d.numel) return;
  const int nf = d.nface[c];
  const double coef = coefdif[d.mat[c] - 1];
  const size_t fs = d.fs;
  constexpr bool kPre = NDF > 1;
  int nbs[kPre ? kMV : 1];
  double un[kPre ? kMV : 1][NDF];
  if constexpr (kPre) neighbour_values<NDF, kMV>(d, u, c, nf, nbs, un);
  double uC[NDF], gr[NDF][3];
#pragma unroll
  for (int k = 0; k < NDF; ++k) {
    uC[k] = u[static_cast<size_t>(c) * NDF + k];
#pragma unroll
    for (int j = 0; j < 3; ++j) gr[k][j] = 0.e0;
  }
  int it = 1;
  for (int pass = 0; pass < it; ++pass) {
    double acc[NDF][3];
#pragma unroll
    for (int k = 0; k < NDF; ++k)
#pragma unroll
      for (int j = 0; j < 3; ++j) acc[k][j] = 0.e0;
    auto face = [&](int f) {
      const size_t o = static_cast<size_t>(f) * d.numel + c;
      const int nb = kPre ? nbs[kPre ? f : 0] : d.nb[o];
      const double *g = d.geo + o;
      double du[NDF];
#pragma unroll
      for (int k = 0; k < NDF; ++k) du[k] = 0.e0;
      if (nb >= 0) {
#pragma unroll
        for (int k = 0; k < NDF; ++k)
          du[k] = xsub(kPre ? un[kPre ? f : 0][k] : u[static_cast<size_t>(nb) * NDF + k], uC[k]);
      } else {
        const double x[3] = {g[3 * fs], g[4 * fs], g[5 * fs]};
        if (nb == -1) {
          it = 2;
#pragma unroll
          for (int k = 0; k < NDF; ++k) du[k] = extrap(0.e0, gr[k], x);
        } else {
          const int li = -nb - 2;
          const GradLoad &L = ld[li];
          if (NDF == 1) {
            if (L.type == kDirichlet || L.type == kMoveWall || L.type == kInlet) {
              du[0] = xsub(L.par[0], uC[0]);
            } else if (L.type == kFluxPres) {
              du[0] = xadd(xadd(xmul(0.0, x[0]), xmul(0.0, x[1])), xmul(0.0, x[2]));
            } else if (L.type == kNeumann) {
              if (coef != 0.e0) du[0] = xmul(xdiv(L.par[0], coef), g[6 * fs]);
            } else if (L.type == kRobin || L.type == kConvectionHeat) {
              it = 2;
              du[0] = extrap(0.e0, gr[0], x);
            }
          } else {
            if (L.type == kDirichlet || L.type == kMoveWall) {
#pragma unroll
              for (int k = 0; k < NDF; ++k) du[k] = xsub(L.par[k], uC[k]);
            } else if (li + 1 == kStaticWall) {
              // the reference compares the load's index, not its type, with
              // STATICWALL (CellLib.c:3118)
#pragma unroll
              for (int k = 0; k < NDF; ++k) du[k] = -uC[k];
            } else if (L.type == kInlet) {
#pragma unroll
              for (int k = 0; k < NDF; ++k) du[k] = xsub(L.par[k], uC[k]);
            }
          }
        }
      }
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        const double l = g[i * fs];
#pragma unroll
        for (int k = 0; k < NDF; ++k) acc[k][i] = xadd(acc[k][i], xmul(l, du[k]));
      }
    };
    if constexpr (kPre) {
#pragma unroll
      for (int f = 0; f < kMV; ++f)
        if (f < nf) face(f);
    } else {
      for (int f = 0; f < nf; ++f) face(f);
    }
#pragma unroll
    for (int k = 0; k < NDF; ++k)
#pragma unroll
      for (int j = 0; j < 3; ++j) gr[k][j] = acc[k][j];
  }
#pragma unroll
  for (int k = 0; k < NDF; ++k)
#pragma unroll
    for (int j = 0; j < 3; ++j) gradu[(static_cast<size_t>(c) * NDF + k) * 3 + j] = gr[k][j];
}

int bad(const char *why) {
  set_last_error(why);
  return SFR_BAD_INPUT;
}

int unsupported(const char *why) {
  set_last_error(why);
  return SFR_UNSUPPORTED;
}

#define SFR_CUG(expr)                              \
  do {                                             \
    cudaError_t e_ = (expr);                       \
    if (e_ != cudaSuccess) {                       \
      set_last_error(cudaGetErrorString(e_));      \
      return SFR_CUDA_ERROR;                       \
    }                                              \
  } while (0)

template <typename T>
cudaError_t upload(T **d, const std::vector<T> &h, int64_t *bytes) {
  const size_t b = sizeof(T) * std::max<size_t>(h.size(), 1);
  cudaError_t e = cudaMalloc(d, b);
  if (e != cudaSuccess) return e;
  *bytes += static_cast<int64_t>(b);
  if (h.empty()) return cudaSuccess;
  return cudaMemcpy(*d, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice);
}

// leastSquareMatrix with RCLSQUARE, ndm = 3 (CellLib.c:3500-3590): L (3 x
// nf) of one cell from its faces' ch-signed ksi and |ksi|
void ls_matrix(int nf, const double (*ksi)[3], const double *mk, double (*L)[kGradMaxViz]) {
  double dx[kGradMaxViz][3], w[kGradMaxViz], a[6] = {0, 0, 0, 0, 0, 0}, inv[6];
  for (int f = 0; f < nf; ++f) {
    w[f] = 1.e0 / std::pow(mk[f], 2.0);
    for (int j = 0; j < 3; ++j) dx[f][j] = ksi[f][j] * mk[f];
    a[0] += w[f] * dx[f][0] * dx[f][0];
    a[1] += w[f] * dx[f][0] * dx[f][1];
    a[2] += w[f] * dx[f][0] * dx[f][2];
    a[3] += w[f] * dx[f][1] * dx[f][1];
    a[4] += w[f] * dx[f][1] * dx[f][2];
    a[5] += w[f] * dx[f][2] * dx[f][2];
  }
  double det = a[0] * a[3] * a[5] + 2.e0 * a[1] * a[4] * a[2] -
               (a[2] * a[2] * a[3] + a[4] * a[4] * a[0] + a[1] * a[1] * a[5]);
  det = 1.e0 / det;
  inv[0] = (a[3] * a[5] - a[4] * a[4]) * det;
  inv[1] = -(a[1] * a[5] - a[2] * a[4]) * det;
  inv[2] = (a[1] * a[4] - a[2] * a[3]) * det;
  inv[3] = (a[0] * a[5] - a[2] * a[2]) * det;
  inv[4] = -(a[0] * a[4] - a[1] * a[2]) * det;
  inv[5] = (a[0] * a[3] - a[1] * a[1]) * det;
  for (int f = 0; f < nf; ++f) {
    L[0][f] = w[f] * (dx[f][0] * inv[0] + dx[f][1] * inv[1] + dx[f][2] * inv[2]);
    L[1][f] = w[f] * (dx[f][0] * inv[1] + dx[f][1] * inv[3] + dx[f][2] * inv[4]);
    L[2][f] = w[f] * (dx[f][0] * inv[2] + dx[f][1] * inv[4] + dx[f][2] * inv[5]);
  }
}

}  // namespace
}  // namespace sfr

using sfr::bad;
using sfr::unsupported;

extern "C" {

int sfr_gpu_grad_plan_create(int32_t device, const sfr_dif_mesh *mesh, int32_t type,
                             sfr_grad_plan **out) {
  using namespace sfr;
  if (!mesh || !out) return bad("NULL argument");
  *out = nullptr;
  const sfr_dif_mesh &m = *mesh;
  if (type != 1 && type != 3)
    return unsupported("rcGrad type: Green-Gauss cell (1) and least squares (3) are restated");
  if (m.numel < 1 || m.maxviz < 1 || m.maxviz > kGradMaxViz || m.nfaces < 1 || m.nmat < 1 ||
      m.nmat > 64)
    return bad("mesh sizes out of range (maxviz 1..8, nmat 1..64)");
  const void *need[] = {m.nelcon, m.nviz, m.cellface, m.owner, m.volume, m.dcca, m.xmcc,
                        m.mksi,   m.ksi,  m.area,     m.normal, m.vskew, m.mat,  m.facer};
  for (const void *q : need)
    if (!q) return bad("a mesh array is NULL");
  const int32_t numel = m.numel, mv = m.maxviz;
  const size_t fsz = static_cast<size_t>(mv) * numel;
  const int nw = type == 1 ? kGaussWords : kLsqWords;
  std::vector<int32_t> nb(fsz, -1);
  std::vector<double> geo(static_cast<size_t>(nw) * fsz, 0.0);
  std::vector<int16_t> nface(numel), mat(numel);
  std::vector<double> inv_vol(type == 1 ? numel : 0);
  std::vector<uint64_t> load_mats(kGradMaxLoads, 0);
  uint64_t used = 0;
  for (int32_t c = 0; c < numel; ++c) {
    const int nf = m.nviz[c];
    if (nf < 1 || nf > mv) return bad("a cell's face count is out of range");
    if (m.mat[c] < 1 || m.mat[c] > m.nmat) return bad("a cell's material is out of range");
    nface[c] = static_cast<int16_t>(nf);
    mat[c] = m.mat[c];
    if (type == 1) inv_vol[c] = 1.e0 / m.volume[c];
    double ksi[kGradMaxViz][3], mk[kGradMaxViz], L[3][kGradMaxViz];
    for (int f = 0; f < nf; ++f) {
      const size_t q = static_cast<size_t>(c) * mv + f;
      const int64_t face = static_cast<int64_t>(m.cellface[q]) - 1;
      if (face < 0 || face >= m.nfaces) return bad("a cell face is out of range");
      const int64_t own = m.owner[2 * face] - 1;
      if (own < 0 || own >= numel) return bad("a face owner is out of range");
      const double ch = own == c ? 1.0 : -1.0;
      mk[f] = m.mksi[face];
      for (int j = 0; j < 3; ++j) ksi[f][j] = ch * m.ksi[3 * face + j];
    }
    if (type == 3) ls_matrix(nf, ksi, mk, L);
    for (int f = 0; f < nf; ++f) {
      const size_t q = static_cast<size_t>(c) * mv + f;
      const size_t o = static_cast<size_t>(f) * numel + c;
      const int64_t face = static_cast<int64_t>(m.cellface[q]) - 1;
      const double ch = m.owner[2 * face] - 1 == c ? 1.0 : -1.0;
      const int viz = m.nelcon[q] - 1;
      auto G = [&](int w) -> double & { return geo[static_cast<size_t>(w) * fsz + o]; };
      if (viz > -1) {
        if (viz >= numel) return bad("a neighbour is out of range");
        nb[o] = viz;
      } else if (viz == -2) {
        const int ld = m.facer[static_cast<size_t>(c) * (mv + 1) + f];
        if (ld < 0 || ld > kGradMaxLoads) return bad("a face load is out of range (0..32)");
        if (ld > 0) {
          nb[o] = -(ld - 1) - 2;
          used |= 1ull << (ld - 1);
          load_mats[ld - 1] |= 1ull << (m.mat[c] - 1);
        }
      } else {
        return bad("a neighbour is out of range");
      }
      if (type == 1) {
        // interpolFace, INTPOLFACELINEAR (CellLib.c:7174-7200), called with
        // the cell's skew and xmcc arrays themselves (CellLib.c:2513, 2640):
        // every face reads its first face's vSkew and xmcc, |ksi| its own
        const size_t q0 = static_cast<size_t>(c) * mv;
        const int64_t face0 = static_cast<int64_t>(m.cellface[q0]) - 1;
        double v[3];
        for (int j = 0; j < 3; ++j) v[j] = m.vskew[3 * face0 + j] + m.xmcc[3 * q0 + j];
        G(0) = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]) / m.mksi[face];
        G(1) = m.area[face];
        for (int j = 0; j < 3; ++j) {
          G(2 + j) = ch * m.normal[3 * face + j];
          G(5 + j) = m.xmcc[3 * q + j];
        }
        G(8) = m.dcca[q];
      } else {
        for (int j = 0; j < 3; ++j) {
          G(j) = L[j][f];
          G(3 + j) = m.xmcc[3 * q + j];
        }
        G(6) = m.dcca[q];
      }
    }
  }
  SFR_CUG(cudaSetDevice(device));
  auto *p = new sfr_grad_plan;
  p->device = device;
  p->type = type;
  p->numel = numel;
  p->maxviz = mv;
  p->nmat = m.nmat;
  p->used_loads = used;
  p->load_mats = load_mats;
  cudaError_t e = upload(&p->nb, nb, &p->bytes);
  if (e == cudaSuccess) e = upload(&p->geo, geo, &p->bytes);
  if (e == cudaSuccess) e = upload(&p->nface, nface, &p->bytes);
  if (e == cudaSuccess) e = upload(&p->mat, mat, &p->bytes);
  if (e == cudaSuccess && type == 1) e = upload(&p->inv_vol, inv_vol, &p->bytes);
  if (e == cudaSuccess)
    e = cudaMalloc(&p->table, sizeof(GradLoad) * kGradMaxLoads + sizeof(double) * 64);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    set_last_error(cudaGetErrorString(e));
    sfr_gpu_grad_plan_destroy(p);
    return SFR_CUDA_ERROR;
  }
  *out = p;
  return SFR_OK;
}

int sfr_gpu_grad_plan_destroy(sfr_grad_plan *p) {
  if (!p) return SFR_OK;
  cudaSetDevice(p->device);
  if (p->stream) cudaStreamSynchronize(p->stream);
  cudaFree(p->nb);
  cudaFree(p->geo);
  cudaFree(p->nface);
  cudaFree(p->mat);
  cudaFree(p->inv_vol);
  cudaFree(p->table);
  cudaFree(p->d_u);
  cudaFree(p->d_g);
  if (p->stream) cudaStreamDestroy(p->stream);
  delete p;
  return SFR_OK;
}

int sfr_gpu_grad_device(sfr_grad_plan *p, const sfr_load *loads, int32_t nloads,
                        const double *prop, int32_t ndf, const double *d_u, double *d_gradu,
                        void *stream) {
  using namespace sfr;
  if (!p || !prop || !d_u || !d_gradu) return bad("NULL argument");
  if (ndf != 1 && ndf != 3) return bad("ndf must be 1 or 3");
  if (nloads < 0 || nloads > kGradMaxLoads || (nloads > 0 && !loads))
    return bad("nloads must be 0..32");
  // the loads the faces name, against what each branch of the reference
  // defines (an undefined face value is SFR_BAD_INPUT, as the oracle's -1)
  for (int l = 0; l < kGradMaxLoads; ++l) {
    if (!(p->used_loads & (1ull << l))) continue;
    if (l >= nloads) return bad("a boundary face names a load beyond nloads");
    const sfr_load &L = loads[l];
    if (L.type == kSinbc) return unsupported("SINBC faces are not restated");
    if ((L.type == kDirichlet || L.type == kInlet) && L.var != 0)
      return unsupported("loads given as functions (nTypeVar 1) are not restated");
    bool zero_coef = false;
    for (int k = 0; k < p->nmat; ++k)
      if ((p->load_mats[l] & (1ull << k)) && prop[k * 10 + 0] == 0.e0) zero_coef = true;
    if (p->type == 1) {
      if (ndf == 1) {
        const int ok[] = {kDirichlet, kInlet, kFluxPres, kFluxPresC, kNeumann, kRobin,
                          kConvectionHeat, kOutlet};
        bool hit = false;
        for (int t : ok) hit |= L.type == t;
        if (!hit) return bad("greenGaussCell (ndf 1) defines no face value for this load type");
      } else {
        const int ok[] = {kDirichlet, kMoveWall, kStaticWall, kInlet, kNeumann, kOutlet,
                          kInletStatic, kOpen};
        bool hit = false;
        for (int t : ok) hit |= L.type == t;
        if (!hit) return bad("greenGaussCell (ndf 3) defines no face value for this load type");
      }
      if (L.type == kNeumann && zero_coef)
        return bad("greenGaussCell leaves a NEUMANN face undefined where COEFDIF is 0");
    } else if (ndf == 3 && (L.type == kRobin || L.type == kConvectionHeat)) {
      return bad("leastSquare (ndf 3) stops on ROBIN faces");
    }
  }
  std::vector<unsigned char> h(sizeof(GradLoad) * kGradMaxLoads + sizeof(double) * 64, 0);
  auto *t = reinterpret_cast<GradLoad *>(h.data());
  for (int l = 0; l < nloads; ++l) {
    t[l].type = loads[l].type;
    for (int k = 0; k < 3; ++k) t[l].par[k] = loads[l].par[k];
  }
  auto *cd = reinterpret_cast<double *>(h.data() + sizeof(GradLoad) * kGradMaxLoads);
  for (int k = 0; k < p->nmat; ++k) cd[k] = prop[k * 10 + 0];  // MAXPROP 10, COEFDIF 0
  SFR_CUG(cudaSetDevice(p->device));
  cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : p->stream;
  if (h != p->table_host) {
    SFR_CUG(cudaMemcpyAsync(p->table, h.data(), h.size(), cudaMemcpyHostToDevice, st));
    SFR_CUG(cudaStreamSynchronize(st));  // h is this call's local
    p->table_host = h;
  }
  GradDev d{p->numel, static_cast<size_t>(p->maxviz) * p->numel, p->nb, p->geo, p->nface,
            p->mat, p->inv_vol};
  const auto *ld = static_cast<const GradLoad *>(p->table);
  const auto *coef = reinterpret_cast<const double *>(static_cast<const char *>(p->table) +
                                                      sizeof(GradLoad) * kGradMaxLoads);
  const int blocks = (p->numel + 255) / 256;
  // hexahedral meshes (six faces) get their own unrolled instantiation
  auto launch = [&](auto kernel) { kernel<<<blocks, 256, 0, st>>>(d, ld, coef, d_u, d_gradu); };
  const bool hex = p->maxviz == 6;
  if (p->type == 1) {
    if (ndf == 1)
      hex ? launch(gauss_cell_kernel<1, 6>) : launch(gauss_cell_kernel<1, kGradMaxViz>);
    else
      hex ? launch(gauss_cell_kernel<3, 6>) : launch(gauss_cell_kernel<3, kGradMaxViz>);
  } else {
    if (ndf == 1)
      hex ? launch(least_squares_kernel<1, 6>) : launch(least_squares_kernel<1, kGradMaxViz>);
    else
      hex ? launch(least_squares_kernel<3, 6>) : launch(least_squares_kernel<3, kGradMaxViz>);
  }
  SFR_CUG(cudaGetLastError());
  return SFR_OK;
}

int sfr_gpu_grad(sfr_grad_plan *p, const sfr_load *loads, int32_t nloads, const double *prop,
                 int32_t ndf, const double *u, double *gradu) {
  using namespace sfr;
  if (!p || !u || !gradu) return bad("NULL argument");
  if (ndf != 1 && ndf != 3) return bad("ndf must be 1 or 3");
  SFR_CUG(cudaSetDevice(p->device));
  const size_t nu = static_cast<size_t>(p->numel) * ndf;
  if (!p->d_u) {
    SFR_CUG(cudaMalloc(&p->d_u, sizeof(double) * static_cast<size_t>(p->numel) * 3));
    SFR_CUG(cudaMalloc(&p->d_g, sizeof(double) * static_cast<size_t>(p->numel) * 9));
  }
  SFR_CUG(cudaMemcpyAsync(p->d_u, u, sizeof(double) * nu, cudaMemcpyHostToDevice, p->stream));
  SFR_CUG(cudaMemcpyAsync(p->d_g, gradu, sizeof(double) * nu * 3, cudaMemcpyHostToDevice,
                          p->stream));
  const int rc = sfr_gpu_grad_device(p, loads, nloads, prop, ndf, p->d_u, p->d_g, p->stream);
  if (rc != SFR_OK) {
    cudaStreamSynchronize(p->stream);
    return rc;
  }
  SFR_CUG(cudaMemcpyAsync(gradu, p->d_g, sizeof(double) * nu * 3, cudaMemcpyDeviceToHost,
                          p->stream));
  SFR_CUG(cudaStreamSynchronize(p->stream));
  return SFR_OK;
}

}  // extern "C"
