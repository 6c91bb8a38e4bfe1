// Adjoint of a linear solve: for J(x) with x = A^-1 b and g = dJ/dx,
//   A^T lam = g,  dJ/db = lam,  dJ/dA_ij = -lam_i x_j  on the pattern.
// The reference has no adjoint; the transpose solve runs the same Krylov
// kernels on the transposed SELL copy (A^T row j = column j of A, diagonal
// first, then increasing column: the order of a sorted transposed CSRD).
#include <cuda_runtime.h>

#include <algorithm>

#include "common.cuh"
#include "internal.h"

namespace sfr {

namespace {

// g_src[src(e)] += -lam[row(e)] * x[col(e)] over every real slot e of A.
// A value stored once for two mirrored entries (strict-lower storage of a
// symmetric matrix) collects both terms; a sum of two terms does not depend
// on their order, so the result is deterministic.
__global__ void grad_values_kernel(const int *sptr, const int *col, const int *src, int nslices,
                                   int n, const double *lam, const double *x, double *g_src) {
  const int stride = gridDim.x * blockDim.x;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nslices * 32; t += stride) {
    const int s = t >> 5, lane = t & 31, row = t;
    if (row >= n) continue;
    const int base = sptr[s];
    const int w = (sptr[s + 1] - base) >> 5;
    const double li = lam[row];
    for (int k = 0; k < w; ++k) {
      const int e = base + k * 32 + lane;
      const int q = src[e];
      if (q >= 0) atomicAdd(g_src + q, -(li * x[col[e]]));
    }
  }
}

__global__ void grad_diag_kernel(const double *lam, const double *x, int n, double *g_ad) {
  const int stride = gridDim.x * blockDim.x;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) g_ad[i] = -(lam[i] * x[i]);
}

}  // namespace

int adjoint_gradients(sfr_system *s, const double *d_lam, const double *d_x, double *d_gsrc,
                      double *d_gad, cudaStream_t st) {
  if (cudaMemsetAsync(d_gsrc, 0, sizeof(double) * std::max(s->nsrc, 1), st) != cudaSuccess)
    return SFR_CUDA_ERROR;
  const int grid = static_cast<int>(
      std::min<int64_t>((static_cast<int64_t>(s->A.nslices) * 32 + 255) / 256, 4096));
  grad_values_kernel<<<std::max(grid, 1), 256, 0, st>>>(s->A.sptr, s->A.col, s->A.src,
                                                        s->A.nslices, s->n, d_lam, d_x, d_gsrc);
  grad_diag_kernel<<<std::max(1, std::min((s->n + 255) / 256, 4096)), 256, 0, st>>>(d_lam, d_x,
                                                                                    s->n, d_gad);
  return cudaGetLastError() == cudaSuccess ? SFR_OK : SFR_CUDA_ERROR;
}

}  // namespace sfr
