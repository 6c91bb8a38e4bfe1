// Device copies of the SELL matrix, value gathers, and the solve workspace.
#include <cuda_runtime.h>

#include <algorithm>

#include "internal.h"

namespace sfr {

namespace {

template <typename T>
cudaError_t upload(T **dst, const std::vector<T> &src, int64_t *bytes) {
  const size_t nb = sizeof(T) * std::max<size_t>(src.size(), 1);
  cudaError_t e = cudaMalloc(reinterpret_cast<void **>(dst), nb);
  if (e != cudaSuccess) return e;
  *bytes += static_cast<int64_t>(nb);
  if (!src.empty()) e = cudaMemcpy(*dst, src.data(), sizeof(T) * src.size(), cudaMemcpyHostToDevice);
  return e;
}

// val[e] = stage[src[e]] (or 0 for a padded slot); FP32 copy alongside.
__global__ void gather_kernel(const int *src, const double *stage, double *val, float *val32,
                              int64_t nslots) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; e < nslots;
       e += stride) {
    const int s = src[e];
    const double v = s >= 0 ? stage[s] : 0.0;
    val[e] = v;
    if (val32) val32[e] = __double2float_rn(v);
  }
}

__global__ void to_float_kernel(const double *src, float *dst, int n) {
  const int stride = gridDim.x * blockDim.x;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
    dst[i] = __double2float_rn(src[i]);
}

// comp[row] = -sum_e (fl32(val_e) - val_e) over the row's slots: the FP32
// operator with diagonal (ad + comp) has the same row sums as the FP64 one,
// so rounding the couplings does not disturb the near-null (smooth) modes
// of a diffusion operator.
__global__ void compensation_kernel(const int *sptr, const double *val, int n, int nslices,
                                    double *comp) {
  const int stride = gridDim.x * blockDim.x;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nslices * 32; t += stride) {
    const int s = t >> 5, lane = t & 31, row = t;
    if (row >= n) continue;
    const int base = sptr[s];
    const int w = (sptr[s + 1] - base) >> 5;
    double acc = 0.0;
    for (int k = 0; k < w; ++k) {
      const double v = val[base + k * 32 + lane];
      acc += static_cast<double>(__double2float_rn(v)) - v;
    }
    comp[row] = -acc;
  }
}

}  // namespace

int row_compensation(sfr_system *s, const DevSell &d, cudaStream_t st) {
  if (!s->d_comp) {
    if (cudaMalloc(&s->d_comp, sizeof(double) * std::max(s->n, 1)) != cudaSuccess)
      return SFR_CUDA_ERROR;
    s->bytes += static_cast<int64_t>(sizeof(double)) * s->n;
  }
  const int grid = static_cast<int>(std::min<int64_t>((static_cast<int64_t>(d.nslices) * 32 + 255) / 256, 4096));
  compensation_kernel<<<std::max(grid, 1), 256, 0, st>>>(d.sptr, d.val, s->n, d.nslices, s->d_comp);
  return cudaGetLastError() == cudaSuccess ? SFR_OK : SFR_CUDA_ERROR;
}

int upload_sell(const HostSell &h, DevSell *d, int64_t *bytes) {
  d->n = h.n;
  d->nslices = h.nslices;
  d->nslots = h.sptr.empty() ? 0 : h.sptr.back();
  d->max_width = h.max_width;
  if (upload(&d->sptr, h.sptr, bytes) != cudaSuccess) return SFR_CUDA_ERROR;
  if (upload(&d->col, h.col, bytes) != cudaSuccess) return SFR_CUDA_ERROR;
  if (upload(&d->src, h.src, bytes) != cudaSuccess) return SFR_CUDA_ERROR;
  if (h.bandwidth <= 32767) {  // 16-bit column offsets: 2 bytes a slot instead of 4
    std::vector<int16_t> off(h.col.size(), 0);
    for (int32_t s = 0; s < h.nslices; ++s)
      for (int32_t e = h.sptr[s]; e < h.sptr[s + 1]; ++e) {
        const int32_t row = s * kWarpHost + (e - h.sptr[s]) % kWarpHost;
        if (row < h.n) off[e] = static_cast<int16_t>(h.col[e] - row);
      }
    if (upload(&d->off, off, bytes) != cudaSuccess) return SFR_CUDA_ERROR;
  }
  const size_t ns = static_cast<size_t>(std::max<int64_t>(d->nslots, 1));
  if (cudaMalloc(&d->val, sizeof(double) * ns) != cudaSuccess) return SFR_CUDA_ERROR;
  if (cudaMalloc(&d->val32, sizeof(float) * ns) != cudaSuccess) return SFR_CUDA_ERROR;
  *bytes += static_cast<int64_t>((sizeof(double) + sizeof(float)) * ns);
  return SFR_OK;
}

void free_sell(DevSell *d) {
  cudaFree(d->sptr);
  cudaFree(d->col);
  cudaFree(d->src);
  cudaFree(d->off);
  cudaFree(d->val);
  cudaFree(d->val32);
  *d = DevSell{};
}

int gather_values(sfr_system *s, DevSell *d, cudaStream_t st) {
  if (d->nslots == 0) return SFR_OK;
  const int grid = static_cast<int>(std::min<int64_t>((d->nslots + 255) / 256, 4096));
  gather_kernel<<<grid, 256, 0, st>>>(d->src, s->d_stage, d->val, d->val32, d->nslots);
  return cudaGetLastError() == cudaSuccess ? SFR_OK : SFR_CUDA_ERROR;
}

cudaError_t convert_diag32(const double *src, float *dst, int n, cudaStream_t st) {
  const int grid = std::min((n + 255) / 256, 4096);
  to_float_kernel<<<std::max(grid, 1), 256, 0, st>>>(src, dst, n);
  return cudaGetLastError();
}

int ensure_workspace(sfr_system *s, size_t bytes) {
  if (s->ws.bytes >= bytes) return SFR_OK;
  if (s->ws.base) {
    cudaFree(s->ws.base);
    s->bytes -= static_cast<int64_t>(s->ws.bytes);
    s->ws = Workspace{};
  }
  void *p = nullptr;
  if (cudaMalloc(&p, bytes) != cudaSuccess) return SFR_CUDA_ERROR;
  s->ws.base = p;
  s->ws.bytes = bytes;
  s->bytes += static_cast<int64_t>(bytes);
  return SFR_OK;
}

}  // namespace sfr
