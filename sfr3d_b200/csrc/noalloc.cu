// sfr_gpu_dot_noalloc: the deterministic dot product for callers that must
// not have this library allocate device memory.
//
// Who needs it: a program that reserves its device memory once at start-up
// and hands out pieces itself -- the way SFR3D manages host memory through a
// single arena (Memoria.c initMem/alloc) -- or one that runs while another
// allocator holds nearly all of the GPU's memory.  sfr_gpu_dot allocates its
// reduction scratch with cudaMalloc on first use; such a caller cannot let
// that happen mid-run.  This entry point keeps its scratch in a fixed
// file-scope device array instead, so it never calls cudaMalloc or cudaFree.
//
// Limits and rules:
//   * The scratch is 594 doubles (4,752 bytes) held by every GPU that loads
//     the library until the process exits: 592 block partials, one result,
//     one arrival counter.  The launch takes the same shape as sfr_gpu_dot
//     (4 blocks of 256 threads per SM, at most one block per 256 elements),
//     so both return the same bits; 592 partials cover a GPU of up to 148
//     SMs (a B200).  On a GPU with more SMs, or for a negative length, the
//     call returns SFR_BAD_INPUT, with the reason in sfr_last_error(),
//     before anything runs.
//   * The first call on a device looks up the array's device address (one
//     cudaGetSymbolAddress with that device current) and keeps it for the
//     life of the process.  Make that first call before any stream capture
//     starts.  cudaDeviceReset is not supported afterwards: the kept address
//     would go stale.
//   * Every call shares the one array and it keeps the last call's contents;
//     the arrival counter is cleared at the start of each call.  Calls whose
//     kernels overlap on the GPU (different streams, or different host
//     threads) race on the array: serialise them.
#include <cuda_runtime.h>

#include <mutex>

#include "internal.h"
#include "kernels.cuh"

namespace {

constexpr int kNoAllocBlocks = 592;               // block partials
constexpr int kNoAllocSlots = kNoAllocBlocks + 2; // + result + counter
constexpr int kNoAllocThreads = 256;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double g_noalloc_scratch[kNoAllocSlots];

double *g_scratch_addr[kMaxDevices] = {};
std::mutex g_scratch_mu;

// Device address of the scratch on the current device; looked up once per
// device (host code may not use the array's name as a device pointer).
int scratch_address(int device, double **out) {
  std::lock_guard<std::mutex> lk(g_scratch_mu);
  if (!g_scratch_addr[device]) {
    void *p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p)
      return SFR_CUDA_ERROR;
    g_scratch_addr[device] = static_cast<double *>(p);
  }
  *out = g_scratch_addr[device];
  return SFR_OK;
}

}  // namespace

extern "C" int sfr_gpu_dot_noalloc(const double *d_a, const double *d_b, int32_t n,
                                   double *dot_out, void *stream) {
  if (!d_a || !d_b || !dot_out) return SFR_BAD_INPUT;
  if (n < 0) {
    sfr::set_last_error("sfr_gpu_dot_noalloc: negative length");
    return SFR_BAD_INPUT;
  }
  int device = 0;
  if (cudaGetDevice(&device) != cudaSuccess) return SFR_CUDA_ERROR;
  if (device < 0 || device >= kMaxDevices) return SFR_BAD_INPUT;
  // sfr_gpu_dot's launch shape; its partials must fit the fixed scratch
  const int grid = sfr::stat_grid(device, n);
  static_assert(kNoAllocThreads == 256, "the launch shape of sfr_gpu_dot");
  if (grid > kNoAllocBlocks) {
    sfr::set_last_error("sfr_gpu_dot_noalloc: the device has more SMs than the fixed scratch "
                        "holds partials for (148)");
    return SFR_BAD_INPUT;
  }
  double *scratch = nullptr;
  const int rc = scratch_address(device, &scratch);
  if (rc != SFR_OK) return rc;
  double *partials = scratch;
  double *result = scratch + kNoAllocBlocks;
  unsigned *counter = reinterpret_cast<unsigned *>(scratch + kNoAllocBlocks + 1);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (cudaMemsetAsync(counter, 0, sizeof(unsigned), st) != cudaSuccess) return SFR_CUDA_ERROR;
  sfr::dot_kernel<<<grid, kNoAllocThreads, 0, st>>>(d_a, d_b, n, partials, counter, result);
  if (cudaGetLastError() != cudaSuccess) return SFR_CUDA_ERROR;
  if (cudaMemcpyAsync(dot_out, result, sizeof(double), cudaMemcpyDeviceToHost, st) != cudaSuccess)
    return SFR_CUDA_ERROR;
  return cudaStreamSynchronize(st) == cudaSuccess ? SFR_OK : SFR_CUDA_ERROR;
}
