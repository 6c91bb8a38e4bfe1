// Declarations of kernels launched from more than one translation unit.
#pragma once

#include <cstdint>

namespace sfr {

// Deterministic (a, b): per-block partials, the last block to finish sums
// them in a fixed order and resets *counter (krylov.cu).
__global__ void dot_kernel(const double *a, const double *b, int n, double *part,
                           unsigned *counter, double *out);

}  // namespace sfr
