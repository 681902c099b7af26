// SPDX-License-Identifier: Apache-2.0
// Block-level folds of the per-world float64 reductions (256 threads).
#pragma once

#include <cuda_runtime.h>

namespace adf {

// Fixed tree order (the oracle mirrors it): lanes fold in groups of 32 with offsets 16..1, then the 8 group sums
// with offsets 4, 2, 1. Chunks of 256 particles are aligned to each world's start in the caller's order.
__device__ __forceinline__ double fold256(double v, double* sm) {
#pragma unroll
  for (int o = 16; o >= 1; o >>= 1) v = v + __shfl_down_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = v;
  __syncthreads();
  double r = 0.0;
  if (threadIdx.x == 0) {
    double s[8];
#pragma unroll
    for (int g = 0; g < 8; ++g) s[g] = sm[g];
#pragma unroll
    for (int o = 4; o >= 1; o >>= 1)
#pragma unroll
      for (int l = 0; l < o; ++l) s[l] = s[l] + s[l + o];
    r = s[0];
  }
  __syncthreads();
  return r;
}

__device__ __forceinline__ float block_max256(float v, float* sm) {
#pragma unroll
  for (int o = 16; o >= 1; o >>= 1) v = fmaxf(v, __shfl_down_sync(0xffffffffu, v, o));
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = v;
  __syncthreads();
  float r = -3.4e38f;
  if (threadIdx.x == 0)
    for (int g = 0; g < 8; ++g) r = fmaxf(r, sm[g]);
  __syncthreads();
  return r;
}

}  // namespace adf
