// reduce.cuh — deterministic FP64 block reductions shared by the observables kernels and the
// measuring heatbath pass.
#pragma once
#include <cuda_runtime.h>

namespace qcb {

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// Block-wide sum of v (valid in thread 0); sh holds NT/32 doubles.  Every thread of the block
// must call it.
template <int NT>
__device__ __forceinline__ double block_sum(double v, double* sh) {
  v = warp_sum(v);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) sh[w] = v;
  __syncthreads();
  double r = 0;
  if (w == 0) {
    r = (lane < NT / 32) ? sh[lane] : 0.0;
    r = warp_sum(r);
  }
  __syncthreads();
  return r;
}

__device__ __forceinline__ void neumaier_add(double& s, double& c, double v) {
  const double t = s + v;
  if (fabs(s) >= fabs(v))
    c += (s - t) + v;
  else
    c += (v - t) + s;
  s = t;
}

}  // namespace qcb
