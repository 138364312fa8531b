// Device helpers shared by the kernels of librstg.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace rstg {

constexpr double kPi = 3.14159265358979323846;
constexpr double kKScale = 0.73;  // gb_energy.rs:300

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ float warp_sumf(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ int warp_sumi(int v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Deterministic block sum of one double per thread (blockDim multiple of 32,
// at most 1024 threads).  Result valid in thread 0.
__device__ __forceinline__ double block_sum(double v, double* sh) {
  v = warp_sum(v);
  int w = threadIdx.x >> 5, l = threadIdx.x & 31, nw = blockDim.x >> 5;
  __syncthreads();
  if (l == 0) sh[w] = v;
  __syncthreads();
  double r = 0.0;
  if (w == 0) {
    r = l < nw ? sh[l] : 0.0;
    r = warp_sum(r);
  }
  return r;
}

}  // namespace rstg
