// Deterministic block reductions shared by the FCG kernels (256-thread
// blocks): per-block partial sums written in block order, then summed by one
// block in a fixed tree order.
#pragma once

#include "common.cuh"
#include "kernels.h"

namespace bcmg {

constexpr int kRedThreads = 256;

// Block sum of NV doubles per thread into partials[blockIdx.x * 4 + k].
template <int NV>
__device__ __forceinline__ void block_partials(double (&v)[NV], double *partials) {
  __shared__ double sh[kRedThreads / 32][4];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < NV; ++k) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
    if (lane == 0) sh[wid][k] = v[k];
  }
  __syncthreads();
  if (threadIdx.x < NV) {
    double s = 0.0;
    for (int w = 0; w < kRedThreads / 32; ++w) s += sh[w][threadIdx.x];
    partials[blockIdx.x * 4 + threadIdx.x] = s;
  }
}

// Fixed-order sum of partial k over kRedBlocks blocks, by one block.
__device__ __forceinline__ double reduce_partials(const double *partials, int k) {
  __shared__ double sh[kRedThreads];
  double s = 0.0;
  for (int b = threadIdx.x; b < kRedBlocks; b += blockDim.x) s += partials[b * 4 + k];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  const double r = sh[0];
  __syncthreads();
  return r;
}

}  // namespace bcmg
