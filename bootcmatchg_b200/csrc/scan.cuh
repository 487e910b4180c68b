// Device-wide exclusive prefix sum of int32 (three passes: tile totals, scan
// of tile totals, tile scans plus offsets).  Deterministic; replaces the
// reference's CUB/Thrust scans (src/utility/utils.cu:70-133,
// kernel_spgemm_hash_d.cu:1183).
#pragma once

#include "common.cuh"

namespace bcmg {
namespace {  // kernels get internal linkage in every file that includes this
namespace scan_detail {

constexpr int kBlock = 256;
constexpr int kItems = 8;
constexpr int kTile = kBlock * kItems;

// Inclusive scan of one value per thread across the block; returns the
// inclusive prefix and the block total in *total.
__device__ __forceinline__ int block_inclusive(int v, int *warp_tot, int *total) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int t = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += t;
  }
  if (lane == 31) warp_tot[wid] = v;
  __syncthreads();
  if (wid == 0) {
    int w = lane < (kBlock / 32) ? warp_tot[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int t = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += t;
    }
    if (lane < (kBlock / 32)) warp_tot[lane] = w;
  }
  __syncthreads();
  const int add = wid > 0 ? warp_tot[wid - 1] : 0;
  *total = warp_tot[kBlock / 32 - 1];
  return v + add;
}

__global__ void tile_sums(const int32_t *__restrict__ in, int64_t n, int32_t *tile_tot) {
  __shared__ int wt[kBlock / 32];
  const int64_t base = static_cast<int64_t>(blockIdx.x) * kTile;
  int s = 0;
#pragma unroll
  for (int k = 0; k < kItems; ++k) {
    int64_t i = base + static_cast<int64_t>(threadIdx.x) * kItems + k;
    if (i < n) s += in[i];
  }
  int tot;
  block_inclusive(s, wt, &tot);
  if (threadIdx.x == 0) tile_tot[blockIdx.x] = tot;
}

__global__ void scan_tiles(int32_t *tile_tot, int nt, int32_t *total) {
  __shared__ int wt[kBlock / 32];
  __shared__ int carry_s;
  if (threadIdx.x == 0) carry_s = 0;
  __syncthreads();
  for (int b = 0; b < nt; b += kBlock) {
    const int i = b + threadIdx.x;
    const int v = i < nt ? tile_tot[i] : 0;
    int tot;
    const int inc = block_inclusive(v, wt, &tot);
    const int carry = carry_s;
    if (i < nt) tile_tot[i] = carry + inc - v;
    __syncthreads();
    if (threadIdx.x == 0) carry_s = carry + tot;
    __syncthreads();
  }
  if (threadIdx.x == 0 && total) *total = carry_s;
}

__global__ void scan_apply(const int32_t *__restrict__ in, int64_t n,
                           const int32_t *__restrict__ tile_off, int32_t *out) {
  __shared__ int wt[kBlock / 32];
  const int64_t base = static_cast<int64_t>(blockIdx.x) * kTile +
                       static_cast<int64_t>(threadIdx.x) * kItems;
  int v[kItems];
  int s = 0;
#pragma unroll
  for (int k = 0; k < kItems; ++k) {
    v[k] = (base + k < n) ? in[base + k] : 0;
    s += v[k];
  }
  int tot;
  const int inc = block_inclusive(s, wt, &tot);
  int run = tile_off[blockIdx.x] + inc - s;
#pragma unroll
  for (int k = 0; k < kItems; ++k) {
    if (base + k < n) out[base + k] = run;
    run += v[k];
  }
}

}  // namespace scan_detail
}  // namespace

// out[i] = sum_{k<i} in[i]; *total_dev (device, may be null) = sum of all.
// `in` and `out` may alias.  tmp must hold ceil(n / 2048) ints.
inline bcmg_status exclusive_scan(const int32_t *in, int32_t *out, int64_t n,
                                  int32_t *total_dev, int32_t *tmp, cudaStream_t s) {
  using namespace scan_detail;
  if (n <= 0) {
    if (total_dev) BCMG_CUDA(cudaMemsetAsync(total_dev, 0, sizeof(int32_t), s));
    return BCMG_OK;
  }
  const int nt = ceil_div(n, kTile);
  launch(tile_sums, nt, kBlock, 0, s, in, n, tmp);
  launch(scan_tiles, 1, kBlock, 0, s, tmp, nt, total_dev);
  launch(scan_apply, nt, kBlock, 0, s, in, n, tmp, out);
  BCMG_LAUNCH_CHECK();
  return BCMG_OK;
}

inline int64_t scan_tmp_size(int64_t n) { return ceil_div(n > 0 ? n : 1, scan_detail::kTile); }

}  // namespace bcmg
