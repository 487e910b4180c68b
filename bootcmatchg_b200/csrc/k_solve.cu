// Solve-phase kernels in FP64: Jacobi / l1-Jacobi sweeps, SpMV, residual,
// restriction, prolongation and the fused FCG reductions.  All reductions
// are deterministic: fixed grids, fixed thread-to-row mapping and a
// fixed-order final reduction replace the reference's FP64 atomics
// (_triple_innerproduct, src/SOLVER/FCG.cu:6-63) and cuBLAS calls
// (src/matrix/vector.cu:345-416).
#include <cfloat>

#include "common.cuh"
#include "kernels.h"

namespace bcmg {
namespace {

constexpr int kThreads = 256;

template <int G>
__device__ __forceinline__ double group_sum(double v) {
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o, G);
  return v;
}

// Row-group dot product of row i with x.
template <int G>
__device__ __forceinline__ double row_dot(const int32_t *__restrict__ row,
                                          const int32_t *__restrict__ col,
                                          const double *__restrict__ val,
                                          const double *__restrict__ x, int32_t i,
                                          int lane) {
  double t = 0.0;
  if (i >= 0) {
    const int32_t e = row[i + 1];
    for (int32_t j = row[i] + lane; j < e; j += G) t = fma(val[j], __ldg(x + col[j]), t);
  }
  return group_sum<G>(t);
}

// One sweep u_out = ((-(A u) + f) ./ d) + u  (_jacobi_it<0,MW>,
// src/AMG/relaxation.cu:176-209).
template <int G>
__global__ void __launch_bounds__(kThreads)
    k_relax(int32_t n, const int32_t *__restrict__ row, const int32_t *__restrict__ col,
            const double *__restrict__ val, const double *__restrict__ d,
            const double *__restrict__ f, const double *__restrict__ u,
            double *__restrict__ u_out) {
  const int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  int32_t i = static_cast<int32_t>(t / G);
  const int lane = threadIdx.x % G;
  if (i >= n) i = -1;
  const double T = row_dot<G>(row, col, val, u, i, lane);
  if (i >= 0 && lane == 0) u_out[i] = ((-T + f[i]) / d[i]) + u[i];
}

// First sweep from u = 0: ((-0 + f) ./ d) + 0 = f ./ d.
__global__ void k_relax_zero(int32_t n, const double *__restrict__ d,
                             const double *__restrict__ f, double *__restrict__ u_out) {
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) u_out[i] = f[i] / d[i];
}

template <int G>
__global__ void __launch_bounds__(kThreads)
    k_spmv(int32_t n, const int32_t *__restrict__ row, const int32_t *__restrict__ col,
           const double *__restrict__ val, double alpha, const double *__restrict__ x,
           double beta, double *__restrict__ y) {
  const int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  int32_t i = static_cast<int32_t>(t / G);
  const int lane = threadIdx.x % G;
  if (i >= n) i = -1;
  const double T = row_dot<G>(row, col, val, x, i, lane);
  if (i >= 0 && lane == 0) y[i] = (beta == 0.0) ? alpha * T : fma(alpha, T, beta * y[i]);
}

template <int G>
__global__ void __launch_bounds__(kThreads)
    k_residual(int32_t n, const int32_t *__restrict__ row,
               const int32_t *__restrict__ col, const double *__restrict__ val,
               const double *__restrict__ f, const double *__restrict__ u,
               double *__restrict__ res) {
  const int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  int32_t i = static_cast<int32_t>(t / G);
  const int lane = threadIdx.x % G;
  if (i >= n) i = -1;
  const double T = row_dot<G>(row, col, val, u, i, lane);
  if (i >= 0 && lane == 0) res[i] = f[i] - T;
}

__global__ void k_restrict(int32_t nc, const int32_t *__restrict__ rptr,
                           const int32_t *__restrict__ ridx, const double *__restrict__ p,
                           const double *__restrict__ x, double *__restrict__ y) {
  const int32_t I = blockIdx.x * blockDim.x + threadIdx.x;
  if (I >= nc) return;
  double s = 0.0;
  for (int32_t k = rptr[I]; k < rptr[I + 1]; ++k) {
    const int32_t i = ridx[k];
    s = fma(p[i], x[i], s);
  }
  y[I] = s;
}

__global__ void k_prolong(int32_t n, const int32_t *__restrict__ agg,
                          const double *__restrict__ p, const double *__restrict__ xc,
                          double *__restrict__ xf) {
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) xf[i] = fma(p[i], xc[agg[i]], xf[i]);
}

__global__ void k_fill(double *x, int64_t n, double v) {
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    x[i] = v;
}

__global__ void k_axpy(int64_t n, double a, const double *__restrict__ x,
                       double *__restrict__ y) {
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    y[i] = fma(a, x[i], y[i]);
}

__global__ void k_scale(int64_t n, double a, double *x) {
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    x[i] = x[i] * a;
}

// Block sum of NV doubles per thread into partials[blockIdx.x * 4 + k].
template <int NV>
__device__ __forceinline__ void block_partials(double (&v)[NV], double *partials) {
  __shared__ double sh[kThreads / 32][4];
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
    for (int w = 0; w < kThreads / 32; ++w) s += sh[w][threadIdx.x];
    partials[blockIdx.x * 4 + threadIdx.x] = s;
  }
}

// Fixed-order sum of the partials of NV quantities by one block.
__device__ __forceinline__ double reduce_partials(const double *partials, int k) {
  __shared__ double sh[kThreads];
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

__global__ void __launch_bounds__(kThreads)
    k_dot_partials(int64_t n, const double *__restrict__ a, const double *__restrict__ b,
                   double *partials) {
  double v[1] = {0.0};
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    v[0] = fma(a[i], b[i], v[0]);
  block_partials<1>(v, partials);
}

__global__ void k_dot_final(const double *partials, double *out) {
  const double s = reduce_partials(partials, 0);
  if (threadIdx.x == 0) *out = s;
}

// w = A v with alpha = r.v, beta = w.v, gamma = q.v accumulated on the fly
// (the SpMV of FCG.cu:508-512 fused with _triple_innerproduct).
template <int G>
__global__ void __launch_bounds__(kThreads)
    k_fcg_spmv_dots(int32_t n, const int32_t *__restrict__ row,
                    const int32_t *__restrict__ col, const double *__restrict__ val,
                    const double *__restrict__ v, double *__restrict__ w,
                    const double *__restrict__ r, const double *__restrict__ q,
                    double *partials) {
  double acc[3] = {0.0, 0.0, 0.0};
  const int lane = threadIdx.x % G;
  const int64_t groups = static_cast<int64_t>(gridDim.x) * blockDim.x / G;
  const int64_t g0 = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) / G;
  const int64_t rounds = (n + groups - 1) / groups;
  for (int64_t rd = 0; rd < rounds; ++rd) {
    const int64_t gi = g0 + rd * groups;
    const int32_t i = gi < n ? static_cast<int32_t>(gi) : -1;
    const double T = row_dot<G>(row, col, val, v, i, lane);
    if (i >= 0 && lane == 0) {
      w[i] = T;
      const double vi = v[i];
      acc[0] = fma(r[i], vi, acc[0]);
      acc[1] = fma(T, vi, acc[1]);
      if (q) acc[2] = fma(q[i], vi, acc[2]);
    }
  }
  block_partials<3>(acc, partials);
}

// FCG scalar recurrences (FCG.cu:475-478 for the first step, :531-534 in
// the loop), kept on the device.
__global__ void k_fcg_scalars(const double *partials, double *scal, int first) {
  const double alpha = reduce_partials(partials, 0);
  const double beta = reduce_partials(partials, 1);
  const double gamma = reduce_partials(partials, 2);
  if (threadIdx.x != 0) return;
  scal[kAlpha] = alpha;
  scal[kBeta] = beta;
  scal[kGamma] = gamma;
  if (first) {
    scal[kDelta] = beta;
    scal[kTheta] = alpha / beta;
    if (!(beta > 0.0)) scal[kIndef] = 1.0;
  } else {
    const double delta = scal[kDelta];
    const double theta = gamma / delta;
    const double nd = beta - (gamma * gamma) / delta;
    scal[kTheta] = theta;
    scal[kDelta] = nd;
    scal[kTheta2] = alpha / nd;
    if (!(nd > 0.0)) scal[kIndef] = 1.0;
  }
}

// first:  x += theta v; r -= theta w                        (FCG.cu:481-484)
// loop:   z = -theta zp + z; x += theta2 z;                 (_double_merged_axpy,
//         az = -theta azp + az; r -= theta2 az               FCG.cu:88-98,536-556)
// plus the partial sums of r.r for ||r||.
__global__ void __launch_bounds__(kThreads)
    k_fcg_update(int64_t n, int first, double *__restrict__ z,
                 const double *__restrict__ zp, double *__restrict__ az,
                 const double *__restrict__ azp, double *__restrict__ x,
                 double *__restrict__ r, const double *__restrict__ scal,
                 double *partials) {
  double acc[1] = {0.0};
  const double theta = scal[kTheta];
  const double theta2 = first ? theta : scal[kTheta2];
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    double zi = z[i], ai = az[i];
    if (!first) {
      zi = fma(-theta, zp[i], zi);
      ai = fma(-theta, azp[i], ai);
      z[i] = zi;
      az[i] = ai;
    }
    x[i] = fma(theta2, zi, x[i]);
    const double ri = fma(-theta2, ai, r[i]);
    r[i] = ri;
    acc[0] = fma(ri, ri, acc[0]);
  }
  block_partials<1>(acc, partials);
}

__global__ void k_norm_final(const double *partials, double *scal) {
  const double s = reduce_partials(partials, 0);
  if (threadIdx.x == 0) scal[kNorm] = sqrt(s);
}

template <template <int> class K>
struct Dispatch;

inline int grid_for(int64_t work) {
  const int64_t b = (work + kThreads - 1) / kThreads;
  return static_cast<int>(b < 1 ? 1 : b);
}

}  // namespace

bcmg_status relax(const CsrView &A, const double *d, const double *f, double *u,
                  double *u_tmp, int k, bool zero_start, double **result, cudaStream_t s) {
  *result = u;
  const int32_t n = A.n;
  if (n <= 0) return BCMG_OK;
  if (k <= 0) {
    if (zero_start) BCMG_TRY(fill(u, n, 0.0, s));
    return BCMG_OK;
  }
  const int G = group_for(A.nnz, n);
  const int blocks = grid_for(static_cast<int64_t>(n) * G);
  auto sweep = [&](const double *src, double *dst) {
    switch (G) {
      case 4: k_relax<4><<<blocks, kThreads, 0, s>>>(n, A.row, A.col, A.val, d, f, src, dst); break;
      case 8: k_relax<8><<<blocks, kThreads, 0, s>>>(n, A.row, A.col, A.val, d, f, src, dst); break;
      case 16: k_relax<16><<<blocks, kThreads, 0, s>>>(n, A.row, A.col, A.val, d, f, src, dst); break;
      default: k_relax<32><<<blocks, kThreads, 0, s>>>(n, A.row, A.col, A.val, d, f, src, dst); break;
    }
  };
  // Arrange the ping-pong so the final iterate lands in u.
  double *cur;
  int left = k;
  if (zero_start) {
    cur = (k % 2 == 1) ? u : u_tmp;
    k_relax_zero<<<ceil_div(n, kThreads), kThreads, 0, s>>>(n, d, f, cur);
    --left;
  } else if (k % 2 == 1) {
    BCMG_CUDA(cudaMemcpyAsync(u_tmp, u, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
    cur = u_tmp;
  } else {
    cur = u;
  }
  for (; left > 0; --left) {
    double *dst = (cur == u) ? u_tmp : u;
    sweep(cur, dst);
    cur = dst;
  }
  BCMG_LAUNCH_CHECK();
  return BCMG_OK;
}

bcmg_status spmv(const CsrView &A, double alpha, const double *x, double beta, double *y,
                 cudaStream_t s) {
  const int32_t n = A.n;
  if (n <= 0) return BCMG_OK;
  const int G = group_for(A.nnz, n);
  const int blocks = grid_for(static_cast<int64_t>(n) * G);
  switch (G) {
    case 4: k_spmv<4><<<blocks, kThreads, 0, s>>>(n, A.row, A.col, A.val, alpha, x, beta, y); break;
    case 8: k_spmv<8><<<blocks, kThreads, 0, s>>>(n, A.row, A.col, A.val, alpha, x, beta, y); break;
    case 16: k_spmv<16><<<blocks, kThreads, 0, s>>>(n, A.row, A.col, A.val, alpha, x, beta, y); break;
    default: k_spmv<32><<<blocks, kThreads, 0, s>>>(n, A.row, A.col, A.val, alpha, x, beta, y); break;
  }
  BCMG_LAUNCH_CHECK();
  return BCMG_OK;
}

bcmg_status residual(const CsrView &A, const double *f, const double *u, double *res,
                     cudaStream_t s) {
  const int32_t n = A.n;
  if (n <= 0) return BCMG_OK;
  const int G = group_for(A.nnz, n);
  const int blocks = grid_for(static_cast<int64_t>(n) * G);
  switch (G) {
    case 4: k_residual<4><<<blocks, kThreads, 0, s>>>(n, A.row, A.col, A.val, f, u, res); break;
    case 8: k_residual<8><<<blocks, kThreads, 0, s>>>(n, A.row, A.col, A.val, f, u, res); break;
    case 16: k_residual<16><<<blocks, kThreads, 0, s>>>(n, A.row, A.col, A.val, f, u, res); break;
    default: k_residual<32><<<blocks, kThreads, 0, s>>>(n, A.row, A.col, A.val, f, u, res); break;
  }
  BCMG_LAUNCH_CHECK();
  return BCMG_OK;
}

bcmg_status restrict_vec(int32_t nc, const int32_t *rptr, const int32_t *ridx,
                         const double *p, const double *x, double *y, cudaStream_t s) {
  if (nc <= 0) return BCMG_OK;
  k_restrict<<<ceil_div(nc, kThreads), kThreads, 0, s>>>(nc, rptr, ridx, p, x, y);
  BCMG_LAUNCH_CHECK();
  return BCMG_OK;
}

bcmg_status prolong_add(int32_t n, const int32_t *agg, const double *p, const double *xc,
                        double *xf, cudaStream_t s) {
  if (n <= 0) return BCMG_OK;
  k_prolong<<<ceil_div(n, kThreads), kThreads, 0, s>>>(n, agg, p, xc, xf);
  BCMG_LAUNCH_CHECK();
  return BCMG_OK;
}

bcmg_status fill(double *x, int64_t n, double v, cudaStream_t s) {
  if (n <= 0) return BCMG_OK;
  const int blocks = static_cast<int>(std::min<int64_t>(grid_for(n), 8 * kNumSM));
  k_fill<<<blocks, kThreads, 0, s>>>(x, n, v);
  BCMG_LAUNCH_CHECK();
  return BCMG_OK;
}

bcmg_status copy(double *dst, const double *src, int64_t n, cudaStream_t s) {
  if (n <= 0 || dst == src) return BCMG_OK;
  BCMG_CUDA(cudaMemcpyAsync(dst, src, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
  return BCMG_OK;
}

bcmg_status axpy(int64_t n, double alpha, const double *x, double *y, cudaStream_t s) {
  if (n <= 0) return BCMG_OK;
  const int blocks = static_cast<int>(std::min<int64_t>(grid_for(n), 8 * kNumSM));
  k_axpy<<<blocks, kThreads, 0, s>>>(n, alpha, x, y);
  BCMG_LAUNCH_CHECK();
  return BCMG_OK;
}

bcmg_status scale(int64_t n, double alpha, double *x, cudaStream_t s) {
  if (n <= 0) return BCMG_OK;
  const int blocks = static_cast<int>(std::min<int64_t>(grid_for(n), 8 * kNumSM));
  k_scale<<<blocks, kThreads, 0, s>>>(n, alpha, x);
  BCMG_LAUNCH_CHECK();
  return BCMG_OK;
}

bcmg_status dot_dev(int64_t n, const double *a, const double *b, double *out,
                    double *partials, cudaStream_t s) {
  k_dot_partials<<<kRedBlocks, kThreads, 0, s>>>(n, a, b, partials);
  k_dot_final<<<1, kThreads, 0, s>>>(partials, out);
  BCMG_LAUNCH_CHECK();
  return BCMG_OK;
}

bcmg_status fcg_spmv_dots(const CsrView &A, const double *v, double *w, const double *r,
                          const double *q, double *partials, double *scal,
                          cudaStream_t s) {
  (void)scal;
  const int32_t n = A.n;
  const int G = group_for(A.nnz, n);
  switch (G) {
    case 4: k_fcg_spmv_dots<4><<<kRedBlocks, kThreads, 0, s>>>(n, A.row, A.col, A.val, v, w, r, q, partials); break;
    case 8: k_fcg_spmv_dots<8><<<kRedBlocks, kThreads, 0, s>>>(n, A.row, A.col, A.val, v, w, r, q, partials); break;
    case 16: k_fcg_spmv_dots<16><<<kRedBlocks, kThreads, 0, s>>>(n, A.row, A.col, A.val, v, w, r, q, partials); break;
    default: k_fcg_spmv_dots<32><<<kRedBlocks, kThreads, 0, s>>>(n, A.row, A.col, A.val, v, w, r, q, partials); break;
  }
  BCMG_LAUNCH_CHECK();
  return BCMG_OK;
}

bcmg_status fcg_scalars(double *partials, double *scal, bool first, cudaStream_t s) {
  k_fcg_scalars<<<1, kThreads, 0, s>>>(partials, scal, first ? 1 : 0);
  BCMG_LAUNCH_CHECK();
  return BCMG_OK;
}

bcmg_status fcg_update(int64_t n, bool first, double *z, const double *zp, double *az,
                       const double *azp, double *x, double *r, double *partials,
                       double *scal, cudaStream_t s) {
  k_fcg_update<<<kRedBlocks, kThreads, 0, s>>>(n, first ? 1 : 0, z, zp, az, azp, x, r,
                                               scal, partials);
  k_norm_final<<<1, kThreads, 0, s>>>(partials, scal);
  BCMG_LAUNCH_CHECK();
  return BCMG_OK;
}

}  // namespace bcmg
