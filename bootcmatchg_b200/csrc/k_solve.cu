// FCG kernels in FP64: SpMV, dot products and the fused FCG reductions.  All reductions
// are deterministic: fixed grids, fixed thread-to-row mapping and a
// fixed-order final reduction replace the reference's FP64 atomics
// (_triple_innerproduct, src/SOLVER/FCG.cu:6-63) and cuBLAS calls
// (src/matrix/vector.cu:345-416).
#include <cfloat>

#include "common.cuh"
#include "kernels.h"
#include "reduce.cuh"

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

__global__ void __launch_bounds__(kThreads)
    k_dot_partials(int64_t n, const double *__restrict__ a, const double *__restrict__ b,
                   double *partials) {
  pdl_wait();
  pdl_trigger();
  double v[1] = {0.0};
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    v[0] = fma(a[i], b[i], v[0]);
  block_partials<1>(v, partials);
}

__global__ void k_dot_final(const double *partials, double *out) {
  pdl_wait();
  pdl_trigger();
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
  pdl_wait();
  pdl_trigger();
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
  pdl_wait();
  pdl_trigger();
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
    if (nd > 0.0) {
      scal[kTheta] = theta;
      scal[kDelta] = nd;
      scal[kTheta2] = alpha / nd;
    } else if (alpha == 0.0 && gamma == 0.0) {
      // r = 0 exactly (so z = B r = 0): the previous step was exact.  The
      // reference's do-while still runs this iteration and divides 0 by 0
      // (FCG.cu:531-534); here the update becomes a no-op instead.
      scal[kTheta] = 0.0;
      scal[kTheta2] = 0.0;
    } else {
      scal[kTheta] = theta;
      scal[kDelta] = nd;
      scal[kTheta2] = alpha / nd;
      scal[kIndef] = 1.0;
    }
  }
}

// first:  x += theta z; r -= theta az; zp = z; azp = az     (FCG.cu:481-495)
// loop:   zp = -theta zp + z; x += theta2 zp;               (_double_merged_axpy,
//         azp = -theta azp + az; r -= theta2 azp             FCG.cu:88-98,536-556)
// plus the partial sums of r.r for ||r||.  The new direction overwrites the
// previous one in (zp, azp), so every iteration uses the same buffers (the
// reference alternates (v,w) and (d,q) instead, FCG.cu:499-556).
__global__ void __launch_bounds__(kThreads)
    k_fcg_update(int64_t n, int first, const double *__restrict__ z,
                 double *__restrict__ zp, const double *__restrict__ az,
                 double *__restrict__ azp, double *__restrict__ x,
                 double *__restrict__ r, const double *__restrict__ scal,
                 double *partials) {
  pdl_wait();
  pdl_trigger();
  double acc[1] = {0.0};
  const double theta = scal[kTheta];
  const double theta2 = first ? theta : scal[kTheta2];
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    double zi = z[i], ai = az[i];
    if (!first) {
      zi = fma(-theta, zp[i], zi);
      ai = fma(-theta, azp[i], ai);
    }
    zp[i] = zi;
    azp[i] = ai;
    x[i] = fma(theta2, zi, x[i]);
    const double ri = fma(-theta2, ai, r[i]);
    r[i] = ri;
    acc[0] = fma(ri, ri, acc[0]);
  }
  block_partials<1>(acc, partials);
}

__global__ void k_norm_final(const double *partials, double *scal) {
  pdl_wait();
  pdl_trigger();
  const double s = reduce_partials(partials, 0);
  if (threadIdx.x == 0) scal[kNorm] = sqrt(s);
}

// End of one FCG iteration: count it and decide whether the do-while of
// FCG.cu:497-565 continues (||r|| > rtol delta0 and iter < itnlim and no
// breakdown).  Inside a graph the decision drives the WHILE node.
__global__ void k_fcg_continue(double *scal, cudaGraphConditionalHandle cond, int use_cond) {
  pdl_wait();
  pdl_trigger();
  const double iter = scal[kIter] + 1.0;
  scal[kIter] = iter;
  const bool go = scal[kNorm] > scal[kTarget] && iter < scal[kItnlim] && scal[kIndef] == 0.0;
  if (use_cond) cudaGraphSetConditional(cond, go ? 1u : 0u);
}


// Residual replacement (mixed precision): after iteration i the recursive
// residual is replaced by the true one r = b - A x in FP64 when i is a
// multiple of `every` or when the recursive norm has reached the target, so
// convergence is always decided on the true residual.
__global__ void k_replace_flag(double *scal, int every) {
  pdl_wait();
  pdl_trigger();
  const int i = static_cast<int>(scal[kIter]) + 1;
  const bool due = (every > 0 && i % every == 0) || scal[kNorm] <= scal[kTarget];
  scal[kReplace] = due ? 1.0 : 0.0;
}

template <int G>
__global__ void __launch_bounds__(kThreads)
    k_true_residual(int32_t n, const int32_t *__restrict__ row,
                    const int32_t *__restrict__ col, const double *__restrict__ val,
                    const double *__restrict__ b, const double *__restrict__ x,
                    double *__restrict__ r, const double *__restrict__ scal,
                    double *partials) {
  if (scal[kReplace] == 0.0) return;
  double acc[1] = {0.0};
  const int lane = threadIdx.x % G;
  const int64_t groups = static_cast<int64_t>(gridDim.x) * blockDim.x / G;
  const int64_t g0 = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) / G;
  const int64_t rounds = (n + groups - 1) / groups;
  for (int64_t rd = 0; rd < rounds; ++rd) {
    const int64_t gi = g0 + rd * groups;
    const int32_t i = gi < n ? static_cast<int32_t>(gi) : -1;
    const double T = row_dot<G>(row, col, val, x, i, lane);
    if (i >= 0 && lane == 0) {
      const double ri = b[i] - T;
      r[i] = ri;
      acc[0] = fma(ri, ri, acc[0]);
    }
  }
  block_partials<1>(acc, partials);
}

__global__ void k_norm_final_if(const double *partials, double *scal) {
  pdl_wait();
  pdl_trigger();
  if (scal[kReplace] == 0.0) return;
  const double s = reduce_partials(partials, 0);
  if (threadIdx.x == 0) scal[kNorm] = sqrt(s);
}

inline int grid_for(int64_t work) {
  const int64_t b = (work + kThreads - 1) / kThreads;
  return static_cast<int>(b < 1 ? 1 : b);
}


// Structural check of a device CSR matrix, one thread per row: row bounds,
// columns in range and strictly increasing, finite values, a diagonal entry.
// The smallest offending row wins: err = (row << 8) | code.
__global__ void k_csr_validate(int32_t n, int32_t m, int32_t nnz,
                               const int32_t *__restrict__ row,
                               const int32_t *__restrict__ col,
                               const double *__restrict__ val, int need_diag,
                               unsigned long long *err) {
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int32_t b = row[i], e = row[i + 1];
  int code = 0;
  if (b < 0 || e < b || e > nnz) {
    code = kCsrBadRow;
  } else {
    bool diag = false;
    int32_t prev = -1;
    for (int32_t j = b; j < e && !code; ++j) {
      const int32_t c = col[j];
      if (c < 0 || c >= m) code = kCsrBadColumn;
      else if (c <= prev) code = kCsrUnsorted;
      else if (!isfinite(val[j])) code = kCsrNonFinite;
      diag = diag || c == i;
      prev = c;
    }
    if (!code && need_diag && !diag) code = kCsrNoDiagonal;
  }
  if (code) atomicMin(err, (static_cast<unsigned long long>(i) << 8) | code);
}

}  // namespace

bcmg_status spmv(const CsrView &A, double alpha, const double *x, double beta, double *y,
                 cudaStream_t s) {
  const int32_t n = A.n;
  if (n <= 0) return BCMG_OK;
  const int G = group_for(A.nnz, n);
  const int blocks = grid_for(static_cast<int64_t>(n) * G);
  switch (G) {
    case 4: launch(k_spmv<4>, blocks, kThreads, 0, s, n, A.row, A.col, A.val, alpha, x, beta, y); break;
    case 8: launch(k_spmv<8>, blocks, kThreads, 0, s, n, A.row, A.col, A.val, alpha, x, beta, y); break;
    case 16: launch(k_spmv<16>, blocks, kThreads, 0, s, n, A.row, A.col, A.val, alpha, x, beta, y); break;
    default: launch(k_spmv<32>, blocks, kThreads, 0, s, n, A.row, A.col, A.val, alpha, x, beta, y); break;
  }
  BCMG_LAUNCH_CHECK();
  return BCMG_OK;
}

bcmg_status dot_dev(int64_t n, const double *a, const double *b, double *out,
                    double *partials, cudaStream_t s) {
  launch_pdl(k_dot_partials, kRedBlocks, kThreads, 0, s, n, a, b, partials);
  launch_pdl(k_dot_final, 1, kThreads, 0, s, partials, out);
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
    case 4: launch_pdl(k_fcg_spmv_dots<4>, kRedBlocks, kThreads, 0, s, n, A.row, A.col, A.val, v, w, r, q, partials); break;
    case 8: launch_pdl(k_fcg_spmv_dots<8>, kRedBlocks, kThreads, 0, s, n, A.row, A.col, A.val, v, w, r, q, partials); break;
    case 16: launch_pdl(k_fcg_spmv_dots<16>, kRedBlocks, kThreads, 0, s, n, A.row, A.col, A.val, v, w, r, q, partials); break;
    default: launch_pdl(k_fcg_spmv_dots<32>, kRedBlocks, kThreads, 0, s, n, A.row, A.col, A.val, v, w, r, q, partials); break;
  }
  BCMG_LAUNCH_CHECK();
  return BCMG_OK;
}

bcmg_status fcg_scalars(double *partials, double *scal, bool first, cudaStream_t s) {
  launch_pdl(k_fcg_scalars, 1, kThreads, 0, s, partials, scal, first ? 1 : 0);
  BCMG_LAUNCH_CHECK();
  return BCMG_OK;
}

bcmg_status fcg_continue(double *scal, cudaGraphConditionalHandle cond, bool use_cond,
                         cudaStream_t s) {
  launch_pdl(k_fcg_continue, 1, 1, 0, s, scal, cond, use_cond ? 1 : 0);
  BCMG_LAUNCH_CHECK();
  return BCMG_OK;
}

bcmg_status fcg_update(int64_t n, bool first, const double *z, double *zp,
                       const double *az, double *azp, double *x, double *r,
                       double *partials, double *scal, cudaStream_t s) {
  launch_pdl(k_fcg_update, kRedBlocks, kThreads, 0, s, n, first ? 1 : 0, z, zp, az, azp, x, r,
                                               scal, partials);
  launch_pdl(k_norm_final, 1, kThreads, 0, s, partials, scal);
  BCMG_LAUNCH_CHECK();
  return BCMG_OK;
}

bcmg_status fcg_replace(const CsrView &A, const SlicedView *S, const double *b, const double *x,
                        double *r, double *partials, double *scal, int every, cudaStream_t s) {
  launch_pdl(k_replace_flag, 1, 1, 0, s, scal, every);
  if (S && S->nslices) {
    BCMG_TRY(sliced_replace(*S, b, x, r, partials, scal, s));
    launch_pdl(k_norm_final_if, 1, kThreads, 0, s, partials, scal);
    BCMG_LAUNCH_CHECK();
    return BCMG_OK;
  }
  const int G = group_for(A.nnz, A.n);
  switch (G) {
    case 4: launch(k_true_residual<4>, kRedBlocks, kThreads, 0, s, A.n, A.row, A.col, A.val, b, x, r, scal, partials); break;
    case 8: launch(k_true_residual<8>, kRedBlocks, kThreads, 0, s, A.n, A.row, A.col, A.val, b, x, r, scal, partials); break;
    case 16: launch(k_true_residual<16>, kRedBlocks, kThreads, 0, s, A.n, A.row, A.col, A.val, b, x, r, scal, partials); break;
    default: launch(k_true_residual<32>, kRedBlocks, kThreads, 0, s, A.n, A.row, A.col, A.val, b, x, r, scal, partials); break;
  }
  launch_pdl(k_norm_final_if, 1, kThreads, 0, s, partials, scal);
  BCMG_LAUNCH_CHECK();
  return BCMG_OK;
}

namespace {
bcmg_status csr_check(const CsrView &A, int32_t m, bool need_diag, cudaStream_t s) {
  if (A.n <= 0 || m <= 0) return set_error(BCMG_ERR_INVALID_MATRIX, "matrix must have n > 0");
  DevBuf<unsigned long long> err;
  BCMG_TRY(err.alloc(1, s));
  BCMG_CUDA(cudaMemsetAsync(err.get(), 0xff, sizeof(unsigned long long), s));
  launch(k_csr_validate, ceil_div(A.n, kThreads), kThreads, 0, s, A.n, m, A.nnz, A.row, A.col,
         A.val, need_diag ? 1 : 0, err.get());
  BCMG_LAUNCH_CHECK();
  unsigned long long h = 0;
  BCMG_CUDA(cudaMemcpyAsync(&h, err.get(), sizeof(h), cudaMemcpyDeviceToHost, s));
  BCMG_CUDA(cudaStreamSynchronize(s));
  if (h == ~0ull) return BCMG_OK;
  const long long r = static_cast<long long>(h >> 8);
  switch (static_cast<int>(h & 0xff)) {
    case kCsrBadRow:
      return set_error(BCMG_ERR_INVALID_MATRIX, "row %lld has a bad row pointer range", r);
    case kCsrBadColumn:
      return set_error(BCMG_ERR_INVALID_MATRIX, "row %lld: column out of range", r);
    case kCsrUnsorted:
      return set_error(BCMG_ERR_INVALID_MATRIX, "row %lld: columns not strictly increasing",
                       r);
    case kCsrNonFinite:
      return set_error(BCMG_ERR_INVALID_MATRIX, "row %lld: non-finite value", r);
    default:
      return set_error(BCMG_ERR_INVALID_MATRIX,
                       "row %lld has no diagonal entry (the AH builder needs one)", r);
  }
}
}  // namespace

bcmg_status csr_validate(const CsrView &A, cudaStream_t s) {
  return csr_check(A, A.n, true, s);
}

bcmg_status csr_validate_rect(const CsrView &A, int32_t m, cudaStream_t s) {
  return csr_check(A, m, false, s);
}

}  // namespace bcmg
