// Cycle kernels, templated on the value type of the level matrix (FP64, FP32,
// BF16, FP16) and on the vector type (FP64 for the FP64 path, FP32 for the
// mixed-precision cycle; low-precision values are widened and accumulated in
// FP32).  Relaxation follows _jacobi_it<0,MW> (src/AMG/relaxation.cu:176-209):
// u' = ((-(A u) + f) ./ d) + u; residual / restriction / prolongation follow
// GAMG_cycle (src/SOLVER/GAMG_cycle.cu:57-119).
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "common.cuh"
#include "kernels.h"
#include "reduce.cuh"

namespace bcmg {
namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ double widen(double v) { return v; }
__device__ __forceinline__ float widen(float v) { return v; }
__device__ __forceinline__ float widen(__nv_bfloat16 v) { return __bfloat162float(v); }
__device__ __forceinline__ float widen(__half v) { return __half2float(v); }

template <int G, typename XT>
__device__ __forceinline__ XT group_sum(XT v) {
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o, G);
  return v;
}

template <int G, typename VT, typename XT>
__device__ __forceinline__ XT row_dot(const int32_t *__restrict__ row,
                                      const int32_t *__restrict__ col,
                                      const VT *__restrict__ val, const XT *__restrict__ x,
                                      int32_t i, int lane) {
  XT t = XT(0);
  if (i >= 0) {
    const int32_t e = row[i + 1];
    for (int32_t j = row[i] + lane; j < e; j += G)
      t = fma(static_cast<XT>(widen(val[j])), __ldg(x + col[j]), t);
  }
  return group_sum<G, XT>(t);
}

template <int G, typename VT, typename XT>
__global__ void __launch_bounds__(kThreads)
    k_relax_t(int32_t n, const int32_t *__restrict__ row, const int32_t *__restrict__ col,
              const VT *__restrict__ val, const XT *__restrict__ d,
              const XT *__restrict__ f, const XT *__restrict__ u, XT *__restrict__ u_out) {
  pdl_wait();
  pdl_trigger();
  const int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  int32_t i = static_cast<int32_t>(t / G);
  const int lane = threadIdx.x % G;
  if (i >= n) i = -1;
  const XT T = row_dot<G, VT, XT>(row, col, val, u, i, lane);
  if (i >= 0 && lane == 0) u_out[i] = ((-T + f[i]) / d[i]) + u[i];
}

// First sweep from u = 0: ((-0 + f) ./ d) + 0 = f ./ d.
template <typename XT>
__global__ void k_relax_zero_t(int32_t n, const XT *__restrict__ d, const XT *__restrict__ f,
                               XT *__restrict__ u_out) {
  pdl_wait();
  pdl_trigger();
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) u_out[i] = f[i] / d[i];
}

template <int G, typename VT, typename XT>
__global__ void __launch_bounds__(kThreads)
    k_residual_t(int32_t n, const int32_t *__restrict__ row, const int32_t *__restrict__ col,
                 const VT *__restrict__ val, const XT *__restrict__ f,
                 const XT *__restrict__ u, XT *__restrict__ res) {
  pdl_wait();
  pdl_trigger();
  const int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  int32_t i = static_cast<int32_t>(t / G);
  const int lane = threadIdx.x % G;
  if (i >= n) i = -1;
  const XT T = row_dot<G, VT, XT>(row, col, val, u, i, lane);
  if (i >= 0 && lane == 0) res[i] = f[i] - T;
}

template <typename XT>
__global__ void k_restrict_t(int32_t nc, const int32_t *__restrict__ rptr,
                             const int32_t *__restrict__ ridx, const XT *__restrict__ p,
                             const XT *__restrict__ x, XT *__restrict__ y) {
  pdl_wait();
  pdl_trigger();
  const int32_t I = blockIdx.x * blockDim.x + threadIdx.x;
  if (I >= nc) return;
  XT s = XT(0);
  for (int32_t k = rptr[I]; k < rptr[I + 1]; ++k) {
    const int32_t i = ridx[k];
    s = fma(p[i], x[i], s);
  }
  y[I] = s;
}

// k_restrict_t fused with the coarse level's first sweep from zero.
template <typename XT>
__global__ void k_restrict_first_t(int32_t nc, const int32_t *__restrict__ rptr,
                                   const int32_t *__restrict__ ridx, const XT *__restrict__ p,
                                   const XT *__restrict__ x, XT *__restrict__ y,
                                   const XT *__restrict__ dc, XT *__restrict__ u1) {
  pdl_wait();
  pdl_trigger();
  const int32_t I = blockIdx.x * blockDim.x + threadIdx.x;
  if (I >= nc) return;
  XT s = XT(0);
  for (int32_t k = rptr[I]; k < rptr[I + 1]; ++k) {
    const int32_t i = ridx[k];
    s = fma(p[i], x[i], s);
  }
  y[I] = s;
  u1[I] = s / dc[I];
}

// FP64 -> FP32 conversion fused with the first sweep from zero.
__global__ void k_convert_first(int64_t n, const double *__restrict__ in,
                                const float *__restrict__ d, float *__restrict__ out,
                                float *__restrict__ u1) {
  pdl_wait();
  pdl_trigger();
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const float v = static_cast<float>(in[i]);
    out[i] = v;
    u1[i] = v / d[i];
  }
}

template <typename XT>
__global__ void k_prolong_t(int32_t n, const int32_t *__restrict__ agg,
                            const XT *__restrict__ p, const XT *__restrict__ xc,
                            XT *__restrict__ xf) {
  pdl_wait();
  pdl_trigger();
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) xf[i] = fma(p[i], xc[agg[i]], xf[i]);
}

template <typename XT>
__global__ void k_fill_t(XT *x, int64_t n, XT v) {
  pdl_wait();
  pdl_trigger();
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    x[i] = v;
}

template <typename XT>
__global__ void k_axpy_t(int64_t n, XT a, const XT *__restrict__ x, XT *__restrict__ y) {
  pdl_wait();
  pdl_trigger();
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    y[i] = fma(a, x[i], y[i]);
}

// dst = src, a kernel in the programmatic-launch chain (see pdl_fence).
template <typename XT>
__global__ void k_copy_t(int64_t n, const XT *__restrict__ src, XT *__restrict__ dst) {
  pdl_wait();
  pdl_trigger();
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    dst[i] = src[i];
}

template <typename XT>
__global__ void k_scale_t(int64_t n, XT a, XT *x) {
  pdl_wait();
  pdl_trigger();
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    x[i] = x[i] * a;
}

template <typename From, typename To>
__global__ void k_convert(int64_t n, const From *__restrict__ in, To *__restrict__ out) {
  pdl_wait();
  pdl_trigger();
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    out[i] = static_cast<To>(in[i]);
}

__global__ void k_to_bf16(int64_t n, const double *__restrict__ in, __nv_bfloat16 *out) {
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    out[i] = __double2bfloat16(in[i]);
}

__global__ void k_to_f16(int64_t n, const double *__restrict__ in, __half *out) {
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    out[i] = __double2half(in[i]);
}

template <int G, typename VT, typename XT>
__global__ void __launch_bounds__(kThreads)
    k_spmv_t(int32_t n, const int32_t *__restrict__ row, const int32_t *__restrict__ col,
             const VT *__restrict__ val, const XT *__restrict__ x, XT *__restrict__ y) {
  pdl_wait();
  pdl_trigger();
  const int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  int32_t i = static_cast<int32_t>(t / G);
  const int lane = threadIdx.x % G;
  if (i >= n) i = -1;
  const XT T = row_dot<G, VT, XT>(row, col, val, x, i, lane);
  if (i >= 0 && lane == 0) y[i] = T;
}

// a . b with FP64 accumulation, fixed grid and order (deterministic).
template <typename XT>
__global__ void __launch_bounds__(kRedThreads)
    k_dot_t(int64_t n, const XT *__restrict__ a, const XT *__restrict__ b, double *partials) {
  pdl_wait();
  pdl_trigger();
  double v[1] = {0.0};
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    v[0] = fma(static_cast<double>(a[i]), static_cast<double>(b[i]), v[0]);
  block_partials<1>(v, partials);
}

__global__ void k_dot_t_final(const double *partials, double *out) {
  pdl_wait();
  pdl_trigger();
  const double s = reduce_partials(partials, 0);
  if (threadIdx.x == 0) *out = s;
}

inline int grid_for(int64_t work) {
  const int64_t b = (work + kThreads - 1) / kThreads;
  return static_cast<int>(b < 1 ? 1 : b);
}

inline int stream_grid(int64_t n) {
  return static_cast<int>(std::min<int64_t>(grid_for(n), 8 * kNumSM));
}

template <typename VT, typename XT>
void launch_relax(int G, int blocks, cudaStream_t s, const MatView &A, const XT *d,
                  const XT *f, const XT *src, XT *dst) {
  const VT *val = static_cast<const VT *>(A.val);
  switch (G) {
    case 4: launch_pdl(k_relax_t<4, VT, XT>, blocks, kThreads, 0, s, A.n, A.row, A.col, val, d, f, src, dst); break;
    case 8: launch_pdl(k_relax_t<8, VT, XT>, blocks, kThreads, 0, s, A.n, A.row, A.col, val, d, f, src, dst); break;
    case 16: launch_pdl(k_relax_t<16, VT, XT>, blocks, kThreads, 0, s, A.n, A.row, A.col, val, d, f, src, dst); break;
    default: launch_pdl(k_relax_t<32, VT, XT>, blocks, kThreads, 0, s, A.n, A.row, A.col, val, d, f, src, dst); break;
  }
}

template <typename VT, typename XT>
void launch_residual(int G, int blocks, cudaStream_t s, const MatView &A, const XT *f,
                     const XT *u, XT *res) {
  const VT *val = static_cast<const VT *>(A.val);
  switch (G) {
    case 4: launch_pdl(k_residual_t<4, VT, XT>, blocks, kThreads, 0, s, A.n, A.row, A.col, val, f, u, res); break;
    case 8: launch_pdl(k_residual_t<8, VT, XT>, blocks, kThreads, 0, s, A.n, A.row, A.col, val, f, u, res); break;
    case 16: launch_pdl(k_residual_t<16, VT, XT>, blocks, kThreads, 0, s, A.n, A.row, A.col, val, f, u, res); break;
    default: launch_pdl(k_residual_t<32, VT, XT>, blocks, kThreads, 0, s, A.n, A.row, A.col, val, f, u, res); break;
  }
}

// Value-type dispatch: FP64 vectors only with FP64 values; FP32 vectors with
// FP32 / BF16 / FP16 values.
template <typename XT>
bcmg_status check_types(const MatView &A) {
  if (A.has_sl) return BCMG_OK;  // the sliced launchers check their own types
  const bool ok = std::is_same<XT, double>::value ? A.vtype == kValF64 : A.vtype != kValF64;
  if (!ok) return set_error(BCMG_ERR_INTERNAL, "value/vector type mismatch (%d)", A.vtype);
  return BCMG_OK;
}

template <typename XT>
void relax_sweep(int G, int blocks, cudaStream_t s, const MatView &A, const XT *d, const XT *f,
                 const XT *src, XT *dst);

template <>
void relax_sweep<double>(int G, int blocks, cudaStream_t s, const MatView &A, const double *d,
                         const double *f, const double *src, double *dst) {
  launch_relax<double, double>(G, blocks, s, A, d, f, src, dst);
}

template <>
void relax_sweep<float>(int G, int blocks, cudaStream_t s, const MatView &A, const float *d,
                        const float *f, const float *src, float *dst) {
  if (A.vtype == kValF32) launch_relax<float, float>(G, blocks, s, A, d, f, src, dst);
  else if (A.vtype == kValBF16) launch_relax<__nv_bfloat16, float>(G, blocks, s, A, d, f, src, dst);
  else launch_relax<__half, float>(G, blocks, s, A, d, f, src, dst);
}

template <typename XT>
void residual_pass(int G, int blocks, cudaStream_t s, const MatView &A, const XT *f,
                   const XT *u, XT *res);

template <>
void residual_pass<double>(int G, int blocks, cudaStream_t s, const MatView &A,
                           const double *f, const double *u, double *res) {
  launch_residual<double, double>(G, blocks, s, A, f, u, res);
}

template <>
void residual_pass<float>(int G, int blocks, cudaStream_t s, const MatView &A, const float *f,
                          const float *u, float *res) {
  if (A.vtype == kValF32) launch_residual<float, float>(G, blocks, s, A, f, u, res);
  else if (A.vtype == kValBF16) launch_residual<__nv_bfloat16, float>(G, blocks, s, A, f, u, res);
  else launch_residual<__half, float>(G, blocks, s, A, f, u, res);
}

}  // namespace

template <typename XT>
bcmg_status relax_t(const MatView &A, const XT *d, const XT *f, XT *u, XT *u_tmp, int k,
                    int start, cudaStream_t s, double *widen_out) {
  const int32_t n = A.n;
  if (n <= 0) return BCMG_OK;
  BCMG_TRY(check_types<XT>(A));
  if (start == kStartFirstDone && !first_sweep_fusable(A, k))
    return set_error(BCMG_ERR_INTERNAL, "first sweep fused where it cannot be");
  if (widen_out && (!std::is_same<XT, float>::value || !widen_fusable(A, k)))
    return set_error(BCMG_ERR_INTERNAL, "widened sweep where it cannot be");
  // A small level held by one thread-block cluster: all sweeps in one launch.
  if (A.has_sl && A.sl.cl_size > 0 && k >= 2)
    return sliced_cluster<XT>(A.sl, d, f, u, k, start != kStartLive, nullptr, s);
  if (k <= 0) {
    if (start != kStartLive) BCMG_TRY(fill_t<XT>(u, n, XT(0), s));
    return BCMG_OK;
  }
  const int G = group_for(A.nnz, n);
  const int blocks = grid_for(static_cast<int64_t>(n) * G);
  // Arrange the ping-pong so the final iterate lands in u.
  XT *cur;
  int left = k;
  if (start != kStartLive) {
    cur = first_sweep_dst(u, u_tmp, k);
    if (start == kStartZero)
      launch_pdl(k_relax_zero_t<XT>, ceil_div(n, kThreads), kThreads, 0, s, n, d, f, cur);
    --left;
  } else if (k % 2 == 1) {
    BCMG_TRY(copy_t<XT>(u_tmp, u, n, s));  // a kernel: ordered before the first sweep
    cur = u_tmp;
  } else {
    cur = u;
  }
  for (; left > 0; --left) {
    XT *dst = (cur == u) ? u_tmp : u;
    if constexpr (std::is_same<XT, float>::value) {
      if (widen_out && left == 1)  // the last sweep, widened (widen_fusable: sliced)
        return sliced_relax_sweep_widen(A.sl, d, f, cur, widen_out, s);
    }
    if (A.has_sl)
      BCMG_TRY(sliced_relax_sweep<XT>(A.sl, d, f, cur, dst, s));
    else
      relax_sweep<XT>(G, blocks, s, A, d, f, cur, dst);
    cur = dst;
  }
  BCMG_LAUNCH_CHECK();
  if constexpr (std::is_same<XT, float>::value) {
    if (widen_out) return convert_f2d(n, u, widen_out, s);  // no sweep after the first
  }
  return BCMG_OK;
}

template <typename XT>
bcmg_status relax_residual_t(const MatView &A, const XT *d, const XT *f, XT *u, XT *u_tmp,
                             int k, int start, XT *res, cudaStream_t s) {
  if (A.n > 0 && A.has_sl && A.sl.cl_size > 0 && k >= 1) {
    BCMG_TRY(check_types<XT>(A));
    if (start == kStartFirstDone)
      return set_error(BCMG_ERR_INTERNAL, "first sweep fused where it cannot be");
    return sliced_cluster<XT>(A.sl, d, f, u, k, start != kStartLive, res, s);
  }
  BCMG_TRY(relax_t<XT>(A, d, f, u, u_tmp, k, start, s));
  return residual_t<XT>(A, f, u, res, s);
}

template <typename XT>
bcmg_status residual_t(const MatView &A, const XT *f, const XT *u, XT *res, cudaStream_t s) {
  if (A.n <= 0) return BCMG_OK;
  BCMG_TRY(check_types<XT>(A));
  if (A.has_sl) return sliced_residual<XT>(A.sl, f, u, res, s);
  const int G = group_for(A.nnz, A.n);
  residual_pass<XT>(G, grid_for(static_cast<int64_t>(A.n) * G), s, A, f, u, res);
  BCMG_LAUNCH_CHECK();
  return BCMG_OK;
}

template <typename XT>
bcmg_status restrict_t(int32_t nc, const int32_t *rptr, const int32_t *ridx, const XT *p,
                       const XT *x, XT *y, cudaStream_t s) {
  if (nc <= 0) return BCMG_OK;
  launch_pdl(k_restrict_t<XT>, ceil_div(nc, kThreads), kThreads, 0, s, nc, rptr, ridx, p, x, y);
  BCMG_LAUNCH_CHECK();
  return BCMG_OK;
}

template <typename XT>
bcmg_status prolong_t(int32_t n, const int32_t *agg, const XT *p, const XT *xc, XT *xf,
                      cudaStream_t s) {
  if (n <= 0) return BCMG_OK;
  launch_pdl(k_prolong_t<XT>, ceil_div(n, kThreads), kThreads, 0, s, n, agg, p, xc, xf);
  BCMG_LAUNCH_CHECK();
  return BCMG_OK;
}

template <typename XT>
bcmg_status fill_t(XT *x, int64_t n, XT v, cudaStream_t s) {
  if (n <= 0) return BCMG_OK;
  launch_pdl(k_fill_t<XT>, stream_grid(n), kThreads, 0, s, x, n, v);
  BCMG_LAUNCH_CHECK();
  return BCMG_OK;
}

template <typename XT>
bcmg_status axpy_t(int64_t n, XT a, const XT *x, XT *y, cudaStream_t s) {
  if (n <= 0) return BCMG_OK;
  launch_pdl(k_axpy_t<XT>, stream_grid(n), kThreads, 0, s, n, a, x, y);
  BCMG_LAUNCH_CHECK();
  return BCMG_OK;
}

template <typename XT>
bcmg_status scale_t(int64_t n, XT a, XT *x, cudaStream_t s) {
  if (n <= 0) return BCMG_OK;
  launch_pdl(k_scale_t<XT>, stream_grid(n), kThreads, 0, s, n, a, x);
  BCMG_LAUNCH_CHECK();
  return BCMG_OK;
}

template <typename XT>
bcmg_status copy_t(XT *dst, const XT *src, int64_t n, cudaStream_t s) {
  if (n <= 0 || dst == src) return BCMG_OK;
  launch_pdl(k_copy_t<XT>, stream_grid(n), kThreads, 0, s, n, src, dst);
  BCMG_LAUNCH_CHECK();
  return BCMG_OK;
}

template <typename XT>
bcmg_status restrict_first_sweep_t(int32_t nc, const int32_t *rptr, const int32_t *ridx,
                                   const XT *p, const XT *x, XT *y, const XT *dc, XT *u1,
                                   cudaStream_t s) {
  if (nc <= 0) return BCMG_OK;
  launch_pdl(k_restrict_first_t<XT>, ceil_div(nc, kThreads), kThreads, 0, s, nc, rptr, ridx,
             p, x, y, dc, u1);
  BCMG_LAUNCH_CHECK();
  return BCMG_OK;
}

bcmg_status convert_first_sweep(int64_t n, const double *in, const float *d, float *out,
                                float *u1, cudaStream_t s) {
  if (n <= 0) return BCMG_OK;
  launch_pdl(k_convert_first, stream_grid(n), kThreads, 0, s, n, in, d, out, u1);
  BCMG_LAUNCH_CHECK();
  return BCMG_OK;
}

bcmg_status convert_d2f(int64_t n, const double *in, float *out, cudaStream_t s) {
  if (n <= 0) return BCMG_OK;
  launch_pdl(k_convert<double, float>, stream_grid(n), kThreads, 0, s, n, in, out);
  BCMG_LAUNCH_CHECK();
  return BCMG_OK;
}

bcmg_status convert_f2d(int64_t n, const float *in, double *out, cudaStream_t s) {
  if (n <= 0) return BCMG_OK;
  launch_pdl(k_convert<float, double>, stream_grid(n), kThreads, 0, s, n, in, out);
  BCMG_LAUNCH_CHECK();
  return BCMG_OK;
}

bcmg_status convert_values(int64_t n, const double *in, void *out, int vtype, cudaStream_t s) {
  if (n <= 0) return BCMG_OK;
  switch (vtype) {
    case kValF32:
      launch_pdl(k_convert<double, float>, stream_grid(n), kThreads, 0, s, n, in,
             static_cast<float *>(out));
      break;
    case kValBF16:
      launch(k_to_bf16, stream_grid(n), kThreads, 0, s, n, in, static_cast<__nv_bfloat16 *>(out));
      break;
    case kValF16:
      launch(k_to_f16, stream_grid(n), kThreads, 0, s, n, in, static_cast<__half *>(out));
      break;
    default:
      return set_error(BCMG_ERR_INTERNAL, "bad value type %d", vtype);
  }
  BCMG_LAUNCH_CHECK();
  return BCMG_OK;
}

template <typename XT>
bcmg_status spmv_t(const MatView &A, const XT *x, XT *y, cudaStream_t s) {
  if (A.n <= 0) return BCMG_OK;
  BCMG_TRY(check_types<XT>(A));
  if (A.has_sl) return sliced_spmv_t<XT>(A.sl, x, y, s);
  const int G = group_for(A.nnz, A.n);
  const int blocks = grid_for(static_cast<int64_t>(A.n) * G);
#define BCMG_SPMV_G(VT_)                                                                       \
  switch (G) {                                                                                 \
    case 4: launch_pdl(k_spmv_t<4, VT_, XT>, blocks, kThreads, 0, s, A.n, A.row, A.col, static_cast<const VT_ *>(A.val), x, y); break;  \
    case 8: launch_pdl(k_spmv_t<8, VT_, XT>, blocks, kThreads, 0, s, A.n, A.row, A.col, static_cast<const VT_ *>(A.val), x, y); break;  \
    case 16: launch_pdl(k_spmv_t<16, VT_, XT>, blocks, kThreads, 0, s, A.n, A.row, A.col, static_cast<const VT_ *>(A.val), x, y); break; \
    default: launch_pdl(k_spmv_t<32, VT_, XT>, blocks, kThreads, 0, s, A.n, A.row, A.col, static_cast<const VT_ *>(A.val), x, y); break; \
  }
  if (std::is_same<XT, double>::value) {
    BCMG_SPMV_G(double)
  } else if (A.vtype == kValF32) {
    BCMG_SPMV_G(float)
  } else if (A.vtype == kValBF16) {
    BCMG_SPMV_G(__nv_bfloat16)
  } else {
    BCMG_SPMV_G(__half)
  }
#undef BCMG_SPMV_G
  BCMG_LAUNCH_CHECK();
  return BCMG_OK;
}

template <typename XT>
bcmg_status dot_t(int64_t n, const XT *a, const XT *b, double *out, double *partials,
                  cudaStream_t s) {
  launch_pdl(k_dot_t<XT>, kRedBlocks, kRedThreads, 0, s, n, a, b, partials);
  launch_pdl(k_dot_t_final, 1, kRedThreads, 0, s, partials, out);
  BCMG_LAUNCH_CHECK();
  return BCMG_OK;
}

#define BCMG_INSTANTIATE(XT)                                                               \
  template bcmg_status relax_t<XT>(const MatView &, const XT *, const XT *, XT *, XT *, int, \
                                   int, cudaStream_t, double *);                           \
  template bcmg_status relax_residual_t<XT>(const MatView &, const XT *, const XT *, XT *,  \
                                            XT *, int, int, XT *, cudaStream_t);           \
  template bcmg_status restrict_first_sweep_t<XT>(int32_t, const int32_t *, const int32_t *, \
                                                  const XT *, const XT *, XT *, const XT *, \
                                                  XT *, cudaStream_t);                     \
  template bcmg_status residual_t<XT>(const MatView &, const XT *, const XT *, XT *,       \
                                      cudaStream_t);                                       \
  template bcmg_status restrict_t<XT>(int32_t, const int32_t *, const int32_t *, const XT *, \
                                      const XT *, XT *, cudaStream_t);                     \
  template bcmg_status prolong_t<XT>(int32_t, const int32_t *, const XT *, const XT *, XT *, \
                                     cudaStream_t);                                        \
  template bcmg_status fill_t<XT>(XT *, int64_t, XT, cudaStream_t);                        \
  template bcmg_status axpy_t<XT>(int64_t, XT, const XT *, XT *, cudaStream_t);            \
  template bcmg_status scale_t<XT>(int64_t, XT, XT *, cudaStream_t);                       \
  template bcmg_status copy_t<XT>(XT *, const XT *, int64_t, cudaStream_t);               \
  template bcmg_status spmv_t<XT>(const MatView &, const XT *, XT *, cudaStream_t);         \
  template bcmg_status dot_t<XT>(int64_t, const XT *, const XT *, double *, double *,       \
                                 cudaStream_t);

BCMG_INSTANTIATE(double)
BCMG_INSTANTIATE(float)

}  // namespace bcmg
