// Sliced matrix format for the solve phase and its kernels.
//
// Rows are cut into slices of 32 (one warp, one thread per row).  A slice
// stores W slots of 32 values in slot-major order, so every value load of a
// warp is one contiguous 32-element segment.  Two slot kinds:
//   offset slice: the slice's rows share a set of W column offsets
//                 (col - row), e.g. a stencil; column indices are implicit
//                 (row + offset) and only W offsets are stored per slice;
//   column slice: W = longest row; explicit int32 columns per slot (SELL-32).
// Missing entries are stored as 0 (with an in-range column), which adds exact
// zeros to the row sums.  Built on the device from the level's CSR after
// setup; CSR stays the setup / introspection format.
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <algorithm>
#include <climits>
#include <vector>

#include "common.cuh"
#include "kernels.h"
#include "reduce.cuh"
#include "scan.cuh"

namespace bcmg {
namespace {

constexpr int kWarpsPerBlock = 8;
constexpr int kMaxOffsetSlots = 64;  // wider unions fall back to column slices

__device__ __forceinline__ double widen(double v) { return v; }
__device__ __forceinline__ float widen(float v) { return v; }
__device__ __forceinline__ float widen(__nv_bfloat16 v) { return __bfloat162float(v); }
__device__ __forceinline__ float widen(__half v) { return __half2float(v); }

template <typename VT>
__device__ __forceinline__ VT narrow(double v);
template <>
__device__ __forceinline__ double narrow<double>(double v) { return v; }
template <>
__device__ __forceinline__ float narrow<float>(double v) { return static_cast<float>(v); }
template <>
__device__ __forceinline__ __nv_bfloat16 narrow<__nv_bfloat16>(double v) {
  return __double2bfloat16(v);
}
template <>
__device__ __forceinline__ __half narrow<__half>(double v) { return __double2half(v); }

// Pass 1: per slice, the longest row and the size of the union of column
// offsets (merging the 32 sorted rows); chooses the slice kind and width.
__global__ void k_slice_shape(int32_t n, int32_t nslices, const int32_t *__restrict__ row,
                              const int32_t *__restrict__ col, int32_t *width,
                              int32_t *kind) {
  const int lane = threadIdx.x & 31;
  const int32_t s = blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5);
  if (s >= nslices) return;
  const int32_t r = s * 32 + lane;
  int32_t b = 0, e = 0;
  if (r < n) {
    b = row[r];
    e = row[r + 1];
  }
  int len = e - b;
  int maxlen = len;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) maxlen = max(maxlen, __shfl_xor_sync(0xffffffffu, maxlen, o));
  // Merge the sorted offset lists; count distinct offsets up to the cap.
  int32_t pos = b;
  int distinct = 0;
  while (distinct <= kMaxOffsetSlots) {
    const int32_t cur = pos < e ? col[pos] - r : INT_MAX;
    int32_t m = cur;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = min(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (m == INT_MAX) break;
    ++distinct;
    if (cur == m) ++pos;
  }
  if (lane == 0) {
    const bool offsets = distinct <= kMaxOffsetSlots && distinct <= maxlen + maxlen / 4 + 2;
    kind[s] = offsets ? 1 : 0;
    width[s] = offsets ? distinct : maxlen;
  }
}

// Pass 2: fill values (and columns or offsets).
template <typename VT>
__global__ void k_slice_fill(int32_t n, int32_t nslices, const int32_t *__restrict__ row,
                             const int32_t *__restrict__ col,
                             const double *__restrict__ val,
                             const int32_t *__restrict__ sptr,
                             const int32_t *__restrict__ width,
                             const int32_t *__restrict__ kind, VT *sval, int32_t *scol,
                             int32_t *soff) {
  const int lane = threadIdx.x & 31;
  const int32_t s = blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5);
  if (s >= nslices) return;
  const int32_t r = s * 32 + lane;
  const int32_t rr = r < n ? r : n - 1;
  int32_t b = 0, e = 0;
  if (r < n) {
    b = row[r];
    e = row[r + 1];
  }
  const int64_t base = static_cast<int64_t>(sptr[s]) * 32;
  const int W = width[s];
  if (kind[s]) {
    int32_t pos = b;
    for (int k = 0; k < W; ++k) {
      const int32_t cur = pos < e ? col[pos] - r : INT_MAX;
      int32_t m = cur;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) m = min(m, __shfl_xor_sync(0xffffffffu, m, o));
      double v = 0.0;
      if (cur == m) {
        v = val[pos];
        ++pos;
      }
      sval[base + static_cast<int64_t>(k) * 32 + lane] = narrow<VT>(v);
      if (lane == 0) soff[sptr[s] + k] = m;
    }
  } else {
    for (int k = 0; k < W; ++k) {
      const int32_t j = b + k;
      const bool have = j < e;
      sval[base + static_cast<int64_t>(k) * 32 + lane] = narrow<VT>(have ? val[j] : 0.0);
      scol[base + static_cast<int64_t>(k) * 32 + lane] = have ? col[j] : rr;
    }
  }
}

// Row sum of one slice row: t = sum_k val[k] * x[col_k].  Slots are taken
// eight at a time with all eight value loads issued before the gathers and
// the FMAs, so each thread keeps eight independent loads in flight (the
// sweep is bound by memory latency, not by issue).
constexpr int kBatch = 8;

template <typename VT, typename XT, bool OFFSETS>
__device__ __forceinline__ XT sliced_dot_kind(const SlicedView &S, const VT *__restrict__ v,
                                              const XT *__restrict__ x, int32_t sp, int W,
                                              int32_t r) {
  XT t[4] = {XT(0), XT(0), XT(0), XT(0)};
  const int32_t *off = S.soff + sp;
  const int32_t *cidx =
      OFFSETS ? nullptr : S.scol + static_cast<int64_t>(sp) * 32 + (threadIdx.x & 31);
  const int32_t hi = S.n - 1;
#define BCMG_SLICED_COLUMN(k_)                                                       \
  (OFFSETS ? min(max(r + __ldg(off + (k_)), 0), hi) : cidx[static_cast<int64_t>(k_) * 32])
  int k = 0;
  for (; k + kBatch <= W; k += kBatch) {
    VT a[kBatch];
    int32_t c[kBatch];
#pragma unroll
    for (int u = 0; u < kBatch; ++u) {
      a[u] = v[static_cast<int64_t>(k + u) * 32];
      c[u] = BCMG_SLICED_COLUMN(k + u);
    }
    XT xv[kBatch];
#pragma unroll
    for (int u = 0; u < kBatch; ++u) xv[u] = __ldg(x + c[u]);
#pragma unroll
    for (int u = 0; u < kBatch; ++u) t[u & 3] = fma(static_cast<XT>(widen(a[u])), xv[u], t[u & 3]);
  }
  for (; k < W; ++k)
    t[k & 3] = fma(static_cast<XT>(widen(v[static_cast<int64_t>(k) * 32])),
                   __ldg(x + BCMG_SLICED_COLUMN(k)), t[k & 3]);
#undef BCMG_SLICED_COLUMN
  return (t[0] + t[1]) + (t[2] + t[3]);
}

template <typename VT, typename XT>
__device__ __forceinline__ XT sliced_dot(const SlicedView &S, const VT *__restrict__ val,
                                         const XT *__restrict__ x, int32_t s, int32_t r,
                                         int lane) {
  const int32_t sp = S.sptr[s];
  const int W = S.width[s];
  const VT *v = val + static_cast<int64_t>(sp) * 32 + lane;
  if (S.kind[s]) return sliced_dot_kind<VT, XT, true>(S, v, x, sp, W, r);
  return sliced_dot_kind<VT, XT, false>(S, v, x, sp, W, r);
}

template <typename VT, typename XT>
__global__ void __launch_bounds__(kWarpsPerBlock * 32, 4)
    k_sl_relax(SlicedView S, const VT *__restrict__ val, const XT *__restrict__ d,
               const XT *__restrict__ f, const XT *__restrict__ u, XT *__restrict__ u_out) {
  const int lane = threadIdx.x & 31;
  const int32_t s = blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5);
  if (s >= S.nslices) return;
  const int32_t r = s * 32 + lane;
  const XT T = sliced_dot<VT, XT>(S, val, u, s, r, lane);
  if (r < S.n) u_out[r] = ((-T + f[r]) / d[r]) + u[r];
}

template <typename VT, typename XT>
__global__ void __launch_bounds__(kWarpsPerBlock * 32, 4)
    k_sl_residual(SlicedView S, const VT *__restrict__ val, const XT *__restrict__ f,
                  const XT *__restrict__ u, XT *__restrict__ res) {
  const int lane = threadIdx.x & 31;
  const int32_t s = blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5);
  if (s >= S.nslices) return;
  const int32_t r = s * 32 + lane;
  const XT T = sliced_dot<VT, XT>(S, val, u, s, r, lane);
  if (r < S.n) res[r] = f[r] - T;
}

// FCG SpMV on the sliced FP64 copy with the three dot products fused; fixed
// grid (kRedBlocks) and slice-to-block mapping keep the partials deterministic.
__global__ void __launch_bounds__(kWarpsPerBlock * 32, 4)
    k_sl_fcg_spmv_dots(SlicedView S, const double *__restrict__ v, double *__restrict__ w,
                       const double *__restrict__ r, const double *__restrict__ q,
                       double *partials) {
  double acc[3] = {0.0, 0.0, 0.0};
  const int lane = threadIdx.x & 31;
  const double *val = static_cast<const double *>(S.val);
  for (int32_t s = blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5); s < S.nslices;
       s += gridDim.x * kWarpsPerBlock) {
    const int32_t row = s * 32 + lane;
    const double T = sliced_dot<double, double>(S, val, v, s, row, lane);
    if (row < S.n) {
      w[row] = T;
      const double vi = v[row];
      acc[0] = fma(r[row], vi, acc[0]);
      acc[1] = fma(T, vi, acc[1]);
      if (q) acc[2] = fma(q[row], vi, acc[2]);
    }
  }
  block_partials<3>(acc, partials);
}

__global__ void __launch_bounds__(kWarpsPerBlock * 32, 4)
    k_sl_spmv(SlicedView S, const double *__restrict__ val, const double *__restrict__ x,
              double *__restrict__ y) {
  const int lane = threadIdx.x & 31;
  const int32_t s = blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5);
  if (s >= S.nslices) return;
  const int32_t r = s * 32 + lane;
  const double T = sliced_dot<double, double>(S, val, x, s, r, lane);
  if (r < S.n) y[r] = T;
}

template <typename VT, typename XT>
void sl_relax_launch(const SlicedView &S, const XT *d, const XT *f, const XT *src, XT *dst,
                     cudaStream_t st) {
  launch(k_sl_relax<VT, XT>, ceil_div(S.nslices, kWarpsPerBlock), kWarpsPerBlock * 32, 0, st,
         S, static_cast<const VT *>(S.val), d, f, src, dst);
}

template <typename VT, typename XT>
void sl_residual_launch(const SlicedView &S, const XT *f, const XT *u, XT *res,
                        cudaStream_t st) {
  launch(k_sl_residual<VT, XT>, ceil_div(S.nslices, kWarpsPerBlock), kWarpsPerBlock * 32, 0,
         st, S, static_cast<const VT *>(S.val), f, u, res);
}

}  // namespace

size_t SlicedMat::bytes() const {
  if (!nslices) return 0;
  const size_t vbytes = vtype == kValF64 ? 8 : (vtype == kValF32 ? 4 : 2);
  const size_t sl = static_cast<size_t>(slots) * 32;
  return vbytes * sl + 16 + (has_columns ? 4 * sl : 0) + 4 * (static_cast<size_t>(slots) + 1) +
         4 * (3 * static_cast<size_t>(nslices) + 1);
}

void SlicedMat::release(cudaStream_t s) {
  dev_free(sptr, s);
  dev_free(width, s);
  dev_free(kind, s);
  dev_free(scol, s);
  dev_free(soff, s);
  if (val) cudaFreeAsync(val, s);
  val = nullptr;
  nslices = 0;
  has_columns = false;
}

SlicedView SlicedMat::view() const {
  SlicedView v;
  v.n = n;
  v.nslices = nslices;
  v.sptr = sptr;
  v.width = width;
  v.kind = kind;
  v.scol = scol;
  v.soff = soff;
  v.val = val;
  v.vtype = vtype;
  return v;
}

bcmg_status sliced_build(const CsrView &A, int vtype, SlicedMat *out, cudaStream_t s) {
  out->release(s);
  const int32_t n = A.n;
  if (n <= 0) return BCMG_OK;
  const int32_t ns = ceil_div(n, 32);
  out->n = n;
  out->nslices = ns;
  out->vtype = vtype;
  BCMG_TRY(dev_alloc(&out->sptr, ns + 1, s));
  BCMG_TRY(dev_alloc(&out->width, ns, s));
  BCMG_TRY(dev_alloc(&out->kind, ns, s));
  const int blocks = ceil_div(ns, kWarpsPerBlock);
  launch(k_slice_shape, blocks, kWarpsPerBlock * 32, 0, s, n, ns, A.row, A.col, out->width,
         out->kind);
  DevBuf<int32_t> tmp;
  BCMG_TRY(tmp.alloc(scan_tmp_size(ns), s));
  BCMG_TRY(exclusive_scan(out->width, out->sptr, ns, out->sptr + ns, tmp.get(), s));
  int32_t slots = 0;
  std::vector<int32_t> kinds(ns);
  BCMG_CUDA(cudaMemcpyAsync(&slots, out->sptr + ns, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  BCMG_CUDA(cudaMemcpyAsync(kinds.data(), out->kind, sizeof(int32_t) * ns,
                            cudaMemcpyDeviceToHost, s));
  BCMG_CUDA(cudaStreamSynchronize(s));
  out->slots = slots;
  const size_t vbytes = vtype == kValF64 ? 8 : (vtype == kValF32 ? 4 : 2);
  BCMG_CUDA(cudaMallocAsync(&out->val, vbytes * static_cast<size_t>(slots) * 32 + 16, s));
  // Explicit columns are only read in column slices; a matrix made of offset
  // slices alone (a stencil) stores none.
  out->has_columns = std::any_of(kinds.begin(), kinds.end(), [](int32_t k) { return k == 0; });
  if (out->has_columns) BCMG_TRY(dev_alloc(&out->scol, static_cast<int64_t>(slots) * 32, s));
  BCMG_TRY(dev_alloc(&out->soff, slots + 1, s));
  switch (vtype) {
    case kValF64:
      launch(k_slice_fill<double>, blocks, kWarpsPerBlock * 32, 0, s, n, ns, A.row, A.col,
             A.val, out->sptr, out->width, out->kind, static_cast<double *>(out->val),
             out->scol, out->soff);
      break;
    case kValF32:
      launch(k_slice_fill<float>, blocks, kWarpsPerBlock * 32, 0, s, n, ns, A.row, A.col,
             A.val, out->sptr, out->width, out->kind, static_cast<float *>(out->val),
             out->scol, out->soff);
      break;
    case kValBF16:
      launch(k_slice_fill<__nv_bfloat16>, blocks, kWarpsPerBlock * 32, 0, s, n, ns, A.row,
             A.col, A.val, out->sptr, out->width, out->kind,
             static_cast<__nv_bfloat16 *>(out->val), out->scol, out->soff);
      break;
    default:
      launch(k_slice_fill<__half>, blocks, kWarpsPerBlock * 32, 0, s, n, ns, A.row, A.col,
             A.val, out->sptr, out->width, out->kind, static_cast<__half *>(out->val),
             out->scol, out->soff);
      break;
  }
  BCMG_LAUNCH_CHECK();
  return BCMG_OK;
}

template <typename XT>
bcmg_status sliced_relax_sweep(const SlicedView &S, const XT *d, const XT *f, const XT *u,
                               XT *u_out, cudaStream_t s) {
  if (std::is_same<XT, double>::value) {
    if (S.vtype != kValF64) return set_error(BCMG_ERR_INTERNAL, "sliced type mismatch");
    sl_relax_launch<double, double>(S, reinterpret_cast<const double *>(d),
                                    reinterpret_cast<const double *>(f),
                                    reinterpret_cast<const double *>(u),
                                    reinterpret_cast<double *>(u_out), s);
  } else {
    const float *df = reinterpret_cast<const float *>(d);
    const float *ff = reinterpret_cast<const float *>(f);
    const float *uf = reinterpret_cast<const float *>(u);
    float *of = reinterpret_cast<float *>(u_out);
    if (S.vtype == kValF32) sl_relax_launch<float, float>(S, df, ff, uf, of, s);
    else if (S.vtype == kValBF16) sl_relax_launch<__nv_bfloat16, float>(S, df, ff, uf, of, s);
    else if (S.vtype == kValF16) sl_relax_launch<__half, float>(S, df, ff, uf, of, s);
    else return set_error(BCMG_ERR_INTERNAL, "sliced type mismatch");
  }
  BCMG_LAUNCH_CHECK();
  return BCMG_OK;
}

template <typename XT>
bcmg_status sliced_residual(const SlicedView &S, const XT *f, const XT *u, XT *res,
                            cudaStream_t s) {
  if (std::is_same<XT, double>::value) {
    if (S.vtype != kValF64) return set_error(BCMG_ERR_INTERNAL, "sliced type mismatch");
    sl_residual_launch<double, double>(S, reinterpret_cast<const double *>(f),
                                       reinterpret_cast<const double *>(u),
                                       reinterpret_cast<double *>(res), s);
  } else {
    const float *ff = reinterpret_cast<const float *>(f);
    const float *uf = reinterpret_cast<const float *>(u);
    float *rf = reinterpret_cast<float *>(res);
    if (S.vtype == kValF32) sl_residual_launch<float, float>(S, ff, uf, rf, s);
    else if (S.vtype == kValBF16) sl_residual_launch<__nv_bfloat16, float>(S, ff, uf, rf, s);
    else if (S.vtype == kValF16) sl_residual_launch<__half, float>(S, ff, uf, rf, s);
    else return set_error(BCMG_ERR_INTERNAL, "sliced type mismatch");
  }
  BCMG_LAUNCH_CHECK();
  return BCMG_OK;
}

bcmg_status sliced_fcg_spmv_dots(const SlicedView &S, const double *v, double *w,
                                 const double *r, const double *q, double *partials,
                                 cudaStream_t s) {
  if (S.vtype != kValF64) return set_error(BCMG_ERR_INTERNAL, "FCG SpMV needs FP64 values");
  launch(k_sl_fcg_spmv_dots, kRedBlocks, kWarpsPerBlock * 32, 0, s, S, v, w, r, q, partials);
  BCMG_LAUNCH_CHECK();
  return BCMG_OK;
}

bcmg_status sliced_spmv(const SlicedView &S, const double *x, double *y, cudaStream_t s) {
  if (S.vtype != kValF64) return set_error(BCMG_ERR_INTERNAL, "sliced SpMV needs FP64 values");
  launch(k_sl_spmv, ceil_div(S.nslices, kWarpsPerBlock), kWarpsPerBlock * 32, 0, s, S,
         static_cast<const double *>(S.val), x, y);
  BCMG_LAUNCH_CHECK();
  return BCMG_OK;
}

template bcmg_status sliced_relax_sweep<double>(const SlicedView &, const double *,
                                                const double *, const double *, double *,
                                                cudaStream_t);
template bcmg_status sliced_relax_sweep<float>(const SlicedView &, const float *,
                                               const float *, const float *, float *,
                                               cudaStream_t);
template bcmg_status sliced_residual<double>(const SlicedView &, const double *,
                                             const double *, double *, cudaStream_t);
template bcmg_status sliced_residual<float>(const SlicedView &, const float *, const float *,
                                            float *, cudaStream_t);

}  // namespace bcmg
