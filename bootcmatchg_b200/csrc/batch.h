// Multi-right-hand-side kernels: W right-hand sides (W a power of two, at
// most 32) share one hierarchy.  Vectors of a batch are stored interleaved,
// element (i, c) of an n x W block at x[i * W + c], so one matrix row is read
// once for all W columns and the gather of x at one column index is one
// contiguous W-element segment.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

#include "bcmg.h"
#include "kernels.h"

namespace bcmg {

constexpr int kBatchMax = 32;

// Launch shape of the row kernels: V consecutive columns per lane (so
// W / V lanes share a row) and threads per block.  Row sums do not depend on
// the shape (each column's row sum is accumulated sequentially in CSR
// order), so the relaxation and residual kernels give the same bits for every
// shape; the per-column dot products fused into bt_fcg_spmv_dots are
// partitioned by it.
struct BtCfg {
  int V = 1;
  int threads = 256;
};

// Per-column FCG scalars: column c's block starts at scal[c * kBtStride]
// and holds the FcgScal entries followed by kBtAct (column still iterating).
constexpr int kBtAct = kNumScal;
constexpr int kBtStride = kNumScal + 1;

template <typename XT>  // k sweeps of u <- ((-(A u) + f) ./ d) + u on W columns
bcmg_status bt_relax(const MatView &A, int W, BtCfg cfg, const XT *d, const XT *f, XT *u,
                     XT *u_tmp, int k, bool zero_start, cudaStream_t s);
template <typename XT>  // res = f - A u on W columns
bcmg_status bt_residual(const MatView &A, int W, BtCfg cfg, const XT *f, const XT *u, XT *res,
                        cudaStream_t s);
template <typename XT>  // y = A x on W columns (A: n rows; x indexed by A's columns)
bcmg_status bt_spmm(const MatView &A, int W, BtCfg cfg, const XT *x, XT *y, cudaStream_t s);
template <typename XT>  // y[I, :] = sum_{i in I} p_i x[i, :]
bcmg_status bt_restrict(int32_t nc, const int32_t *rptr, const int32_t *ridx, const XT *p,
                        const XT *x, XT *y, int W, cudaStream_t s);
template <typename XT>  // xf[i, :] += p_i xc[agg_i, :]
bcmg_status bt_prolong(int32_t n, const int32_t *agg, const XT *p, const XT *xc, XT *xf, int W,
                       cudaStream_t s);

// Column-major (leading dimension ld, m <= W columns) <-> interleaved; the
// columns m..W-1 of the interleaved block are written as zeros by bt_pack.
bcmg_status bt_pack(int32_t n, int m, const double *src, int64_t ld, double *dst, int W,
                    cudaStream_t s);
bcmg_status bt_unpack(int32_t n, int m, const double *src, int W, double *dst, int64_t ld,
                      cudaStream_t s);

// ---- per-column FCG (FP64) --------------------------------------------------
// partials: kRedBlocks * 4 * W doubles; scal: W * kBtStride doubles; flags:
// [0] some column still iterating, [1] some column replaces its residual.
//
// Column norms of r and b: kDelta0, kBnorm, kNorm, kTarget = rtol kDelta0,
// kItnlim; a column is active unless kDelta0 <= DBL_EPSILON kBnorm.
bcmg_status bt_fcg_init(int32_t n, int W, const double *r, const double *b, double rtol,
                        int itnlim, double *partials, double *scal, int *flags, cudaStream_t s);
// w = A v with per-column alpha = r.v, beta = w.v, gamma = q.v (q may be null).
bcmg_status bt_fcg_spmv_dots(const CsrView &A, int W, BtCfg cfg, const double *v, double *w,
                             const double *r, const double *q, double *partials,
                             cudaStream_t s);
bcmg_status bt_fcg_scalars(const double *partials, double *scal, int W, bool first,
                           cudaStream_t s);
bcmg_status bt_fcg_update(int32_t n, int W, bool first, const double *z, double *zp,
                          const double *az, double *azp, double *x, double *r,
                          double *partials, double *scal, cudaStream_t s);
bcmg_status bt_fcg_replace(const CsrView &A, int W, BtCfg cfg, const double *b,
                           const double *x, double *r, double *partials, double *scal,
                           int *flags, int every, cudaStream_t s);
bcmg_status bt_fcg_continue(double *scal, int W, int *flags, cudaGraphConditionalHandle cond,
                            bool use_cond, cudaStream_t s);
// out[c] = ||a[:, c]||_2 for the W columns.
bcmg_status bt_col_norms(int32_t n, int W, const double *a, double *partials, double *out,
                         cudaStream_t s);

}  // namespace bcmg
