// Host-callable launchers for the library's CUDA kernels.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

#include "bcmg.h"

namespace bcmg {

// Read-only view of a device CSR matrix (0-based, sorted columns).
struct CsrView {
  int32_t n = 0;
  int32_t nnz = 0;
  const int32_t *row = nullptr;
  const int32_t *col = nullptr;
  const double *val = nullptr;
};

// ---- setup (k_setup.cu; FP64, no FMA contraction) -------------------------
bcmg_status level_prep(const CsrView &A, double *D, double *M, cudaStream_t s);
bcmg_status pair_aggregate(const CsrView &A, const double *w, int32_t *agg,
                           double *p, int32_t *nc, double *W_out,
                           int32_t *s_out, int32_t *m_out, cudaStream_t s);
bcmg_status transpose_agg(int32_t n, const int32_t *agg, int32_t nc,
                          int32_t *rptr, int32_t *ridx, cudaStream_t s);
bcmg_status galerkin_count(const CsrView &A, const int32_t *agg, const double *p,
                           int32_t nc, const int32_t *rptr, const int32_t *ridx,
                           int32_t *crow, int32_t *cnnz, cudaStream_t s);
bcmg_status galerkin_fill(const CsrView &A, const int32_t *agg, const double *p,
                          int32_t nc, const int32_t *rptr, const int32_t *ridx,
                          const int32_t *crow, int32_t *ccol, double *cval,
                          cudaStream_t s);
bcmg_status restrict_exact(int32_t nc, const int32_t *rptr, const int32_t *ridx,
                           const double *p, const double *x, double *y,
                           cudaStream_t s);
bcmg_status compose_p(int32_t n, int32_t *agg, double *p, const int32_t *agg2,
                      const double *p2, cudaStream_t s);

// ---- solve (k_solve.cu) ----------------------------------------------------
// k sweeps of u <- ((-(A u) + f) ./ d) + u; u_tmp is a ping-pong buffer.
// If zero_start, u is taken as 0 on entry (first sweep is f ./ d).  Returns
// in *result whichever of u / u_tmp holds the final iterate.
bcmg_status relax(const CsrView &A, const double *d, const double *f, double *u,
                  double *u_tmp, int k, bool zero_start, double **result,
                  cudaStream_t s);
// y = alpha A x + beta y
bcmg_status spmv(const CsrView &A, double alpha, const double *x, double beta,
                 double *y, cudaStream_t s);
// res = f - A u
bcmg_status residual(const CsrView &A, const double *f, const double *u, double *res,
                     cudaStream_t s);
// y[I] = sum_{i in I} p_i x_i
bcmg_status restrict_vec(int32_t nc, const int32_t *rptr, const int32_t *ridx,
                         const double *p, const double *x, double *y, cudaStream_t s);
// xf[i] += p_i xc[agg_i]
bcmg_status prolong_add(int32_t n, const int32_t *agg, const double *p,
                        const double *xc, double *xf, cudaStream_t s);
bcmg_status fill(double *x, int64_t n, double v, cudaStream_t s);
bcmg_status copy(double *dst, const double *src, int64_t n, cudaStream_t s);
// y = alpha x + y
bcmg_status axpy(int64_t n, double alpha, const double *x, double *y, cudaStream_t s);
bcmg_status scale(int64_t n, double alpha, double *x, cudaStream_t s);

// Deterministic FP64 reductions into device scalars.
constexpr int kRedBlocks = 4 * 148;
struct Reducer {
  double *partials = nullptr;  // kRedBlocks * 4
  double *scal = nullptr;      // device scalars (see FcgScal)
};
// out = a . b into *out (device)
bcmg_status dot_dev(int64_t n, const double *a, const double *b, double *out,
                    double *partials, cudaStream_t s);

// FCG device scalars.
enum FcgScal {
  kAlpha = 0, kBeta, kGamma, kDelta, kTheta, kTheta2, kNorm, kDelta0,
  kBnorm, kIndef, kNumScal
};
// w = A v fused with alpha = r.v, beta = w.v, gamma = q.v (q may be null).
bcmg_status fcg_spmv_dots(const CsrView &A, const double *v, double *w,
                          const double *r, const double *q, double *partials,
                          double *scal, cudaStream_t s);
// first==true: delta = beta, theta = alpha / delta; else FCG v3 recurrences.
bcmg_status fcg_scalars(double *partials, double *scal, bool first, cudaStream_t s);
// first step: x += theta v; r -= theta w; norm.
// loop step:  z = -theta zp + z; x += theta2 z; az = -theta azp + az;
//             r -= theta2 az; norm.
bcmg_status fcg_update(int64_t n, bool first, double *z, const double *zp,
                       double *az, const double *azp, double *x, double *r,
                       double *partials, double *scal, cudaStream_t s);

}  // namespace bcmg
