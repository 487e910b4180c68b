// Host-callable launchers for the library's CUDA kernels.
#pragma once

#include <cuda_runtime.h>
#include <cstddef>
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

// Phase timing hook (driver.cu): with ext.verbose >= 1 it synchronises the
// stream and charges the elapsed wall time to `name`; otherwise a no-op.
void phase_tick(const char *name);

// ---- setup (k_setup.cu; FP64, no FMA contraction) -------------------------
bcmg_status level_prep(const CsrView &A, double *D, double *M, cudaStream_t s);
// step_limit bounds the steps of each matching thread (0: 8 nnz + 1024); a
// thread that runs out makes it return BCMG_ERR_DEVICE_TIMEOUT.
bcmg_status pair_aggregate(const CsrView &A, const double *w, int32_t *agg,
                           double *p, int32_t *nc, double *W_out,
                           int32_t *s_out, int32_t *m_out, cudaStream_t s,
                           int64_t step_limit = 0);
bcmg_status transpose_agg(int32_t n, const int32_t *agg, int32_t nc,
                          int32_t *rptr, int32_t *ridx, cudaStream_t s);
// A_c = P^T A P into crow (nc+1, caller-allocated) and *ccol/*cval
// (allocated on stream s, *cnnz entries).
bcmg_status galerkin(const CsrView &A, const int32_t *agg, const double *p, int32_t nc,
                     const int32_t *rptr, const int32_t *ridx, int32_t *crow,
                     int32_t **ccol, double **cval, int32_t *cnnz, cudaStream_t s);
bcmg_status restrict_exact(int32_t nc, const int32_t *rptr, const int32_t *ridx,
                           const double *p, const double *x, double *y,
                           cudaStream_t s);
bcmg_status compose_p(int32_t n, int32_t *agg, double *p, const int32_t *agg2,
                      const double *p2, cudaStream_t s);
// C = X Y (X: n rows, Y: m columns) in the canonical summation order; crow
// (n+1) caller-allocated, *ccol/*cval allocated on s (*cnnz entries).
bcmg_status spgemm(const CsrView &X, const CsrView &Y, int32_t m, int32_t *crow,
                   int32_t **ccol, double **cval, int32_t *cnnz, cudaStream_t s);
// A^T (A: n x m) into trow (m+1), tcol, tval (nnz), rows sorted by column.
bcmg_status csr_transpose(const CsrView &A, int32_t m, int32_t *trow, int32_t *tcol,
                          double *tval, cudaStream_t s);
// sval = values of S = I - omega D^{-1} A, omega = 4 / (3 ||D^{-1} A||_inf).
bcmg_status smoothing_operator(const CsrView &A, const double *D, double *sval,
                               cudaStream_t s);
bcmg_status iota(int32_t n, int32_t *x, cudaStream_t s);  // x[i] = i, i <= n

// ---- cycle (k_cycle.cu) ----------------------------------------------------
// Value storage of a level matrix used by the cycle.
enum ValType { kValF64 = 0, kValF32 = 1, kValBF16 = 2, kValF16 = 3 };

// Sliced solve-phase format (k_sliced.cu): 32-row slices, slot-major values.
// meta[s] = {first slot, width W, kind, offset base}: kind 1 = shared column
// offsets soff[base + k] (base = the first slice of a run of slices with the
// same offsets); kind 0 = explicit columns scol[32 first + 32 k + lane].
// Values, columns and offsets are padded past the last slot.
// Default bound on each wait of a pipelined row pass for its staged copies
// (bcmg_ext.max_device_seconds overrides it per handle).
constexpr unsigned long long kDefaultWaitNs = 2000000000ull;

constexpr int kStencilMax = 32;  // the widest slot batch of the sliced kernels

struct SlicedView {
  int32_t n = 0, nslices = 0;
  const int32_t *sptr = nullptr;  // first slot of each slice (nslices + 1)
  const int4 *meta = nullptr;
  const int32_t *scol = nullptr, *soff = nullptr;
  const void *val = nullptr;
  int vtype = kValF64;
  int32_t cap_slots = 0;    // slots one pipeline stage holds
  int32_t cols_staged = 0;  // explicit columns exist (and are staged)
  int32_t batch = 0;        // mean slice width (chooses the slot batch size)
  int xtype = kValF64;      // vector type the copy serves (kValF64 or kValF32)
  unsigned long long wait_ns = kDefaultWaitNs;  // bound on each pipeline wait
  // Small levels (sliced_cluster): the thread-block cluster size that holds
  // the whole copy in shared memory (0: the copy does not fit), slices per
  // CTA and the slot capacity of one CTA's shared memory.
  int32_t cl_size = 0, cl_spc = 0, cl_slots = 0;
  // Stencil slices (meta.z == 3): interior offset slices whose offsets are
  // exactly sten_off[0 .. sten_w), sten_w being the slot batch of the copy;
  // the kernels take those offsets from their parameters.
  int32_t sten_w = 0;
  int32_t sten_off[kStencilMax] = {};
};

struct SlicedMat {
  int32_t n = 0, nslices = 0, slots = 0;
  int32_t *sptr = nullptr, *scol = nullptr, *soff = nullptr;
  int4 *meta = nullptr;
  void *val = nullptr;
  int vtype = kValF64;
  int32_t cap_slots = 0, batch = 0;
  int xtype = kValF64;       // vector type served: kValF64 or kValF32
  bool narrowed = false;     // values stored narrower than xtype (all exact)
  bool has_columns = false;  // scol allocated (some slice is a column slice)
  unsigned long long wait_ns = kDefaultWaitNs;  // copied into every view
  int32_t cl_size = 0, cl_spc = 0, cl_slots = 0;  // see SlicedView
  int32_t sten_w = 0, sten_off[kStencilMax] = {};  // see SlicedView
  bool borrowed = false;  // the arrays belong to another copy (sliced_alias)
  void release(cudaStream_t s);
  size_t bytes() const;  // device bytes held
  SlicedView view() const;
};

// Builds the sliced copy of a CSR matrix with values converted to vtype
// (kValF64: a copy for FP64 vectors; otherwise for FP32 vectors).  narrow
// (FP64 and FP32 copies): store the values in BF16 / FP16 (or FP32 for an
// FP64 copy) instead when every value converts exactly (the kernels widen
// them, so results are bit-identical).
bcmg_status sliced_build(const CsrView &A, int vtype, SlicedMat *out, cudaStream_t s,
                         bool narrow = false);
// A copy serving xtype vectors that shares the arrays of src, a copy whose
// values are stored in 16 bits (narrowed): the same bytes serve FP64 and FP32
// vectors.  src must outlive it.
bcmg_status sliced_alias(const SlicedMat &src, int xtype, SlicedMat *out, cudaStream_t s);
template <typename XT>  // u_out = ((-(A u) + f) ./ d) + u
bcmg_status sliced_relax_sweep(const SlicedView &S, const XT *d, const XT *f, const XT *u,
                               XT *u_out, cudaStream_t s);
template <typename XT>  // res = f - A u
bcmg_status sliced_residual(const SlicedView &S, const XT *f, const XT *u, XT *res,
                            cudaStream_t s);
// sliced_relax_sweep on FP32 vectors with the result widened into FP64 out.
bcmg_status sliced_relax_sweep_widen(const SlicedView &S, const float *d, const float *f,
                                     const float *u, double *out, cudaStream_t s);
// y = A x on a sliced FP64 copy.
bcmg_status sliced_spmv(const SlicedView &S, const double *x, double *y, cudaStream_t s);
template <typename XT>  // y = A x on the copy serving XT vectors
bcmg_status sliced_spmv_t(const SlicedView &S, const XT *x, XT *y, cudaStream_t s);
// FCG SpMV w = A v fused with alpha = r.v, beta = w.v, gamma = q.v (FP64 values).
bcmg_status sliced_fcg_spmv_dots(const SlicedView &S, const double *v, double *w,
                                 const double *r, const double *q, double *partials,
                                 cudaStream_t s);
// k sweeps u <- ((-(A u) + f) ./ d) + u (zero_start: the first is f ./ d),
// then res = f - A u when res is given, in one launch of one thread-block
// cluster that holds the whole copy in shared memory (S.cl_size > 0): the
// iterate lives in distributed shared memory and passes are separated by
// cluster barriers.  Bit-identical to relax_t and residual_t.
template <typename XT>
bcmg_status sliced_cluster(const SlicedView &S, const XT *d, const XT *f, XT *u, int k,
                           bool zero_start, XT *res, cudaStream_t s);

// BCMG_ERR_DEVICE_TIMEOUT (and the flag cleared) if a sliced row pass gave up
// waiting for its staged copies since the last call; synchronises s.
bcmg_status sliced_wait_status(cudaStream_t s);
// Runs a pipeline wait that nothing completes, bounded by limit_ns, beside a
// real staged copy that must drain: BCMG_ERR_DEVICE_TIMEOUT (reported through
// sliced_wait_status) when both behave, BCMG_ERR_INTERNAL otherwise.
bcmg_status wait_selftest(unsigned long long limit_ns, cudaStream_t s);

struct MatView {
  int32_t n = 0, nnz = 0;
  const int32_t *row = nullptr, *col = nullptr;
  const void *val = nullptr;
  int vtype = kValF64;
  bool has_sl = false;  // use the sliced copy for sweeps and residuals
  SlicedView sl;
};

// How a relaxation starts: from the iterate in u, from u = 0 (the first
// sweep is f ./ d), or with that first sweep already written by the caller
// into first_sweep_dst(u, u_tmp, k) (fused into the kernel that made f).
enum RelaxStart { kStartLive = 0, kStartZero = 1, kStartFirstDone = 2 };
template <typename XT>
inline XT *first_sweep_dst(XT *u, XT *u_tmp, int k) {
  return (k % 2 == 1) ? u : u_tmp;
}
// Whether a relaxation of k sweeps on A can take kStartFirstDone (levels run
// by one thread-block cluster compute f ./ d themselves).
inline bool first_sweep_fusable(const MatView &A, int k) {
  return k >= 1 && !(A.has_sl && A.sl.cl_size > 0);
}

// k sweeps of u <- ((-(A u) + f) ./ d) + u, result in u; u_tmp is the
// ping-pong buffer; start: a RelaxStart.  XT = double needs FP64 values;
// XT = float takes FP32 / BF16 / FP16 values.  widen_out (XT = float, sliced
// copies without a cluster plan): the last sweep writes its result widened
// into widen_out instead of u.
template <typename XT>
bcmg_status relax_t(const MatView &A, const XT *d, const XT *f, XT *u, XT *u_tmp, int k,
                    int start, cudaStream_t s, double *widen_out = nullptr);
// Whether relax_t can take widen_out for A and k.
inline bool widen_fusable(const MatView &A, int k) {
  return k >= 1 && A.has_sl && A.sl.cl_size == 0 && A.sl.xtype == kValF32;
}
template <typename XT>  // res = f - A u
bcmg_status residual_t(const MatView &A, const XT *f, const XT *u, XT *res, cudaStream_t s);
// relax_t and then res = f - A u, in one launch on a level with a cluster plan.
template <typename XT>
bcmg_status relax_residual_t(const MatView &A, const XT *d, const XT *f, XT *u, XT *u_tmp,
                             int k, int start, XT *res, cudaStream_t s);
template <typename XT>  // y[I] = sum_{i in I} p_i x_i
bcmg_status restrict_t(int32_t nc, const int32_t *rptr, const int32_t *ridx, const XT *p,
                       const XT *x, XT *y, cudaStream_t s);
// restrict_t and the first sweep from zero of the coarse level: u1 = y ./ dc.
template <typename XT>
bcmg_status restrict_first_sweep_t(int32_t nc, const int32_t *rptr, const int32_t *ridx,
                                   const XT *p, const XT *x, XT *y, const XT *dc, XT *u1,
                                   cudaStream_t s);
// out = float(in) and the first sweep from zero u1 = out ./ d.
bcmg_status convert_first_sweep(int64_t n, const double *in, const float *d, float *out,
                                float *u1, cudaStream_t s);
template <typename XT>  // xf[i] += p_i xc[agg_i]
bcmg_status prolong_t(int32_t n, const int32_t *agg, const XT *p, const XT *xc, XT *xf,
                      cudaStream_t s);
template <typename XT>
bcmg_status fill_t(XT *x, int64_t n, XT v, cudaStream_t s);
template <typename XT>  // y = a x + y
bcmg_status axpy_t(int64_t n, XT a, const XT *x, XT *y, cudaStream_t s);
template <typename XT>
bcmg_status scale_t(int64_t n, XT a, XT *x, cudaStream_t s);
template <typename XT>
bcmg_status copy_t(XT *dst, const XT *src, int64_t n, cudaStream_t s);
template <typename XT>  // y = A x
bcmg_status spmv_t(const MatView &A, const XT *x, XT *y, cudaStream_t s);
template <typename XT>  // *out (device) = a . b, accumulated in FP64 in a fixed order
bcmg_status dot_t(int64_t n, const XT *a, const XT *b, double *out, double *partials,
                  cudaStream_t s);
bcmg_status convert_d2f(int64_t n, const double *in, float *out, cudaStream_t s);
bcmg_status convert_f2d(int64_t n, const float *in, double *out, cudaStream_t s);
// FP64 values to FP32 / BF16 / FP16 storage (vtype).
bcmg_status convert_values(int64_t n, const double *in, void *out, int vtype, cudaStream_t s);

inline MatView mat_f64(const CsrView &A) {
  MatView m;
  m.n = A.n;
  m.nnz = A.nnz;
  m.row = A.row;
  m.col = A.col;
  m.val = A.val;
  m.vtype = kValF64;
  return m;
}
// A's structure with FP32 values val32.
inline MatView mat_f32(const CsrView &A, const float *val32) {
  MatView m = mat_f64(A);
  m.val = val32;
  m.vtype = kValF32;
  return m;
}
inline bcmg_status fill(double *x, int64_t n, double v, cudaStream_t s) {
  return fill_t<double>(x, n, v, s);
}
inline bcmg_status copy(double *dst, const double *src, int64_t n, cudaStream_t s) {
  return copy_t<double>(dst, src, n, s);
}
inline bcmg_status axpy(int64_t n, double a, const double *x, double *y, cudaStream_t s) {
  return axpy_t<double>(n, a, x, y, s);
}
inline bcmg_status scale(int64_t n, double a, double *x, cudaStream_t s) {
  return scale_t<double>(n, a, x, s);
}

// ---- FCG (k_solve.cu) ------------------------------------------------------
// Structural check of a device CSR matrix (row pointers, columns in range and
// strictly increasing, finite values, a diagonal in every row); synchronises s
// and returns BCMG_ERR_INVALID_MATRIX naming the first offending row.
enum CsrFault { kCsrBadRow = 1, kCsrBadColumn, kCsrUnsorted, kCsrNonFinite, kCsrNoDiagonal };
bcmg_status csr_validate(const CsrView &A, cudaStream_t s);
// The same checks for an n x m matrix with no diagonal required (a
// prolongator read from a hierarchy file).
bcmg_status csr_validate_rect(const CsrView &A, int32_t m, cudaStream_t s);

// y = alpha A x + beta y (FP64)
bcmg_status spmv(const CsrView &A, double alpha, const double *x, double beta,
                 double *y, cudaStream_t s);

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
  kBnorm, kIndef, kIter, kTarget, kItnlim, kReplace, kNumScal
};
// w = A v fused with alpha = r.v, beta = w.v, gamma = q.v (q may be null).
bcmg_status fcg_spmv_dots(const CsrView &A, const double *v, double *w,
                          const double *r, const double *q, double *partials,
                          double *scal, cudaStream_t s);
// first==true: delta = beta, theta = alpha / delta; else FCG v3 recurrences.
bcmg_status fcg_scalars(double *partials, double *scal, bool first, cudaStream_t s);
// first step: x += theta z; r -= theta az; zp = z; azp = az; norm.
// loop step:  zp = -theta zp + z; x += theta2 zp; azp = -theta azp + az;
//             r -= theta2 azp; norm.
bcmg_status fcg_update(int64_t n, bool first, const double *z, double *zp,
                       const double *az, double *azp, double *x, double *r,
                       double *partials, double *scal, cudaStream_t s);
// Residual replacement: if iteration kIter+1 is a multiple of `every` or the
// recursive norm reached the target, r = b - A x and ||r|| recomputed (FP64).
// With S (an FP64-vector sliced copy of A) the product runs on it.
bcmg_status fcg_replace(const CsrView &A, const SlicedView *S, const double *b, const double *x,
                        double *r, double *partials, double *scal, int every, cudaStream_t s);
// r = b - A x and the ||r||^2 partials on the sliced copy when scal[kReplace]
// is set (fcg_replace).
bcmg_status sliced_replace(const SlicedView &S, const double *b, const double *x, double *r,
                           double *partials, const double *scal, cudaStream_t s);
// Counts the iteration and evaluates the loop condition (into the graph's
// WHILE condition when use_cond).
bcmg_status fcg_continue(double *scal, cudaGraphConditionalHandle cond, bool use_cond,
                         cudaStream_t s);

}  // namespace bcmg
