// Internal definition of bcmg_handle and the device hierarchy.
#pragma once

#include <cuda_runtime.h>

#include <functional>
#include <vector>

#include "bcmg.h"
#include "common.cuh"
#include "kernels.h"

namespace bcmg {

// One level of a hierarchy on the device.  P (to the next level) has one
// entry per fine row: column agg[i], value p[i]; R = P^T is stored as the
// aggregates' member lists in ascending order (rptr, ridx).  The mixed
// precision cycle reads the low-precision copies (val_lo, D32, M32, p32).
struct DevLevel {
  int32_t n = 0, nnz = 0;
  int32_t *row = nullptr, *col = nullptr;
  double *val = nullptr;
  bool own_A = true;
  double *D = nullptr, *M = nullptr, *w = nullptr;
  int32_t nc = 0;
  int32_t *agg = nullptr, *rptr = nullptr, *ridx = nullptr;
  double *p = nullptr;
  void *val_lo = nullptr;
  int vtype_lo = kValF32;
  bool own_lo = true;
  float *D32 = nullptr, *M32 = nullptr, *p32 = nullptr;
  // Smoothed aggregation (aggrtype 1): P (n x nc) and R = P^T as CSR
  // matrices, with FP32 copies of their values for the mixed cycle.  The
  // cycle uses them instead of agg/p/rptr/ridx when Prow is set.
  int32_t *Prow = nullptr, *Pcol = nullptr, *Rrow = nullptr, *Rcol = nullptr;
  double *Pval = nullptr, *Rval = nullptr;
  float *Pval32 = nullptr, *Rval32 = nullptr;
  int32_t Pnnz = 0;
  CsrView pview() const { return CsrView{n, Pnnz, Prow, Pcol, Pval}; }
  CsrView rview() const { return CsrView{nc, Pnnz, Rrow, Rcol, Rval}; }
  // Sliced solve-phase copies (own64/ownlo owned here; s64/slo may point to
  // the handle's level-0 copies).
  SlicedMat own64, ownlo;
  const SlicedMat *s64 = nullptr, *slo = nullptr;
  CsrView view() const {
    CsrView v;
    v.n = n;
    v.nnz = nnz;
    v.row = row;
    v.col = col;
    v.val = val;
    return v;
  }
  void release(cudaStream_t s);
};

struct DevHierarchy {
  std::vector<DevLevel> lv;
  double op_cmplx = 0, op_wcmplx = 0, avg_cratio = 0;
  void release(cudaStream_t s) {
    for (auto &l : lv) l.release(s);
    lv.clear();
  }
};

// Cycle work vectors of one precision, per level, sized by the largest
// hierarchy.  rhs[0]/x[0] are bound to the caller's vectors during an
// application; in0/out0 hold the FP32 images of the FP64 FCG vectors.
template <typename XT>
struct CycleBufs {
  std::vector<XT *> rhs, x, xt, res;
  std::vector<int32_t> n;
  XT *xk = nullptr, *xadd = nullptr, *in0 = nullptr, *out0 = nullptr;
  // When set, the last post-smoothing sweep of level 0 writes its result
  // widened into this FP64 vector instead of x[0] (mixed cycle).
  double *widen_out = nullptr;
  // K-cycle (cycle_type 3) inner iterations, per coarse level: residual w,
  // directions d0/d1, their products v/v1, the correction kx; kdots holds
  // one device dot product.
  std::vector<XT *> kw, kd0, kd1, kv, kv1, kx;
  std::vector<int32_t> kn;  // allocated length of the K-cycle vectors
  double *kdots = nullptr;
  // Device scalars of the K-cycle's inner steps, kKcStride per level, for
  // the captured FCG loop (the host-driven loop reads them through kdots).
  double *kscal = nullptr;
  size_t kscal_levels = 0;
};

// Multi-right-hand-side solve state (batch.cu), created by the first batched
// solve of a handle.
struct BatchState;
void destroy_batch(bcmg_handle *h);
size_t batch_bytes(const bcmg_handle *h);  // device bytes of the batch state

// Builds sliced copies on a helper thread during a setup (driver.cu).
class SideBuilder;

// Device bytes held by a handle (hierarchies, solve copies, work vectors).
size_t handle_bytes(const bcmg_handle *h);
template <typename XT>
size_t cycle_bytes(const CycleBufs<XT> &B, size_t n0, size_t width);

// Captures body(cond) into the body of a WHILE node (initial condition 1) and
// instantiates the graph.
bcmg_status capture_while_loop(cudaStream_t stream,
                               const std::function<bcmg_status(cudaGraphConditionalHandle)> &body,
                               cudaGraphExec_t *out);

}  // namespace bcmg

struct bcmg_handle {
  bcmg_params prm{};
  bcmg_ext ext{};
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  bcmg::DevLevel A0;  // the input matrix; level 0 of every hierarchy points here
  std::vector<bcmg::DevHierarchy> H;
  double estimated_ratio = 1.0;
  int32_t maxcoarsesize = 0;
  std::vector<int> grid_sweeps;
  bool mixed = false;  // solve with the FP32 cycle
  bcmg::CycleBufs<double> c64;
  bcmg::CycleBufs<float> c32;
  // FCG vectors and device scalars.
  double *r = nullptr, *v = nullptr, *w = nullptr, *d = nullptr, *q = nullptr;
  double *b = nullptr, *xs = nullptr, *tmp = nullptr;
  double *partials = nullptr, *scal = nullptr;
  double host_scal[bcmg::kNumScal] = {};  // host mirror of scal
  cudaGraphExec_t fcg_exec = nullptr;   // captured FCG loop (WHILE node)
  // One stream per level to capture the bodies of the K-cycle's IF nodes
  // on (created before the capture, destroyed with the handle).
  std::vector<cudaStream_t> kc_streams;
  bcmg::BatchState *batch = nullptr;    // multi-right-hand-side solves
  // During a setup of a large matrix: the helper that builds solve-phase
  // copies on a stream of its own (null otherwise; owned by the setup).
  bcmg::SideBuilder *side = nullptr;
  double setup_ms = 0.0;
};
