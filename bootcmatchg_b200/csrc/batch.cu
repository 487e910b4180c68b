// Multi-right-hand-side solves: up to 32 right-hand sides share one
// hierarchy.  The cycle (GAMG_cycle, src/SOLVER/GAMG_cycle.cu:25-140) and the
// composite preconditioner (preconditionApply, src/SOLVER/FCG.cu:112-187) run
// once per iteration for all columns on interleaved blocks, and FCG
// (flexibileConjugateGradients_v3, src/SOLVER/FCG.cu:433-585) keeps one set of
// FP64 scalars per column: a column stops when it converges, hits itnlim or
// breaks down, and the loop (one CUDA graph with a WHILE node) ends when no
// column is left.  Each column follows the single-vector recurrences
// exactly; only the cycle's value storage (FP64 or the mixed-precision
// copies) is shared with bcmg_solve.
//
// Row-kernel shapes of the cycle (columns per lane, block size) are chosen
// per level by timing the candidates once per batch width (ext.autotune), or
// by a fixed rule; every shape gives the same bits.  The FCG SpMV keeps a
// fixed shape: its fused per-column dot products are partitioned by the
// shape, so changing it would change their rounding.
#include <algorithm>
#include <cfloat>
#include <chrono>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
#include <type_traits>
#include <vector>

#include "batch.h"
#include "common.cuh"
#include "handle.h"

namespace bcmg {

struct BatchState {
  int W = 0;
  CycleBufs<double> c64;
  CycleBufs<float> c32;
  // FCG blocks (n x W, FP64, interleaved).
  double *r = nullptr, *v = nullptr, *w = nullptr, *d = nullptr, *q = nullptr, *b = nullptr,
         *x = nullptr, *tmp = nullptr;
  double *partials = nullptr, *scal = nullptr, *colnorm = nullptr;
  int *flags = nullptr;
  std::vector<std::vector<BtCfg>> cfg;  // [hierarchy][level]: cycle row kernels
  BtCfg fcg;                            // level-0 FP64 SpMM of FCG (fixed)
  std::vector<double> host_scal;
  cudaGraphExec_t exec = nullptr;
  double tune_ms = 0.0;
};

namespace {

template <typename XT>
struct BtLv;
template <>
struct BtLv<double> {
  static MatView mat(const DevLevel &l) { return mat_f64(l.view()); }
  static const double *D(const DevLevel &l) { return l.D; }
  static const double *M(const DevLevel &l) { return l.M; }
  static const double *p(const DevLevel &l) { return l.p; }
  // smoothed aggregation: P and R = P^T as CSR
  static MatView P(const DevLevel &l) { return mat_f64(l.pview()); }
  static MatView R(const DevLevel &l) { return mat_f64(l.rview()); }
};
template <>
struct BtLv<float> {
  static MatView mat(const DevLevel &l) {
    MatView m;
    m.n = l.n;
    m.nnz = l.nnz;
    m.row = l.row;
    m.col = l.col;
    m.val = l.val_lo;
    m.vtype = l.vtype_lo;
    return m;
  }
  static const float *D(const DevLevel &l) { return l.D32; }
  static const float *M(const DevLevel &l) { return l.M32; }
  static const float *p(const DevLevel &l) { return l.p32; }
  static MatView P(const DevLevel &l) { return mat_f32(l.pview(), l.Pval32); }
  static MatView R(const DevLevel &l) { return mat_f32(l.rview(), l.Rval32); }
};

template <typename XT>
bcmg_status alloc_bufs(bcmg_handle *h, CycleBufs<XT> &B, int W) {
  cudaStream_t s = h->stream;
  size_t L = 0;
  for (auto &H : h->H) L = std::max(L, H.lv.size());
  B.rhs.assign(L, nullptr);
  B.x.assign(L, nullptr);
  B.xt.assign(L, nullptr);
  B.res.assign(L, nullptr);
  B.n.assign(L, 0);
  for (size_t l = 0; l < L; ++l) {
    int32_t nmax = 0;
    for (auto &H : h->H)
      if (l < H.lv.size()) nmax = std::max(nmax, H.lv[l].n);
    const int64_t cnt = static_cast<int64_t>(nmax) * W;
    if (l > 0) {
      BCMG_TRY(dev_alloc(&B.rhs[l], cnt, s));
      BCMG_TRY(dev_alloc(&B.x[l], cnt, s));
    }
    BCMG_TRY(dev_alloc(&B.xt[l], cnt, s));
    BCMG_TRY(dev_alloc(&B.res[l], cnt, s));
    B.n[l] = nmax;
  }
  const int64_t n0 = static_cast<int64_t>(h->A0.n) * W;
  if (h->prm.solver_type == 2) {
    BCMG_TRY(dev_alloc(&B.xk, n0, s));
    BCMG_TRY(dev_alloc(&B.xadd, n0, s));
  }
  if (std::is_same<XT, float>::value) {
    BCMG_TRY(dev_alloc(&B.in0, n0, s));
    BCMG_TRY(dev_alloc(&B.out0, n0, s));
  }
  return BCMG_OK;
}

template <typename XT>
void free_bufs(CycleBufs<XT> &B, cudaStream_t s) {
  for (size_t l = 0; l < B.xt.size(); ++l) {
    if (l > 0) {
      dev_free(B.rhs[l], s);
      dev_free(B.x[l], s);
    }
    dev_free(B.xt[l], s);
    dev_free(B.res[l], s);
  }
  B.rhs.clear();
  B.x.clear();
  B.xt.clear();
  B.res.clear();
  B.n.clear();
  dev_free(B.xk, s);
  dev_free(B.xadd, s);
  dev_free(B.in0, s);
  dev_free(B.out0, s);
}

void release_state(BatchState *S, cudaStream_t s) {
  if (!S) return;
  if (S->exec) cudaGraphExecDestroy(S->exec);
  free_bufs(S->c64, s);
  free_bufs(S->c32, s);
  for (double **p : {&S->r, &S->v, &S->w, &S->d, &S->q, &S->b, &S->x, &S->tmp, &S->partials,
                     &S->scal, &S->colnorm})
    dev_free(*p, s);
  dev_free(S->flags, s);
  delete S;
}

// The fixed shape rule: the widest access of at most 16 bytes per lane.
BtCfg default_cfg(int W, size_t xbytes) {
  BtCfg c;
  c.V = std::min<int>(W, static_cast<int>(16 / xbytes));
  c.threads = 256;
  return c;
}

// Candidate shapes for a W-column block of XT.
std::vector<BtCfg> candidates(int W, size_t xbytes) {
  std::vector<BtCfg> out;
  for (int V = 1; V <= W && V * static_cast<int>(xbytes) <= 16; V *= 2)
    for (int t : {128, 256}) out.push_back(BtCfg{V, t});
  return out;
}

// Times two relaxation sweeps (u -> out -> u, no copy) of every candidate
// shape on a level (inputs are zero-filled work blocks) and keeps the fastest.
template <typename XT>
bcmg_status tune_level(bcmg_handle *h, const MatView &A, const XT *d, XT *f, XT *u, XT *out,
                       int W, BtCfg *best) {
  cudaStream_t s = h->stream;
  const auto cands = candidates(W, sizeof(XT));
  cudaEvent_t e0, e1;
  BCMG_CUDA(cudaEventCreate(&e0));
  BCMG_CUDA(cudaEventCreate(&e1));
  float best_ms = 1e30f;
  bcmg_status st = BCMG_OK;
  for (const BtCfg &c : cands) {
    // One untimed pass, then the best of three.
    st = bt_relax<XT>(A, W, c, d, f, u, out, 2, false, s);
    if (st != BCMG_OK) break;
    for (int rep = 0; rep < 3 && st == BCMG_OK; ++rep) {
      cudaEventRecord(e0, s);
      st = bt_relax<XT>(A, W, c, d, f, u, out, 2, false, s);
      cudaEventRecord(e1, s);
      if (cudaEventSynchronize(e1) != cudaSuccess) {
        st = set_error(BCMG_ERR_CUDA, "autotune timing failed");
        break;
      }
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      if (ms < best_ms) {
        best_ms = ms;
        *best = c;
      }
    }
    if (st != BCMG_OK) break;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return st;
}

// Tuned shapes by (rows, entries, value type, vector bytes, width), kept for
// the process: a level of the same shape (a repeated matrix, a server's next
// request) takes the earlier choice instead of timing the candidates again.
struct TuneKey {
  int32_t n, nnz;
  int vtype, xbytes, W;
  bool operator<(const TuneKey &o) const {
    return std::tie(n, nnz, vtype, xbytes, W) < std::tie(o.n, o.nnz, o.vtype, o.xbytes, o.W);
  }
};
std::mutex g_tune_mu;
std::map<TuneKey, BtCfg> g_tuned;

template <typename XT>
bcmg_status tune_all(bcmg_handle *h, BatchState &S, CycleBufs<XT> &B) {
  const int W = S.W;
  cudaStream_t s = h->stream;
  for (size_t k = 0; k < h->H.size(); ++k) {
    DevHierarchy &H = h->H[k];
    for (size_t l = 0; l < H.lv.size(); ++l) {
      DevLevel &lv = H.lv[l];
      const TuneKey key{lv.n, lv.nnz, BtLv<XT>::mat(lv).vtype, static_cast<int>(sizeof(XT)), W};
      {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        auto it = g_tuned.find(key);
        if (it != g_tuned.end()) {
          S.cfg[k][l] = it->second;
          continue;
        }
      }
      const int64_t cnt = static_cast<int64_t>(lv.n) * W;
      XT *f = l == 0 ? B.res[0] : B.rhs[l];
      XT *u = l == 0 ? B.xt[0] : B.x[l];
      // Tuning needs three blocks: f, u and the output; level 0 borrows res
      // and xt and writes into the FP64 tmp block (reinterpreted: it is at
      // least as large).
      XT *out = l == 0 ? reinterpret_cast<XT *>(S.tmp) : B.xt[l];
      BCMG_TRY(fill_t<XT>(f, cnt, XT(0), s));
      BCMG_TRY(fill_t<XT>(u, cnt, XT(0), s));
      const XT *d = BtLv<XT>::M(lv) ? BtLv<XT>::M(lv) : BtLv<XT>::D(lv);
      BCMG_TRY(tune_level<XT>(h, BtLv<XT>::mat(lv), d, f, u, out, W, &S.cfg[k][l]));
      std::lock_guard<std::mutex> lk(g_tune_mu);
      g_tuned[key] = S.cfg[k][l];
    }
  }
  return BCMG_OK;
}

bcmg_status create_state(bcmg_handle *h, int W) {
  const auto t0 = std::chrono::steady_clock::now();
  cudaStream_t s = h->stream;
  auto *S = new BatchState();
  S->W = W;
  h->batch = S;
  const int64_t cnt = static_cast<int64_t>(h->A0.n) * W;
  for (double **p : {&S->r, &S->v, &S->w, &S->d, &S->q, &S->b, &S->x, &S->tmp})
    BCMG_TRY(dev_alloc(p, cnt, s));
  BCMG_TRY(dev_alloc(&S->partials, static_cast<int64_t>(kRedBlocks) * 4 * W, s));
  BCMG_TRY(dev_alloc(&S->scal, static_cast<int64_t>(W) * kBtStride, s));
  BCMG_TRY(dev_alloc(&S->colnorm, W, s));
  BCMG_TRY(dev_alloc(&S->flags, 4, s));
  BCMG_CUDA(cudaMemsetAsync(S->scal, 0, sizeof(double) * W * kBtStride, s));
  BCMG_CUDA(cudaMemsetAsync(S->flags, 0, sizeof(int) * 4, s));
  S->host_scal.assign(static_cast<size_t>(W) * kBtStride, 0.0);
  const bool mixed = h->mixed;
  const size_t xbytes = mixed ? sizeof(float) : sizeof(double);
  S->cfg.resize(h->H.size());
  for (size_t k = 0; k < h->H.size(); ++k)
    S->cfg[k].assign(h->H[k].lv.size(), default_cfg(W, xbytes));
  S->fcg = default_cfg(W, sizeof(double));
  if (mixed)
    BCMG_TRY(alloc_bufs<float>(h, S->c32, W));
  else
    BCMG_TRY(alloc_bufs<double>(h, S->c64, W));
  if (h->ext.autotune) {
    if (mixed)
      BCMG_TRY(tune_all<float>(h, *S, S->c32));
    else
      BCMG_TRY(tune_all<double>(h, *S, S->c64));
  }
  BCMG_CUDA(cudaStreamSynchronize(s));
  S->tune_ms =
      std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  return BCMG_OK;
}

// GAMG_cycle on W columns; l is 1-based.  zero[l-1]: the level's iterate is
// identically zero and not materialised.
template <typename XT>
bcmg_status bt_cycle(bcmg_handle *h, BatchState &S, CycleBufs<XT> &B, int k, int l,
                     std::vector<char> &zero) {
  DevHierarchy &H = h->H[k];
  const int L = static_cast<int>(H.lv.size());
  const bcmg_params &p = h->prm;
  cudaStream_t s = h->stream;
  const int W = S.W;
  DevLevel &lv = H.lv[l - 1];
  const MatView A = BtLv<XT>::mat(lv);
  const BtCfg cfg = S.cfg[k][l - 1];
  if (l == L) {
    const XT *d = p.coarse_solver == 0 ? BtLv<XT>::D(lv) : BtLv<XT>::M(lv);
    BCMG_TRY(bt_relax<XT>(A, W, cfg, d, B.rhs[l - 1], B.x[l - 1], B.xt[l - 1],
                          p.relaxnumber_coarse, zero[l - 1] != 0, s));
    zero[l - 1] = 0;
    return BCMG_OK;
  }
  const XT *d = p.relax_type == 0 ? BtLv<XT>::D(lv) : BtLv<XT>::M(lv);
  BCMG_TRY(bt_relax<XT>(A, W, cfg, d, B.rhs[l - 1], B.x[l - 1], B.xt[l - 1], p.prerelax_sweeps,
                        zero[l - 1] != 0, s));
  zero[l - 1] = 0;
  BCMG_TRY(bt_residual<XT>(A, W, cfg, B.rhs[l - 1], B.x[l - 1], B.res[l - 1], s));
  if (lv.Prow)  // smoothed aggregation: rhs_c = R res
    BCMG_TRY(bt_spmm<XT>(BtLv<XT>::R(lv), W, cfg, B.res[l - 1], B.rhs[l], s));
  else
    BCMG_TRY(bt_restrict<XT>(lv.nc, lv.rptr, lv.ridx, BtLv<XT>::p(lv), B.res[l - 1], B.rhs[l],
                             W, s));
  zero[l] = 1;
  for (int i = 1; i <= h->grid_sweeps[l - 1]; ++i) {
    BCMG_TRY(bt_cycle<XT>(h, S, B, k, l + 1, zero));
    if (l == L - 1) break;
  }
  if (lv.Prow) {  // x += P x_c
    BCMG_TRY(bt_spmm<XT>(BtLv<XT>::P(lv), W, cfg, B.x[l], B.xt[l - 1], s));
    BCMG_TRY(axpy_t<XT>(static_cast<int64_t>(lv.n) * W, XT(1), B.xt[l - 1], B.x[l - 1], s));
  } else {
    BCMG_TRY(bt_prolong<XT>(lv.n, lv.agg, BtLv<XT>::p(lv), B.x[l], B.x[l - 1], W, s));
  }
  BCMG_TRY(bt_relax<XT>(A, W, cfg, d, B.rhs[l - 1], B.x[l - 1], B.xt[l - 1],
                        p.postrelax_sweeps, false, s));
  return BCMG_OK;
}

template <typename XT>
bcmg_status bt_run_cycle(bcmg_handle *h, BatchState &S, CycleBufs<XT> &B, int k, const XT *rhs,
                         XT *x, bool x_zero) {
  B.rhs[0] = const_cast<XT *>(rhs);
  B.x[0] = x;
  std::vector<char> zero(B.rhs.size(), 0);
  zero[0] = x_zero ? 1 : 0;
  bcmg_status st = bt_cycle<XT>(h, S, B, k, 1, zero);
  B.rhs[0] = nullptr;
  B.x[0] = nullptr;
  return st;
}

// preconditionApply on W columns (multiplicative, symmetrized, additive).
template <typename XT>
bcmg_status bt_precond_t(bcmg_handle *h, BatchState &S, CycleBufs<XT> &B, const XT *rhs, XT *x,
                         bool x_zero) {
  const int nh = static_cast<int>(h->H.size());
  const int64_t cnt = static_cast<int64_t>(h->A0.n) * S.W;
  cudaStream_t s = h->stream;
  if (h->prm.solver_type == 0) {
    for (int k = 0; k < nh; ++k)
      BCMG_TRY(bt_run_cycle<XT>(h, S, B, k, rhs, x, x_zero && k == 0));
  } else if (h->prm.solver_type == 1) {
    for (int k = 0; k < nh; ++k)
      BCMG_TRY(bt_run_cycle<XT>(h, S, B, k, rhs, x, x_zero && k == 0));
    for (int k = nh - 1; k >= 0; --k) BCMG_TRY(bt_run_cycle<XT>(h, S, B, k, rhs, x, false));
  } else {
    BCMG_TRY(fill_t<XT>(B.xadd, cnt, XT(0), s));
    for (int k = 0; k < nh; ++k) {
      if (x_zero) {
        BCMG_TRY(bt_run_cycle<XT>(h, S, B, k, rhs, B.xk, true));
      } else {
        BCMG_TRY(copy_t<XT>(B.xk, x, cnt, s));
        BCMG_TRY(bt_run_cycle<XT>(h, S, B, k, rhs, B.xk, false));
      }
      BCMG_TRY(axpy_t<XT>(cnt, XT(1), B.xk, B.xadd, s));
    }
    BCMG_TRY(scale_t<XT>(cnt, XT(1) / static_cast<XT>(nh), B.xadd, s));
    BCMG_TRY(copy_t<XT>(x, B.xadd, cnt, s));
  }
  return BCMG_OK;
}

// z = B r on FP64 blocks; the mixed-precision handle runs the FP32 cycle.
bcmg_status bt_precond(bcmg_handle *h, BatchState &S, const double *rhs, double *x,
                       bool x_zero) {
  if (!h->mixed) return bt_precond_t<double>(h, S, S.c64, rhs, x, x_zero);
  const int64_t cnt = static_cast<int64_t>(h->A0.n) * S.W;
  cudaStream_t s = h->stream;
  CycleBufs<float> &B = S.c32;
  BCMG_TRY(convert_d2f(cnt, rhs, B.in0, s));
  if (!x_zero) BCMG_TRY(convert_d2f(cnt, x, B.out0, s));
  BCMG_TRY(bt_precond_t<float>(h, S, B, B.in0, B.out0, x_zero));
  BCMG_TRY(convert_f2d(cnt, B.out0, x, s));
  return BCMG_OK;
}

// One FCG iteration for all columns (the do-while body of FCG.cu:497-565).
bcmg_status bt_iteration(bcmg_handle *h, BatchState &S, cudaGraphConditionalHandle cond,
                         bool use_cond) {
  cudaStream_t s = h->stream;
  const CsrView A = h->A0.view();
  const int W = S.W;
  BCMG_TRY(bt_precond(h, S, S.r, S.v, true));
  BCMG_TRY(bt_fcg_spmv_dots(A, W, S.fcg, S.v, S.w, S.r, S.q, S.partials, s));
  BCMG_TRY(bt_fcg_scalars(S.partials, S.scal, W, false, s));
  BCMG_TRY(bt_fcg_update(A.n, W, false, S.v, S.d, S.w, S.q, S.x, S.r, S.partials, S.scal, s));
  if (h->ext.replace_every > 0)
    BCMG_TRY(bt_fcg_replace(A, W, S.fcg, S.b, S.x, S.r, S.partials, S.scal, S.flags,
                            h->ext.replace_every, s));
  BCMG_TRY(bt_fcg_continue(S.scal, W, S.flags, cond, use_cond, s));
  return BCMG_OK;
}

// FCG on the W columns of S.b with initial guesses S.x (solutions out);
// infos[c] for the first m columns.
bcmg_status bt_fcg(bcmg_handle *h, BatchState &S, int m, bcmg_solve_info *infos,
                   int *indefinite_col) {
  const int32_t n = h->A0.n;
  const int W = S.W;
  cudaStream_t s = h->stream;
  const CsrView A = h->A0.view();
  *indefinite_col = -1;
  // r = b - A x0; per-column delta0, ||b||, targets, active masks.
  BCMG_TRY(bt_residual<double>(mat_f64(A), W, S.fcg, S.b, S.x, S.r, s));
  BCMG_TRY(bt_fcg_init(n, W, S.r, S.b, h->prm.rtol, h->prm.itnlim, S.partials, S.scal, S.flags,
                       s));
  // First step (FCG.cu:464-495) for the active columns.
  BCMG_TRY(bt_precond(h, S, S.r, S.v, true));
  BCMG_TRY(bt_fcg_spmv_dots(A, W, S.fcg, S.v, S.w, S.r, nullptr, S.partials, s));
  BCMG_TRY(bt_fcg_scalars(S.partials, S.scal, W, true, s));
  BCMG_TRY(bt_fcg_update(n, W, true, S.v, S.d, S.w, S.q, S.x, S.r, S.partials, S.scal, s));
  const bool graphs = h->ext.use_graphs && h->stream != nullptr;
  if (graphs && !S.exec) {
    if (capture_while_loop(
            s, [h, &S](cudaGraphConditionalHandle c) { return bt_iteration(h, S, c, true); },
            &S.exec) != BCMG_OK) {
      clear_error();
      S.exec = nullptr;
    }
  }
  if (graphs && S.exec) {
    BCMG_CUDA(cudaGraphLaunch(S.exec, s));
  } else {
    int any = 1;
    while (any) {
      BCMG_TRY(bt_iteration(h, S, 0, false));
      BCMG_CUDA(cudaMemcpyAsync(&any, S.flags, sizeof(int), cudaMemcpyDeviceToHost, s));
      BCMG_CUDA(cudaStreamSynchronize(s));
    }
  }
  // True residual in FP64 per column.
  BCMG_TRY(bt_residual<double>(mat_f64(A), W, S.fcg, S.b, S.x, S.tmp, s));
  BCMG_TRY(bt_col_norms(n, W, S.tmp, S.partials, S.colnorm, s));
  std::vector<double> tr(W);
  BCMG_CUDA(cudaMemcpyAsync(S.host_scal.data(), S.scal, sizeof(double) * W * kBtStride,
                            cudaMemcpyDeviceToHost, s));
  BCMG_CUDA(cudaMemcpyAsync(tr.data(), S.colnorm, sizeof(double) * W, cudaMemcpyDeviceToHost, s));
  BCMG_CUDA(cudaStreamSynchronize(s));
  for (int c = 0; c < m; ++c) {
    const double *hs = S.host_scal.data() + static_cast<size_t>(c) * kBtStride;
    bcmg_solve_info &info = infos[c];
    const double delta0 = hs[kDelta0];
    if (delta0 <= DBL_EPSILON * hs[kBnorm]) {
      info.iters = 0;
      info.converged = 1;
      info.residual = delta0;
      info.rel_residual = 0.0;
      info.true_rel_residual = 0.0;
      continue;
    }
    info.iters = static_cast<int>(hs[kIter]) + 1;  // FCG.cu:569
    info.residual = hs[kNorm];
    info.rel_residual = hs[kNorm] / delta0;
    info.converged = hs[kNorm] <= hs[kTarget] ? 1 : 0;
    info.true_rel_residual = tr[c] / delta0;
    if (hs[kIndef] != 0.0 && *indefinite_col < 0) *indefinite_col = c;
  }
  return BCMG_OK;
}

int batch_width(int nrhs) {
  int W = 1;
  while (W < nrhs && W < kBatchMax) W *= 2;
  return W;
}

bcmg_status ensure_state(bcmg_handle *h, int W) {
  if (h->batch && h->batch->W == W) return BCMG_OK;
  destroy_batch(h);
  bcmg_status st = create_state(h, W);
  if (st != BCMG_OK) destroy_batch(h);
  return st;
}

}  // namespace

size_t batch_bytes(const bcmg_handle *h) {
  if (!h || !h->batch) return 0;
  const BatchState &S = *h->batch;
  const size_t n = static_cast<size_t>(h->A0.n), W = static_cast<size_t>(S.W);
  return 8 * 8 * n * W + 8 * (4 * static_cast<size_t>(kRedBlocks) * W + W * kBtStride + W) +
         cycle_bytes(S.c64, n, W) + cycle_bytes(S.c32, n, W);
}

void destroy_batch(bcmg_handle *h) {
  if (!h || !h->batch) return;
  release_state(h->batch, h->stream);
  h->batch = nullptr;
}

}  // namespace bcmg

using namespace bcmg;

extern "C" {

bcmg_status bcmg_solve_batch(bcmg_handle *h, int32_t nrhs, const double *B, int64_t ldb,
                             double *X, int64_t ldx, int on_device, bcmg_solve_info *infos) {
  clear_error();
  if (!h || !B || !X || nrhs <= 0) return set_error(BCMG_ERR_PARAM, "bad arguments");
  if (h->prm.cycle_type == 3)
    return set_error(BCMG_ERR_UNSUPPORTED, "batched solves do not run the K-cycle");
  const int32_t n = h->A0.n;
  if (ldb < n || ldx < n)
    return set_error(BCMG_ERR_PARAM, "leading dimensions must be >= n (%d)", n);
  BCMG_CUDA(cudaSetDevice(h->device));
  const int W = batch_width(nrhs);
  BCMG_TRY(ensure_state(h, W));
  BatchState &S = *h->batch;
  cudaStream_t s = h->stream;
  std::vector<bcmg_solve_info> local(static_cast<size_t>(nrhs));
  bcmg_status result = BCMG_OK;
  int first_indef = -1;
  for (int32_t c0 = 0; c0 < nrhs; c0 += W) {
    const int m = std::min<int32_t>(W, nrhs - c0);
    const auto tc = std::chrono::steady_clock::now();
    const double *Bc = B + static_cast<int64_t>(c0) * ldb;
    double *Xc = X + static_cast<int64_t>(c0) * ldx;
    if (on_device) {
      BCMG_TRY(bt_pack(n, m, Bc, ldb, S.b, W, s));
      BCMG_TRY(bt_pack(n, m, Xc, ldx, S.x, W, s));
    } else {
      // Host columns go through the tmp block (column-major, leading
      // dimension n) and are interleaved on the device.
      BCMG_CUDA(cudaMemcpy2DAsync(S.tmp, sizeof(double) * n, Bc, sizeof(double) * ldb,
                                  sizeof(double) * n, m, cudaMemcpyHostToDevice, s));
      BCMG_TRY(bt_pack(n, m, S.tmp, n, S.b, W, s));
      BCMG_CUDA(cudaMemcpy2DAsync(S.tmp, sizeof(double) * n, Xc, sizeof(double) * ldx,
                                  sizeof(double) * n, m, cudaMemcpyHostToDevice, s));
      BCMG_TRY(bt_pack(n, m, S.tmp, n, S.x, W, s));
    }
    int indef = -1;
    BCMG_TRY(bt_fcg(h, S, m, local.data() + c0, &indef));
    if (on_device) {
      BCMG_TRY(bt_unpack(n, m, S.x, W, Xc, ldx, s));
    } else {
      BCMG_TRY(bt_unpack(n, m, S.x, W, S.tmp, n, s));
      BCMG_CUDA(cudaMemcpy2DAsync(Xc, sizeof(double) * ldx, S.tmp, sizeof(double) * n,
                                  sizeof(double) * n, m, cudaMemcpyDeviceToHost, s));
    }
    BCMG_CUDA(cudaStreamSynchronize(s));
    const double ms =
        std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - tc).count();
    for (int c = 0; c < m; ++c) {
      bcmg_solve_info &info = local[c0 + c];
      info.solve_ms = ms;
      info.setup_ms = h->setup_ms;
      info.num_hrc = static_cast<int>(h->H.size());
      info.estimated_ratio = h->estimated_ratio;
    }
    if (indef >= 0 && first_indef < 0) first_indef = c0 + indef;
  }
  if (infos) std::memcpy(infos, local.data(), sizeof(bcmg_solve_info) * nrhs);
  if (first_indef >= 0)
    result = set_error(BCMG_ERR_INDEFINITE,
                       "FCG met non-positive curvature on right-hand side %d (A not SPD?)",
                       first_indef);
  return result;
}

bcmg_status bcmg_precond_apply_batch(bcmg_handle *h, int32_t nrhs, const double *d_R,
                                     int64_t ldr, double *d_Z, int64_t ldz) {
  clear_error();
  if (!h || !d_R || !d_Z || nrhs <= 0) return set_error(BCMG_ERR_PARAM, "bad arguments");
  if (h->prm.cycle_type == 3)
    return set_error(BCMG_ERR_UNSUPPORTED, "batched solves do not run the K-cycle");
  const int32_t n = h->A0.n;
  if (ldr < n || ldz < n)
    return set_error(BCMG_ERR_PARAM, "leading dimensions must be >= n (%d)", n);
  BCMG_CUDA(cudaSetDevice(h->device));
  const int W = batch_width(nrhs);
  BCMG_TRY(ensure_state(h, W));
  BatchState &S = *h->batch;
  cudaStream_t s = h->stream;
  for (int32_t c0 = 0; c0 < nrhs; c0 += W) {
    const int m = std::min<int32_t>(W, nrhs - c0);
    BCMG_TRY(bt_pack(n, m, d_R + static_cast<int64_t>(c0) * ldr, ldr, S.r, W, s));
    BCMG_TRY(bt_precond(h, S, S.r, S.v, true));
    BCMG_TRY(bt_unpack(n, m, S.v, W, d_Z + static_cast<int64_t>(c0) * ldz, ldz, s));
  }
  BCMG_CUDA(cudaStreamSynchronize(s));
  return BCMG_OK;
}

bcmg_status bcmg_level_relax_batch(bcmg_handle *h, int hrc, int level, int32_t width,
                                   const void *d_f, void *d_u, int k) {
  clear_error();
  if (!h || !d_f || !d_u || k < 0 || width < 1 || width > kBatchMax || (width & (width - 1)))
    return set_error(BCMG_ERR_PARAM, "bad arguments");
  // The row kernels read up to 16 bytes of a row at once.
  if ((reinterpret_cast<uintptr_t>(d_f) | reinterpret_cast<uintptr_t>(d_u)) % 16)
    return set_error(BCMG_ERR_PARAM, "f and u must be 16-byte aligned");
  if (hrc < 0 || hrc >= static_cast<int>(h->H.size()) || level < 0 ||
      level >= static_cast<int>(h->H[hrc].lv.size()))
    return set_error(BCMG_ERR_PARAM, "no level %d in hierarchy %d", level, hrc);
  BCMG_CUDA(cudaSetDevice(h->device));
  BCMG_TRY(ensure_state(h, width));
  BatchState &S = *h->batch;
  const DevLevel &lv = h->H[hrc].lv[level];
  const BtCfg cfg = S.cfg[hrc][level];
  cudaStream_t s = h->stream;
  if (h->mixed) {
    const float *d = h->prm.relax_type == 0 ? lv.D32 : lv.M32;
    BCMG_TRY(bt_relax<float>(BtLv<float>::mat(lv), width, cfg, d,
                             static_cast<const float *>(d_f), static_cast<float *>(d_u),
                             S.c32.xt[level], k, false, s));
  } else {
    const double *d = h->prm.relax_type == 0 ? lv.D : lv.M;
    BCMG_TRY(bt_relax<double>(BtLv<double>::mat(lv), width, cfg, d,
                              static_cast<const double *>(d_f), static_cast<double *>(d_u),
                              S.c64.xt[level], k, false, s));
  }
  BCMG_CUDA(cudaStreamSynchronize(s));
  return BCMG_OK;
}

bcmg_status bcmg_batch_config(bcmg_handle *h, int32_t nrhs, int hrc, int level,
                              int32_t *width, int32_t *cols_per_lane, int32_t *block_threads,
                              double *tune_ms) {
  clear_error();
  if (!h || nrhs <= 0) return set_error(BCMG_ERR_PARAM, "bad arguments");
  BCMG_CUDA(cudaSetDevice(h->device));
  BCMG_TRY(ensure_state(h, batch_width(nrhs)));
  BatchState &S = *h->batch;
  BtCfg c;
  if (hrc < 0) {
    c = S.fcg;
  } else {
    if (hrc >= static_cast<int>(S.cfg.size()) || level < 0 ||
        level >= static_cast<int>(S.cfg[hrc].size()))
      return set_error(BCMG_ERR_PARAM, "no level %d in hierarchy %d", level, hrc);
    c = S.cfg[hrc][level];
  }
  if (width) *width = S.W;
  if (cols_per_lane) *cols_per_lane = c.V;
  if (block_threads) *block_threads = c.threads;
  if (tune_ms) *tune_ms = S.tune_ms;
  return BCMG_OK;
}

}  // extern "C"
