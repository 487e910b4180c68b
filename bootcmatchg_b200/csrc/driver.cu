// Host orchestration of the solve path: bootstrap setup (hierarchy build),
// the V/H/W cycle, the composite preconditioner and flexible CG, plus the
// C ABI entry points that own a bcmg_handle.
//
// Control flow follows the reference step by step (citations inline); the
// arithmetic runs in the kernels of k_setup.cu / k_solve.cu.
#include <algorithm>
#include <cfloat>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <initializer_list>
#include <memory>
#include <mutex>
#include <string>
#include <thread>

#include <nvtx3/nvToolsExt.h>

#include "handle.h"

namespace bcmg {

std::atomic<unsigned long long> g_kernel_launches{0};
std::atomic<long long> g_live_allocs{0};
std::atomic<long long> g_made_allocs{0};
std::atomic<long long> g_fail_alloc_countdown{-1};

// Bound on each wait of a pipelined row pass, from the handle's extensions.
unsigned long long wait_ns_of(const bcmg_handle *h) {
  const double sec = h->ext.max_device_seconds;
  if (!(sec > 0.0)) return kDefaultWaitNs;
  const double ns = sec * 1e9;
  if (ns >= 1.8e19) return ~0ull;
  return ns < 1.0 ? 1ull : static_cast<unsigned long long>(ns);
}

// A sliced solve copy of this handle: its narrowing rule and wait bound.
bcmg_status build_sliced(bcmg_handle *h, const CsrView &A, int vtype, SlicedMat *out,
                         cudaStream_t s) {
  out->wait_ns = wait_ns_of(h);
  return sliced_build(A, vtype, out, s, h->ext.narrow_values != 0);
}

// The copy a queued build fills: level `lvl` of hierarchy `hrc` (own64, or
// ownlo when `lo`), or the input matrix's FP64 copy when hrc < 0.  Kept as
// indices because the hierarchies' level vectors grow while builds run.
struct SliceTarget {
  int hrc = -1, lvl = 0;
  bool lo = false;
};

// Solve-phase copies of the coarse matrices of unsmoothed aggregation are
// built by a helper thread on a stream of its own, each once its level is
// complete, while the handle's stream goes on coarsening.  A coarse copy's
// build is mostly host round trips (it reads its slice statistics back
// before it sizes its arrays), which the helper takes off the setup's
// critical path; its kernels are small.  (The input matrix's copy is not
// built here: its bandwidth-bound passes took the SMs from the matching
// kernels running beside them, which fill every warp slot, about as much
// time as they saved.)  Each build waits for an event recorded on the
// handle's stream when it was queued (its matrix is complete there).  A
// copy becomes part of the hierarchy only at drain(), which waits for every
// queued build and installs the results; drains come before the bootstrap's
// inner iterations and before the solve formats are finished, so every
// kernel that reads a copy sees the state that building them in line gives
// (same copies, same results).  The destructor drains too: on an error path
// the finished copies go to the handle (freed with it) and partial ones are
// released.
class SideBuilder {
 public:
  explicit SideBuilder(bcmg_handle *h) : h_(h) {}
  SideBuilder(const SideBuilder &) = delete;
  SideBuilder &operator=(const SideBuilder &) = delete;
  ~SideBuilder() {
    drain(false);
    {
      std::lock_guard<std::mutex> lk(m_);
      stop_ = true;
    }
    cv_.notify_all();
    if (worker_.joinable()) worker_.join();
    if (stream_) cudaStreamDestroy(stream_);
  }

  bcmg_status enqueue(const CsrView &A, int vtype, SliceTarget t) {
    if (!stream_) {
      BCMG_CUDA(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
      try {
        worker_ = std::thread([this] { run(); });
      } catch (...) {
        cudaStreamDestroy(stream_);
        stream_ = nullptr;
        return set_error(BCMG_ERR_INTERNAL, "cannot start the copy-building thread");
      }
    }
    Item it;
    it.A = A;
    it.vtype = vtype;
    it.t = t;
    it.wait_ns = wait_ns_of(h_);
    it.narrow = h_->ext.narrow_values != 0;
    BCMG_CUDA(cudaEventCreateWithFlags(&it.ready, cudaEventDisableTiming));
    const cudaError_t e = cudaEventRecord(it.ready, h_->stream);
    if (e != cudaSuccess) {
      cudaEventDestroy(it.ready);
      return set_error(BCMG_ERR_CUDA, "cudaEventRecord: %s", cudaGetErrorString(e));
    }
    {
      std::lock_guard<std::mutex> lk(m_);
      items_.push_back(it);
    }
    cv_.notify_all();
    return BCMG_OK;
  }

  // Waits for every queued build and installs the copies; returns the first
  // failure of a build (its message becomes the last error when `report`).
  bcmg_status drain(bool report = true) {
    std::deque<Item> done;
    {
      std::unique_lock<std::mutex> lk(m_);
      idle_.wait(lk, [this] { return next_ == items_.size(); });
      done.swap(items_);
      next_ = 0;
    }
    bcmg_status first = BCMG_OK;
    std::string msg;
    for (Item &it : done) {
      SlicedMat *dst = target(it.t);
      if (it.st == BCMG_OK && dst && !dst->nslices) {
        *dst = it.out;
      } else {
        it.out.release(h_->stream);
        if (it.st != BCMG_OK && first == BCMG_OK) {
          first = it.st;
          msg = it.err;
        }
      }
    }
    // Level 0 of every hierarchy reads the input matrix's copy.
    if (h_->A0.own64.nslices)
      for (auto &H : h_->H)
        if (!H.lv.empty()) H.lv[0].s64 = &h_->A0.own64;
    if (first != BCMG_OK && report) return set_error(first, "%s", msg.c_str());
    return first;
  }

 private:
  struct Item {
    CsrView A;
    int vtype = kValF64;
    SliceTarget t;
    unsigned long long wait_ns = kDefaultWaitNs;
    bool narrow = false;
    cudaEvent_t ready = nullptr;
    SlicedMat out;
    bcmg_status st = BCMG_OK;
    std::string err;
  };

  SlicedMat *target(const SliceTarget &t) {
    if (t.hrc < 0) return &h_->A0.own64;
    if (static_cast<size_t>(t.hrc) >= h_->H.size()) return nullptr;
    auto &lv = h_->H[t.hrc].lv;
    if (static_cast<size_t>(t.lvl) >= lv.size()) return nullptr;
    return t.lo ? &lv[t.lvl].ownlo : &lv[t.lvl].own64;
  }

  bcmg_status build(Item &it) {
    BCMG_CUDA(cudaStreamWaitEvent(stream_, it.ready, 0));
    it.out.wait_ns = it.wait_ns;
    const bcmg_status st = sliced_build(it.A, it.vtype, &it.out, stream_, it.narrow);
    // Also after a failure: drain() releases a partial copy on the handle's
    // stream, so nothing queued here may still be writing it.
    const cudaError_t e = cudaStreamSynchronize(stream_);
    if (st != BCMG_OK) return st;
    if (e != cudaSuccess)
      return set_error(BCMG_ERR_CUDA, "%s", cudaGetErrorString(e));
    return BCMG_OK;
  }

  void run() {
    cudaSetDevice(h_->device);
    std::unique_lock<std::mutex> lk(m_);
    for (;;) {
      cv_.wait(lk, [this] { return stop_ || next_ < items_.size(); });
      if (next_ >= items_.size()) return;  // stop_ with nothing queued
      Item &it = items_[next_];            // deque: stable under push_back
      lk.unlock();
      it.st = build(it);
      if (it.st != BCMG_OK) it.err = bcmg_last_error();
      cudaEventDestroy(it.ready);
      it.ready = nullptr;
      lk.lock();
      ++next_;
      idle_.notify_all();
    }
  }

  bcmg_handle *h_;
  cudaStream_t stream_ = nullptr;
  std::thread worker_;
  std::mutex m_;
  std::condition_variable cv_, idle_;
  std::deque<Item> items_;
  size_t next_ = 0;  // items_[next_] is the next build (all before it done)
  bool stop_ = false;
};

// Rows of the input matrix from which a setup builds its solve copies on the
// helper thread (below this the copies are built in line: too little work to
// pay for the thread).
constexpr int32_t kSideBuildMinRows = 1 << 17;

// The sliced copy of A in *out (the copy named by t), built now on the
// handle's stream or queued on the setup's helper.
bcmg_status sliced_copy(bcmg_handle *h, const CsrView &A, int vtype, SlicedMat *out,
                        SliceTarget t) {
  if (h->side) return h->side->enqueue(A, vtype, t);
  return build_sliced(h, A, vtype, out, h->stream);
}

// Storage of the coarse levels' values in the mixed cycle (ext.coarse_storage).
int coarse_value_type(const bcmg_handle *h) {
  return h->ext.coarse_storage == BCMG_STORE_BF16   ? kValBF16
         : h->ext.coarse_storage == BCMG_STORE_FP16 ? kValF16
                                                    : kValF32;
}

// NVTX range for the lifetime of a scope (profilers filter on these names).
struct NvtxRange {
  explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
};

void DevLevel::release(cudaStream_t s) {
  if (own_A) {
    dev_free(row, s);
    dev_free(col, s);
    dev_free(val, s);
  }
  row = col = nullptr;
  val = nullptr;
  dev_free(D, s);
  dev_free(M, s);
  dev_free(w, s);
  dev_free(agg, s);
  dev_free(rptr, s);
  dev_free(ridx, s);
  dev_free(p, s);
  if (own_lo) dev_free(val_lo, s);
  val_lo = nullptr;
  dev_free(D32, s);
  dev_free(M32, s);
  dev_free(p32, s);
  dev_free(Prow, s);
  dev_free(Pcol, s);
  dev_free(Pval, s);
  dev_free(Rrow, s);
  dev_free(Rcol, s);
  dev_free(Rval, s);
  dev_free(Pval32, s);
  dev_free(Rval32, s);
  Pnnz = 0;
  own64.release(s);
  ownlo.release(s);
  s64 = slo = nullptr;
}

namespace {

constexpr int kFtcoarseInc = 100;     // FTCOARSE_INC, matchingAggregation.cu:12
constexpr double kCoarseRatio = 1.2;  // COARSERATIO_THRSLD, matchingAggregation.cu:13
constexpr int kBootSolverIt = 15;     // solver_it, AMG.cu:407
// Relative reduction at which the K-cycle stops after its first inner step
// (RTOL, src/SOLVER/GAMG_cycle.cu:5).
constexpr double kKcycleRtol = 0.25;
// Device scalars of one level's K-cycle inner steps (CycleBufs::kscal).
constexpr int kKcStride = 16;
enum KcScal {
  kKcWW = 0,    // ||w||^2 before the first step (delta0 = its root)
  kKcDelta,     // w . d0
  kKcTau,       // d0 . v
  kKcWW2,       // ||w||^2 after the first step
  kKcTau1,      // d1 . v
  kKcTau2,      // d1 . v1
  kKcTau3,      // d1 . w
  kKcA0,        // coefficient of d0 in the correction
  kKcA1,        // coefficient of d1
  kKcNegAlpha,  // -alpha, for w -= alpha v
  kKcSecond     // 1: the second inner step ran
};

using Clock = std::chrono::steady_clock;
double ms_since(Clock::time_point t0) {
  return std::chrono::duration<double, std::milli>(Clock::now() - t0).count();
}

// Phase timing report for ext.verbose >= 1: synchronises the stream at each
// phase boundary and accumulates wall time per phase name (stderr).
struct PhaseClock {
  bool on = false;
  cudaStream_t s = nullptr;
  Clock::time_point t;
  std::vector<std::pair<const char *, double>> acc;
  void start(bool enable, cudaStream_t st) {
    on = enable;
    s = st;
    acc.clear();
    if (on) {
      cudaStreamSynchronize(s);
      t = Clock::now();
    }
  }
  void tick(const char *name) {
    if (!on) return;
    cudaStreamSynchronize(s);
    const double ms = ms_since(t);
    t = Clock::now();
    for (auto &a : acc)
      if (a.first == name) {
        a.second += ms;
        return;
      }
    acc.emplace_back(name, ms);
  }
  void report(const char *what) {
    if (!on) return;
    fprintf(stderr, "[bcmg] %s:", what);
    for (auto &a : acc) fprintf(stderr, " %s=%.2fms", a.first, a.second);
    fprintf(stderr, "\n");
  }
};
thread_local PhaseClock g_clock;
}  // namespace

void phase_tick(const char *name) { g_clock.tick(name); }

namespace {

bcmg_status read_scalar(const double *dev, double *host, cudaStream_t s) {
  BCMG_CUDA(cudaMemcpyAsync(host, dev, sizeof(double), cudaMemcpyDeviceToHost, s));
  BCMG_CUDA(cudaStreamSynchronize(s));
  return BCMG_OK;
}

// ||x||_A = sqrt(x' A x) (CSRm::vectorANorm, src/matrix/CSR.cu:360-368).
bcmg_status anorm(bcmg_handle *h, const double *x, double *out) {
  if (h->A0.own64.nslices)
    BCMG_TRY(sliced_spmv(h->A0.own64.view(), x, h->tmp, h->stream));
  else
    BCMG_TRY(spmv(h->A0.view(), 1.0, x, 0.0, h->tmp, h->stream));
  BCMG_TRY(dot_dev(h->A0.n, h->tmp, x, h->scal + kAlpha, h->partials, h->stream));
  double v = 0;
  BCMG_TRY(read_scalar(h->scal + kAlpha, &v, h->stream));
  *out = std::sqrt(v);
  return BCMG_OK;
}

bcmg_status norm2(bcmg_handle *h, const double *x, double *out) {
  BCMG_TRY(dot_dev(h->A0.n, x, x, h->scal + kAlpha, h->partials, h->stream));
  double v = 0;
  BCMG_TRY(read_scalar(h->scal + kAlpha, &v, h->stream));
  *out = std::sqrt(v);
  return BCMG_OK;
}

// Builds the coarse matrix of one level from `fine` with aggrsweeps pairwise
// sweeps (matchingAggregation, src/AMG/matchingAggregation.cu:211-295).  On
// return fine.agg/p/nc/rptr/ridx describe the composed prolongator, *w_out
// holds the coarse smooth vector (newly allocated) and `coarse` the Galerkin
// matrix.  fine.w is the sweep-0 smooth vector and is left untouched.
bcmg_status matching_aggregation(bcmg_handle *h, DevLevel &fine, double **w_out,
                                 int *ftcoarse, DevLevel &coarse) {
  cudaStream_t s = h->stream;
  CsrView cur = fine.view();
  const double *w_in = fine.w;
  double *cur_w = fine.w;
  DevLevel inter;  // intermediate coarse matrix between sweeps
  bool have_inter = false;
  // On an early return the intermediate matrix and smooth vector are freed
  // here; on success they become `coarse` and *w_out.
  struct Scratch {
    DevLevel &inter;
    bool &have_inter;
    double *&cur_w;
    const double *w_in;
    cudaStream_t s;
    bool handed_over = false;
    ~Scratch() {
      if (handed_over) return;
      if (have_inter) inter.release(s);
      if (cur_w != w_in) dev_free(cur_w, s);
    }
  } scratch{inter, have_inter, cur_w, w_in, s};
  DevBuf<int32_t> agg_acc;
  DevBuf<double> p_acc;
  int32_t nc_acc = 0;
  for (int sweep = 0; sweep < h->prm.aggrsweeps; ++sweep) {
    DevBuf<int32_t> agg_i, rptr_i, ridx_i, crow;
    DevBuf<double> p_i, wi;
    int32_t nci = 0;
    BCMG_TRY(agg_i.alloc(cur.n, s));
    BCMG_TRY(p_i.alloc(cur.n, s));
    g_clock.tick("other");
    BCMG_TRY(pair_aggregate(cur, cur_w, agg_i.get(), p_i.get(), &nci, nullptr, nullptr,
                            nullptr, s, h->ext.match_step_limit));
    g_clock.tick("match+aggregate");
    BCMG_TRY(rptr_i.alloc(nci + 1, s));
    BCMG_TRY(ridx_i.alloc(cur.n, s));
    BCMG_TRY(transpose_agg(cur.n, agg_i.get(), nci, rptr_i.get(), ridx_i.get(), s));
    // Galerkin product (matchingAggregation.cu:239-244).
    int32_t cnnz = 0;
    BCMG_TRY(crow.alloc(nci + 1, s));
    int32_t *ccol_raw = nullptr;
    double *cval_raw = nullptr;
    g_clock.tick("transpose");
    BCMG_TRY(galerkin(cur, agg_i.get(), p_i.get(), nci, rptr_i.get(), ridx_i.get(), crow.get(),
                      &ccol_raw, &cval_raw, &cnnz, s));
    g_clock.tick("galerkin");
    DevBuf<int32_t> ccol;
    DevBuf<double> cval;
    ccol.ptr = ccol_raw;
    ccol.stream = s;
    cval.ptr = cval_raw;
    cval.stream = s;
    // w_i = R_i w_{i-1} (matchingAggregation.cu:253).
    BCMG_TRY(wi.alloc(nci, s));
    BCMG_TRY(restrict_exact(nci, rptr_i.get(), ridx_i.get(), p_i.get(), cur_w, wi.get(), s));
    const double size_precoarse = cur.n;
    const double size_coarse = nci;
    const double coarse_ratio = size_precoarse / size_coarse;
    if (sweep == 0) {
      agg_acc = std::move(agg_i);
      p_acc = std::move(p_i);
    } else {
      // P = P P_i (matchingAggregation.cu:264).
      BCMG_TRY(compose_p(fine.n, agg_acc.get(), p_acc.get(), agg_i.get(), p_i.get(), s));
    }
    nc_acc = nci;
    if (have_inter) inter.release(s);
    DevLevel next;
    next.n = nci;
    next.nnz = cnnz;
    next.row = crow.release();
    next.col = ccol.release();
    next.val = cval.release();
    if (cur_w != w_in) dev_free(cur_w, s);
    cur_w = wi.release();
    inter = next;
    have_inter = true;
    if (coarse_ratio <= kCoarseRatio) *ftcoarse = kFtcoarseInc;
    cur = inter.view();
    if (size_coarse <= static_cast<double>(*ftcoarse * h->maxcoarsesize)) break;
  }
  // The sweep input w (the level's smooth vector) is kept by the fine level.
  fine.agg = agg_acc.release();
  fine.p = p_acc.release();
  fine.nc = nc_acc;
  BCMG_TRY(dev_alloc(&fine.rptr, nc_acc + 1, s));
  BCMG_TRY(dev_alloc(&fine.ridx, fine.n, s));
  BCMG_TRY(transpose_agg(fine.n, fine.agg, nc_acc, fine.rptr, fine.ridx, s));
  coarse = inter;
  *w_out = cur_w;
  scratch.handed_over = true;
  return BCMG_OK;
}

// adaptiveCoarsening (src/AMG/matchingAggregation.cu:298-423).
// An FP64 cycle will read the coarse levels: the FP64 solve, or the
// bootstrap's inner iterations.
bool wants_coarse_f64(const bcmg_handle *h) {
  return h->ext.sliced && (h->ext.precision == BCMG_PREC_FP64 || h->prm.max_hrc > 1);
}

// Smoothed aggregation (aggrtype 1), level by level so that D_j is the
// diagonal of the already smoothed A_j: S_j = I - omega D_j^{-1} A_j with
// omega = 4 / (3 ||D_j^{-1} A_j||_inf), P_j = S_j P_tent (P_tent: column
// agg[i], value p[i] per row), R_j = P_j^T, A_{j+1} = (R_j A_j) P_j.  Every
// product sums in the canonical order of spgemm.
bcmg_status smooth_hierarchy(bcmg_handle *h, DevHierarchy &H) {
  cudaStream_t s = h->stream;
  const int L = static_cast<int>(H.lv.size());
  for (int j = 0; j + 1 < L; ++j) {
    DevLevel &lv = H.lv[j];
    const CsrView A = lv.view();
    DevBuf<double> sval;
    DevBuf<int32_t> trow;
    BCMG_TRY(sval.alloc(std::max(A.nnz, 1), s));
    BCMG_TRY(trow.alloc(static_cast<int64_t>(A.n) + 1, s));
    phase_tick("smoothed aggregation");
    BCMG_TRY(smoothing_operator(A, lv.D, sval.get(), s));
    BCMG_TRY(iota(A.n, trow.get(), s));
    phase_tick("sa smoothing");
    const CsrView S{A.n, A.nnz, A.row, A.col, sval.get()};
    const CsrView Pt{A.n, A.n, trow.get(), lv.agg, lv.p};
    BCMG_TRY(dev_alloc(&lv.Prow, static_cast<int64_t>(A.n) + 1, s));
    BCMG_TRY(spgemm(S, Pt, lv.nc, lv.Prow, &lv.Pcol, &lv.Pval, &lv.Pnnz, s));
    BCMG_TRY(dev_alloc(&lv.Rrow, static_cast<int64_t>(lv.nc) + 1, s));
    BCMG_TRY(dev_alloc(&lv.Rcol, std::max(lv.Pnnz, 1), s));
    BCMG_TRY(dev_alloc(&lv.Rval, std::max(lv.Pnnz, 1), s));
    phase_tick("sa P");
    BCMG_TRY(csr_transpose(lv.pview(), lv.nc, lv.Rrow, lv.Rcol, lv.Rval, s));
    phase_tick("sa transpose");
    DevBuf<int32_t> ra_row, ac_row;
    BCMG_TRY(ra_row.alloc(static_cast<int64_t>(lv.nc) + 1, s));
    int32_t *ra_col = nullptr, *ac_col = nullptr;
    double *ra_val = nullptr, *ac_val = nullptr;
    int32_t ra_nnz = 0, ac_nnz = 0;
    BCMG_TRY(spgemm(lv.rview(), A, A.n, ra_row.get(), &ra_col, &ra_val, &ra_nnz, s));
    DevBuf<int32_t> ra_colb;
    DevBuf<double> ra_valb;
    ra_colb.ptr = ra_col;
    ra_colb.stream = s;
    ra_valb.ptr = ra_val;
    ra_valb.stream = s;
    BCMG_TRY(ac_row.alloc(static_cast<int64_t>(lv.nc) + 1, s));
    const CsrView RA{lv.nc, ra_nnz, ra_row.get(), ra_col, ra_val};
    phase_tick("sa RA");
    BCMG_TRY(spgemm(RA, lv.pview(), lv.nc, ac_row.get(), &ac_col, &ac_val, &ac_nnz, s));
    phase_tick("sa RAP");
    DevLevel &c = H.lv[j + 1];
    if (c.own_A) {
      dev_free(c.row, s);
      dev_free(c.col, s);
      dev_free(c.val, s);
    }
    c.row = ac_row.release();
    c.col = ac_col;
    c.val = ac_val;
    c.nnz = ac_nnz;
    c.own_A = true;
    BCMG_TRY(level_prep(c.view(), c.D, c.M, s));
    c.own64.release(s);
    if (wants_coarse_f64(h))
      BCMG_TRY(build_sliced(h, c.view(), kValF64, &c.own64, s));
  }
  phase_tick("smoothed aggregation");
  return BCMG_OK;
}

bcmg_status adaptive_coarsening(bcmg_handle *h, const double *w_in, DevHierarchy &H) {
  cudaStream_t s = h->stream;
  const int maxlevels = h->prm.max_levels;
  // Every level is owned by H before its arrays are allocated, so a failure
  // part-way leaves nothing that H.release would not free.
  H.lv.emplace_back();
  {
    DevLevel &l0 = H.lv.back();
    l0.n = h->A0.n;
    l0.nnz = h->A0.nnz;
    l0.row = h->A0.row;
    l0.col = h->A0.col;
    l0.val = h->A0.val;
    l0.own_A = false;
    if (h->A0.own64.nslices) l0.s64 = &h->A0.own64;
    BCMG_TRY(dev_alloc(&l0.D, l0.n, s));
    BCMG_TRY(dev_alloc(&l0.M, l0.n, s));
    BCMG_TRY(dev_alloc(&l0.w, l0.n, s));
    BCMG_TRY(copy(l0.w, w_in, l0.n, s));
    BCMG_TRY(level_prep(l0.view(), l0.D, l0.M, s));
  }
  double normw = 0;
  BCMG_TRY(anorm(h, w_in, &normw));
  int ftcoarse = 1;
  double avcoarseratio = 0.0;
  int level = 0;
  if (normw > DBL_EPSILON) {
    for (level = 1; level < maxlevels;) {
      double *w = nullptr;
      DevLevel built;
      BCMG_TRY(matching_aggregation(h, H.lv[level - 1], &w, &ftcoarse, built));
      built.w = w;
      const double fine_n = H.lv[level - 1].n;
      H.lv.push_back(built);  // (invalidates references into H.lv)
      DevLevel &coarse = H.lv.back();
      BCMG_TRY(dev_alloc(&coarse.D, coarse.n, s));
      BCMG_TRY(dev_alloc(&coarse.M, coarse.n, s));
      BCMG_TRY(level_prep(coarse.view(), coarse.D, coarse.M, s));
      // FP64 sliced copy now if an FP64 cycle will read this level (the FP64
      // solve, or the bootstrap's inner iterations); with the setup's helper
      // also the mixed cycle's copy, which is otherwise built after the
      // bootstrap.  (Smoothed aggregation replaces the coarse matrices: built
      // afterwards.)
      const SliceTarget t{static_cast<int>(&H - h->H.data()), static_cast<int>(H.lv.size()) - 1,
                          false};
      if (h->prm.aggrtype == 0 && wants_coarse_f64(h))
        BCMG_TRY(sliced_copy(h, coarse.view(), kValF64, &coarse.own64, t));
      if (h->side && h->prm.aggrtype == 0 && h->ext.precision == BCMG_PREC_MIXED)
        BCMG_TRY(h->side->enqueue(coarse.view(), coarse_value_type(h),
                                  SliceTarget{t.hrc, t.lvl, true}));
      const double size_coarse = coarse.n;
      const double coarse_ratio = fine_n / size_coarse;
      avcoarseratio += coarse_ratio;
      ++level;
      if (size_coarse <= static_cast<double>(ftcoarse * h->maxcoarsesize)) break;
    }
  } else {
    // The reference asserts here (finalize_level with 0 levels): keep one
    // level, i.e. a smoother-only preconditioner.
    level = 1;
  }
  if (h->prm.aggrtype == 1) BCMG_TRY(smooth_hierarchy(h, H));
  const double nnz0 = H.lv[0].nnz;
  double c = 0, cw = 0;
  for (size_t i = 0; i < H.lv.size(); ++i) {
    c += H.lv[i].nnz;
    cw += std::pow(2.0, static_cast<double>(i)) * H.lv[i].nnz;
  }
  H.op_cmplx = c / nnz0;
  H.op_wcmplx = cw / nnz0;
  H.avg_cratio = level > 1 ? avcoarseratio / (level - 1) : 0.0;
  BCMG_CUDA(cudaStreamSynchronize(s));
  return BCMG_OK;
}

template <typename XT>
bcmg_status size_buffers_t(bcmg_handle *h, CycleBufs<XT> &B) {
  cudaStream_t s = h->stream;
  size_t L = 0;
  for (auto &H : h->H) L = std::max(L, H.lv.size());
  const size_t old = B.n.size();
  B.rhs.resize(L, nullptr);
  B.x.resize(L, nullptr);
  B.xt.resize(L, nullptr);
  B.res.resize(L, nullptr);
  B.n.resize(L, 0);
  for (size_t l = 0; l < L; ++l) {
    int32_t nmax = 0;
    for (auto &H : h->H)
      if (l < H.lv.size()) nmax = std::max(nmax, H.lv[l].n);
    if (l < old && nmax <= B.n[l]) continue;
    if (l > 0) {
      dev_free(B.rhs[l], s);
      dev_free(B.x[l], s);
      BCMG_TRY(dev_alloc(&B.rhs[l], nmax, s));
      BCMG_TRY(dev_alloc(&B.x[l], nmax, s));
    }
    dev_free(B.xt[l], s);
    dev_free(B.res[l], s);
    BCMG_TRY(dev_alloc(&B.xt[l], nmax, s));
    BCMG_TRY(dev_alloc(&B.res[l], nmax, s));
    B.n[l] = nmax;
  }
  if (h->prm.cycle_type == 3) {
    for (auto *v : {&B.kw, &B.kd0, &B.kd1, &B.kv, &B.kv1, &B.kx}) v->resize(L, nullptr);
    B.kn.resize(L, 0);
    for (size_t l = 1; l < L; ++l) {
      if (B.kw[l] && B.n[l] <= B.kn[l]) continue;
      for (auto *v : {&B.kw, &B.kd0, &B.kd1, &B.kv, &B.kv1, &B.kx}) {
        dev_free((*v)[l], s);
        BCMG_TRY(dev_alloc(&(*v)[l], B.n[l], s));
      }
      B.kn[l] = B.n[l];
    }
    if (!B.kdots) BCMG_TRY(dev_alloc(&B.kdots, 1, s));
    if (B.kscal_levels < L) {
      dev_free(B.kscal, s);
      BCMG_TRY(dev_alloc(&B.kscal, static_cast<int64_t>(L) * kKcStride, s));
      B.kscal_levels = L;
    }
  }
  const int32_t n = h->A0.n;
  if (!B.xk) {
    BCMG_TRY(dev_alloc(&B.xk, n, s));
    BCMG_TRY(dev_alloc(&B.xadd, n, s));
    BCMG_TRY(dev_alloc(&B.in0, n, s));
    BCMG_TRY(dev_alloc(&B.out0, n, s));
  }
  return BCMG_OK;
}

template <typename XT>
void free_buffers_t(CycleBufs<XT> &B, cudaStream_t s) {
  for (size_t l = 0; l < B.xt.size(); ++l) {
    if (l > 0) {
      dev_free(B.rhs[l], s);
      dev_free(B.x[l], s);
    }
    dev_free(B.xt[l], s);
    dev_free(B.res[l], s);
  }
  dev_free(B.xk, s);
  dev_free(B.xadd, s);
  dev_free(B.in0, s);
  dev_free(B.out0, s);
  for (auto *v : {&B.kw, &B.kd0, &B.kd1, &B.kv, &B.kv1, &B.kx})
    for (auto &p : *v) dev_free(p, s);
  dev_free(B.kdots, s);
  dev_free(B.kscal, s);
  B.kscal_levels = 0;
}

// The level data a cycle of vector type XT reads.
template <typename XT>
struct Lv;
// The sliced copies of a level: level 0 points to the handle's shared copy,
// other levels own theirs (resolved here, never stored as a self-pointer,
// since levels live in a growing std::vector).
inline const SlicedMat *sliced64(const DevLevel &l) {
  if (l.s64) return l.s64;
  return l.own64.nslices ? &l.own64 : nullptr;
}
inline const SlicedMat *slicedlo(const DevLevel &l) {
  if (l.slo) return l.slo;
  return l.ownlo.nslices ? &l.ownlo : nullptr;
}

template <>
struct Lv<double> {
  static MatView mat(const DevLevel &l) {
    MatView m = mat_f64(l.view());
    const SlicedMat *S = sliced64(l);
    if (S && S->nslices) {
      m.has_sl = true;
      m.sl = S->view();
    }
    return m;
  }
  static const double *D(const DevLevel &l) { return l.D; }
  static const double *M(const DevLevel &l) { return l.M; }
  static const double *p(const DevLevel &l) { return l.p; }
  static MatView P(const DevLevel &l) { return mat_f64(l.pview()); }
  static MatView R(const DevLevel &l) { return mat_f64(l.rview()); }
};
template <>
struct Lv<float> {
  static MatView mat(const DevLevel &l) {
    MatView m;
    m.n = l.n;
    m.nnz = l.nnz;
    m.row = l.row;
    m.col = l.col;
    m.val = l.val_lo;
    m.vtype = l.vtype_lo;
    const SlicedMat *S = slicedlo(l);
    if (S && S->nslices) {
      m.has_sl = true;
      m.sl = S->view();
    }
    return m;
  }
  static const float *D(const DevLevel &l) { return l.D32; }
  static const float *M(const DevLevel &l) { return l.M32; }
  static const float *p(const DevLevel &l) { return l.p32; }
  static MatView P(const DevLevel &l) { return mat_f32(l.pview(), l.Pval32); }
  static MatView R(const DevLevel &l) { return mat_f32(l.rview(), l.Rval32); }
};

template <typename XT>
bcmg_status kcycle_inner_t(bcmg_handle *h, CycleBufs<XT> &B, int k, int c);

// GAMG_cycle (src/SOLVER/GAMG_cycle.cu:25-140); l is 1-based as there.
// zero[l-1] says the current iterate of level l-1 is identically zero and
// has not been materialised: the first sweep then reduces to f ./ d.
// The first relaxation a cycle runs on level l (1-based) of hierarchy k: its
// sweep count (*sweeps) and diagonal (pre-smoothing, or the coarse solver
// on the last level).
template <typename XT>
const XT *first_relax(const bcmg_handle *h, int k, int l, int *sweeps) {
  const DevHierarchy &H = h->H[k];
  const bcmg_params &p = h->prm;
  const DevLevel &lv = H.lv[l - 1];
  if (l == static_cast<int>(H.lv.size())) {
    *sweeps = p.relaxnumber_coarse;
    return p.coarse_solver == 0 ? Lv<XT>::D(lv) : Lv<XT>::M(lv);
  }
  *sweeps = p.prerelax_sweeps;
  return p.relax_type == 0 ? Lv<XT>::D(lv) : Lv<XT>::M(lv);
}

template <typename XT>
bcmg_status cycle_t(bcmg_handle *h, CycleBufs<XT> &B, int k, int l, std::vector<char> &zero) {
  DevHierarchy &H = h->H[k];
  const int L = static_cast<int>(H.lv.size());
  const bcmg_params &p = h->prm;
  cudaStream_t s = h->stream;
  DevLevel &lv = H.lv[l - 1];
  const MatView A = Lv<XT>::mat(lv);
  if (l == L) {
    const XT *d = p.coarse_solver == 0 ? Lv<XT>::D(lv) : Lv<XT>::M(lv);
    BCMG_TRY(relax_t<XT>(A, d, B.rhs[l - 1], B.x[l - 1], B.xt[l - 1], p.relaxnumber_coarse,
                         zero[l - 1], s));
    zero[l - 1] = 0;
    return BCMG_OK;
  }
  const XT *d = p.relax_type == 0 ? Lv<XT>::D(lv) : Lv<XT>::M(lv);
  BCMG_TRY(relax_residual_t<XT>(A, d, B.rhs[l - 1], B.x[l - 1], B.xt[l - 1],
                                p.prerelax_sweeps, zero[l - 1], B.res[l - 1], s));
  zero[l - 1] = 0;
  // The coarse level starts from zero: its first sweep (f ./ d) is fused
  // into the restriction where its relaxation can take it.
  int kc = 0;
  const XT *dc = first_relax<XT>(h, k, l + 1, &kc);
  const bool fuse = !lv.Prow && p.cycle_type != 3 &&
                    first_sweep_fusable(Lv<XT>::mat(H.lv[l]), kc);
  if (lv.Prow)
    BCMG_TRY(spmv_t<XT>(Lv<XT>::R(lv), B.res[l - 1], B.rhs[l], s));
  else if (fuse)
    BCMG_TRY(restrict_first_sweep_t<XT>(lv.nc, lv.rptr, lv.ridx, Lv<XT>::p(lv), B.res[l - 1],
                                        B.rhs[l], dc, first_sweep_dst(B.x[l], B.xt[l], kc),
                                        s));
  else
    BCMG_TRY(restrict_t<XT>(lv.nc, lv.rptr, lv.ridx, Lv<XT>::p(lv), B.res[l - 1], B.rhs[l], s));
  zero[l] = fuse ? kStartFirstDone : kStartZero;
  if (p.cycle_type == 3) {
    // K-cycle (GAMG_cycle.cu:88-100): one cycle on the coarsest level, two
    // inner flexible-CG steps on any other.
    if (l == L - 1) {
      BCMG_TRY(cycle_t<XT>(h, B, k, l + 1, zero));
    } else {
      BCMG_TRY(kcycle_inner_t<XT>(h, B, k, l));
      zero[l] = 0;
    }
  } else {
    for (int i = 1; i <= h->grid_sweeps[l - 1]; ++i) {
      BCMG_TRY(cycle_t<XT>(h, B, k, l + 1, zero));
      if (l == L - 1) break;
    }
  }
  if (lv.Prow) {
    BCMG_TRY(spmv_t<XT>(Lv<XT>::P(lv), B.x[l], B.xt[l - 1], s));
    BCMG_TRY(axpy_t<XT>(lv.n, XT(1), B.xt[l - 1], B.x[l - 1], s));
  } else {
    BCMG_TRY(prolong_t<XT>(lv.n, lv.agg, Lv<XT>::p(lv), B.x[l], B.x[l - 1], s));
  }
  BCMG_TRY(relax_t<XT>(A, d, B.rhs[l - 1], B.x[l - 1], B.xt[l - 1], p.postrelax_sweeps,
                       kStartLive, s, l == 1 ? B.widen_out : nullptr));
  return BCMG_OK;
}

// The K-cycle's inner steps with their scalars on the device, for the
// captured FCG loop: the same operations in the same order as the host-driven
// kcycle_inner_t below (so the same bits), the branch on ||w|| an IF node of
// the graph.  A non-positive curvature sets the FCG loop's indefinite flag,
// which ends the loop; the correction is then zero.
__global__ void k_kc_first(double *ks, double *scal) {
  const double delta_old = ks[kKcDelta], tau = ks[kKcTau];
  double alpha = 0.0;
  if (!(delta_old > 0.0) || !(tau > 0.0))
    scal[kIndef] = 1.0;
  else
    alpha = delta_old / tau;
  ks[kKcA0] = alpha;
  ks[kKcNegAlpha] = -alpha;
  ks[kKcA1] = 0.0;
}

__global__ void k_kc_branch(double *ks, cudaGraphConditionalHandle cond) {
  const double delta0 = sqrt(ks[kKcWW]), l2 = sqrt(ks[kKcWW2]);
  const bool second = !(l2 <= kKcycleRtol * delta0);
  ks[kKcSecond] = second ? 1.0 : 0.0;
  cudaGraphSetConditional(cond, second ? 1u : 0u);
}

__global__ void k_kc_second(double *ks) {
  const double tau = ks[kKcTau], tau1 = ks[kKcTau1], tau2 = ks[kKcTau2], tau3 = ks[kKcTau3];
  const double tau4 = tau2 - (tau1 * tau1) / tau;
  ks[kKcA0] = ks[kKcA0] - (tau1 * tau3) / (tau * tau4);
  ks[kKcA1] = tau3 / tau4;
}

// y += coef x with the coefficient read on the device (axpy_t's arithmetic).
template <typename XT>
__global__ void k_kc_axpy(int64_t n, const double *coef, const XT *__restrict__ x,
                          XT *__restrict__ y) {
  const XT a = static_cast<XT>(*coef);
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    y[i] = fma(a, x[i], y[i]);
}

// xk = a0 d0 (+ a1 d1 after a second step): the host path's zero fill and
// one or two axpys, element by element in the same order.
template <typename XT>
__global__ void k_kc_combine(int64_t n, const double *ks, const XT *__restrict__ d0,
                             const XT *__restrict__ d1, XT *__restrict__ xk) {
  const XT a0 = static_cast<XT>(ks[kKcA0]), a1 = static_cast<XT>(ks[kKcA1]);
  const bool second = ks[kKcSecond] != 0.0;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    XT v = fma(a0, d0[i], XT(0));
    if (second) v = fma(a1, d1[i], v);
    xk[i] = v;
  }
}

inline int kc_grid(int64_t n) {
  const int64_t b = (n + 255) / 256;
  return static_cast<int>(b < 1 ? 1 : (b > 4 * kNumSM ? 4 * kNumSM : b));
}

// Adds an IF node at the current point of the capture on h->stream, whose
// condition k_kc_branch sets from ks, and captures body() into it on the
// level's own stream (h->stream points there meanwhile).
bcmg_status capture_kc_if(bcmg_handle *h, int c, double *ks,
                          const std::function<bcmg_status()> &body) {
  cudaStream_t s = h->stream;
  if (c < 0 || c >= static_cast<int>(h->kc_streams.size()))
    return set_error(BCMG_ERR_INTERNAL, "no capture stream for K-cycle level %d", c);
  cudaStream_t s2 = h->kc_streams[c];
  cudaStreamCaptureStatus cs;
  cudaGraph_t g = nullptr;
  const cudaGraphNode_t *deps = nullptr;
  size_t nd = 0;
  BCMG_CUDA(cudaStreamGetCaptureInfo(s, &cs, nullptr, &g, &deps, &nd));
  if (cs != cudaStreamCaptureStatusActive || !g)
    return set_error(BCMG_ERR_INTERNAL, "K-cycle IF node outside a capture");
  cudaGraphConditionalHandle cond;
  BCMG_CUDA(cudaGraphConditionalHandleCreate(&cond, g, 0, 0));
  launch(k_kc_branch, 1, 1, 0, s, ks, cond);
  BCMG_LAUNCH_CHECK();
  BCMG_CUDA(cudaStreamGetCaptureInfo(s, &cs, nullptr, &g, &deps, &nd));
  alignas(cudaGraphNodeParams) unsigned char np_storage[sizeof(cudaGraphNodeParams)];
  std::memset(np_storage, 0, sizeof(np_storage));
  cudaGraphNodeParams &np = *reinterpret_cast<cudaGraphNodeParams *>(np_storage);
  np.type = cudaGraphNodeTypeConditional;
  np.conditional.handle = cond;
  np.conditional.type = cudaGraphCondTypeIf;
  np.conditional.size = 1;
  cudaGraphNode_t node;
  BCMG_CUDA(cudaGraphAddNode(&node, g, deps, nd, &np));
  cudaGraph_t bg = np.conditional.phGraph_out[0];
  BCMG_CUDA(cudaStreamBeginCaptureToGraph(s2, bg, nullptr, nullptr, 0,
                                          cudaStreamCaptureModeThreadLocal));
  h->stream = s2;
  const bcmg_status st = body();
  h->stream = s;
  const cudaError_t e = cudaStreamEndCapture(s2, &bg);
  BCMG_TRY(st);
  if (e != cudaSuccess)
    return set_error(BCMG_ERR_CUDA, "K-cycle IF body capture: %s", cudaGetErrorString(e));
  BCMG_CUDA(cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies));
  return BCMG_OK;
}

template <typename XT>
bcmg_status kcycle_inner_graph(bcmg_handle *h, CycleBufs<XT> &B, int k, int c) {
  const DevLevel &lv = h->H[k].lv[c];
  const MatView A = Lv<XT>::mat(lv);
  const int32_t n = lv.n;
  XT *w = B.kw[c], *d0 = B.kd0[c], *d1 = B.kd1[c], *v = B.kv[c], *v1 = B.kv1[c];
  XT *xk = B.kx[c];
  if (!w || !B.kscal || static_cast<size_t>(c) >= B.kscal_levels)
    return set_error(BCMG_ERR_INTERNAL, "K-cycle buffers missing");
  double *ks = B.kscal + static_cast<size_t>(c) * kKcStride;
  // h->stream is read at every call: inside the IF body it is the body's
  // capture stream.
  auto dot = [&](const XT *a, const XT *b, int slot) -> bcmg_status {
    return dot_t<XT>(n, a, b, ks + slot, h->partials, h->stream);
  };
  auto precond_k = [&](const XT *r, XT *d) -> bcmg_status {
    BCMG_TRY(copy_t<XT>(B.rhs[c], r, n, h->stream));
    std::vector<char> zero(B.rhs.size(), 0);
    zero[c] = 1;
    BCMG_TRY(cycle_t<XT>(h, B, k, c + 1, zero));
    return copy_t<XT>(d, B.x[c], n, h->stream);
  };
  BCMG_TRY(copy_t<XT>(w, B.rhs[c], n, h->stream));
  BCMG_TRY(dot(w, w, kKcWW));
  BCMG_TRY(precond_k(w, d0));
  BCMG_TRY(dot(w, d0, kKcDelta));
  BCMG_TRY(spmv_t<XT>(A, d0, v, h->stream));
  BCMG_TRY(dot(d0, v, kKcTau));
  launch(k_kc_first, 1, 1, 0, h->stream, ks, h->scal);
  launch(k_kc_axpy<XT>, kc_grid(n), 256, 0, h->stream, static_cast<int64_t>(n),
         static_cast<const double *>(ks + kKcNegAlpha), static_cast<const XT *>(v), w);
  BCMG_LAUNCH_CHECK();
  BCMG_TRY(dot(w, w, kKcWW2));
  BCMG_TRY(capture_kc_if(h, c, ks, [&]() -> bcmg_status {
    BCMG_TRY(precond_k(w, d1));
    BCMG_TRY(spmv_t<XT>(A, d1, v1, h->stream));
    BCMG_TRY(dot(d1, v, kKcTau1));
    BCMG_TRY(dot(d1, v1, kKcTau2));
    BCMG_TRY(dot(d1, w, kKcTau3));
    launch(k_kc_second, 1, 1, 0, h->stream, ks);
    BCMG_LAUNCH_CHECK();
    return BCMG_OK;
  }));
  launch(k_kc_combine<XT>, kc_grid(n), 256, 0, h->stream, static_cast<int64_t>(n),
         static_cast<const double *>(ks), static_cast<const XT *>(d0),
         static_cast<const XT *>(d1), xk);
  BCMG_LAUNCH_CHECK();
  return copy_t<XT>(B.x[c], xk, n, h->stream);
}

// inneritkcycle (src/SOLVER/FCG.cu:633-723): two flexible-CG steps on coarse
// level c (0-based) preconditioned by the cycle from that level on fresh
// zero iterates (preconditionApplyK, FCG.cu:590-628); the correction lands
// in x[c], the right-hand side is rhs[c].  Outside a capture the inner
// scalars are read on the host (the reference's branch on ||w|| decides
// whether a second cycle runs); while the FCG loop is captured,
// kcycle_inner_graph keeps them on the device.
template <typename XT>
bcmg_status kcycle_inner_t(bcmg_handle *h, CycleBufs<XT> &B, int k, int c) {
  {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    BCMG_CUDA(cudaStreamIsCapturing(h->stream, &cs));
    if (cs == cudaStreamCaptureStatusActive) return kcycle_inner_graph<XT>(h, B, k, c);
  }
  const DevLevel &lv = h->H[k].lv[c];
  const MatView A = Lv<XT>::mat(lv);
  const int32_t n = lv.n;
  cudaStream_t s = h->stream;
  XT *w = B.kw[c], *d0 = B.kd0[c], *d1 = B.kd1[c], *v = B.kv[c], *v1 = B.kv1[c];
  XT *xk = B.kx[c];
  if (!w || !B.kdots) return set_error(BCMG_ERR_INTERNAL, "K-cycle buffers missing");
  auto dot = [&](const XT *a, const XT *b, double *out) -> bcmg_status {
    BCMG_TRY(dot_t<XT>(n, a, b, B.kdots, h->partials, s));
    BCMG_CUDA(cudaMemcpyAsync(out, B.kdots, sizeof(double), cudaMemcpyDeviceToHost, s));
    BCMG_CUDA(cudaStreamSynchronize(s));
    return BCMG_OK;
  };
  auto precond_k = [&](const XT *r, XT *d) -> bcmg_status {
    BCMG_TRY(copy_t<XT>(B.rhs[c], r, n, s));
    std::vector<char> zero(B.rhs.size(), 0);
    zero[c] = 1;
    BCMG_TRY(cycle_t<XT>(h, B, k, c + 1, zero));
    return copy_t<XT>(d, B.x[c], n, s);
  };
  BCMG_TRY(copy_t<XT>(w, B.rhs[c], n, s));
  double ww = 0, delta_old = 0, tau = 0;
  BCMG_TRY(dot(w, w, &ww));
  const double delta0 = std::sqrt(ww);
  BCMG_TRY(precond_k(w, d0));
  BCMG_TRY(dot(w, d0, &delta_old));
  BCMG_TRY(spmv_t<XT>(A, d0, v, s));
  BCMG_TRY(dot(d0, v, &tau));
  if (!(delta_old > 0.0) || !(tau > 0.0))
    return set_error(BCMG_ERR_INDEFINITE,
                     "K-cycle inner step on level %d: non-positive curvature (%g, %g)", c,
                     delta_old, tau);
  double alpha = delta_old / tau;
  BCMG_TRY(axpy_t<XT>(n, static_cast<XT>(-alpha), v, w, s));
  BCMG_TRY(dot(w, w, &ww));
  const double l2 = std::sqrt(ww);
  BCMG_TRY(fill_t<XT>(xk, n, XT(0), s));
  if (l2 <= kKcycleRtol * delta0) {
    BCMG_TRY(axpy_t<XT>(n, static_cast<XT>(alpha), d0, xk, s));
  } else {
    BCMG_TRY(precond_k(w, d1));
    BCMG_TRY(spmv_t<XT>(A, d1, v1, s));
    double tau1 = 0, tau2 = 0, tau3 = 0;
    BCMG_TRY(dot(d1, v, &tau1));
    BCMG_TRY(dot(d1, v1, &tau2));
    BCMG_TRY(dot(d1, w, &tau3));
    const double tau4 = tau2 - (tau1 * tau1) / tau;
    alpha = alpha - (tau1 * tau3) / (tau * tau4);
    BCMG_TRY(axpy_t<XT>(n, static_cast<XT>(alpha), d0, xk, s));
    alpha = tau3 / tau4;
    BCMG_TRY(axpy_t<XT>(n, static_cast<XT>(alpha), d1, xk, s));
  }
  return copy_t<XT>(B.x[c], xk, n, s);
}

template <typename XT>
bcmg_status run_cycle_t(bcmg_handle *h, CycleBufs<XT> &B, int k, const XT *rhs, XT *x,
                        int start) {
  B.rhs[0] = const_cast<XT *>(rhs);
  B.x[0] = x;
  std::vector<char> zero(B.rhs.size(), 0);
  zero[0] = static_cast<char>(start);
  bcmg_status st = cycle_t<XT>(h, B, k, 1, zero);
  B.rhs[0] = nullptr;
  B.x[0] = nullptr;
  return st;
}

// preconditionApply (src/SOLVER/FCG.cu:112-187).  Level 0 of the cycle works
// directly on the caller's vectors, so the reference's copies into the level
// buffers are not needed.
template <typename XT>
bcmg_status precond_apply_t(bcmg_handle *h, CycleBufs<XT> &B, const XT *rhs, XT *x,
                            bool x_zero) {
  const int nh = static_cast<int>(h->H.size());
  const int32_t n = h->A0.n;
  cudaStream_t s = h->stream;
  if (h->prm.solver_type == 0) {
    for (int k = 0; k < nh; ++k) BCMG_TRY(run_cycle_t<XT>(h, B, k, rhs, x, x_zero && k == 0));
  } else if (h->prm.solver_type == 1) {
    for (int k = 0; k < nh; ++k) BCMG_TRY(run_cycle_t<XT>(h, B, k, rhs, x, x_zero && k == 0));
    for (int k = nh - 1; k >= 0; --k) BCMG_TRY(run_cycle_t<XT>(h, B, k, rhs, x, false));
  } else {
    BCMG_TRY(fill_t<XT>(B.xadd, n, XT(0), s));
    for (int k = 0; k < nh; ++k) {
      if (x_zero) {
        BCMG_TRY(run_cycle_t<XT>(h, B, k, rhs, B.xk, true));
      } else {
        BCMG_TRY(copy_t<XT>(B.xk, x, n, s));
        BCMG_TRY(run_cycle_t<XT>(h, B, k, rhs, B.xk, false));
      }
      BCMG_TRY(axpy_t<XT>(n, XT(1), B.xk, B.xadd, s));
    }
    BCMG_TRY(scale_t<XT>(n, XT(1) / static_cast<XT>(nh), B.xadd, s));
    BCMG_TRY(copy_t<XT>(x, B.xadd, n, s));
  }
  return BCMG_OK;
}

// z = B r on FP64 vectors.  use_mixed selects the FP32 cycle: r is rounded
// to FP32, the cycle runs in FP32 and its result is widened into z.
bcmg_status precond_apply(bcmg_handle *h, const double *rhs, double *x, bool x_zero,
                          bool use_mixed) {
  if (!use_mixed) return precond_apply_t<double>(h, h->c64, rhs, x, x_zero);
  const int32_t n = h->A0.n;
  cudaStream_t s = h->stream;
  CycleBufs<float> &B = h->c32;
  // One V-cycle of one hierarchy: the rounding of r is fused with the first
  // sweep from zero, and the last sweep writes z in FP64 directly.
  const bool single = h->prm.solver_type == 0 && h->H.size() == 1 && h->prm.cycle_type != 3;
  const MatView A0 = single ? Lv<float>::mat(h->H[0].lv[0]) : MatView();
  int k0 = 0;
  const float *d0 = single ? first_relax<float>(h, 0, 1, &k0) : nullptr;
  const bool fuse_first = single && x_zero && first_sweep_fusable(A0, k0);
  const bool fuse_last = single && h->H[0].lv.size() > 1 && widen_fusable(A0, h->prm.postrelax_sweeps);
  if (fuse_first) {
    BCMG_TRY(convert_first_sweep(n, rhs, d0, B.in0, first_sweep_dst(B.out0, B.xt[0], k0), s));
  } else {
    BCMG_TRY(convert_d2f(n, rhs, B.in0, s));
    if (!x_zero) BCMG_TRY(convert_d2f(n, x, B.out0, s));
  }
  B.widen_out = fuse_last ? x : nullptr;
  const bcmg_status st =
      fuse_first ? run_cycle_t<float>(h, B, 0, B.in0, B.out0, kStartFirstDone)
                 : precond_apply_t<float>(h, B, B.in0, B.out0, x_zero);
  B.widen_out = nullptr;
  BCMG_TRY(st);
  if (!fuse_last) BCMG_TRY(convert_f2d(n, B.out0, x, s));
  return BCMG_OK;
}

// Bootstrap::innerIterations (src/BOOT/bootstrap.cu:5-44).  Always FP64 so
// the bootstrapped hierarchies do not depend on the solve precision.
bcmg_status inner_iterations(bcmg_handle *h, double *w) {
  const int32_t n = h->A0.n;
  cudaStream_t s = h->stream;
  double *x = h->xs, *rhs = h->b;
  BCMG_TRY(fill(x, n, 1.0, s));
  BCMG_TRY(fill(rhs, n, 0.0, s));
  double normold = 0, normnew = 0, conv = 1.0;
  BCMG_TRY(anorm(h, x, &normold));
  g_clock.tick("other");
  for (int i = 1; i <= kBootSolverIt; ++i) {
    BCMG_TRY(precond_apply(h, rhs, x, false, false));
    BCMG_TRY(anorm(h, x, &normnew));
    conv = normnew / normold;
    normold = normnew;
  }
  BCMG_TRY(copy(w, x, n, s));
  BCMG_TRY(scale(n, 1.0 / normnew, w, s));
  h->estimated_ratio = conv;
  g_clock.tick("inner_iterations");
  return BCMG_OK;
}

// Low-precision copies of every level for the mixed cycle: level 0 in FP32,
// coarser levels in FP32 / BF16 / FP16 (ext.coarse_storage); D, M and P in
// FP32.
bcmg_status prepare_mixed(bcmg_handle *h) {
  cudaStream_t s = h->stream;
  DevLevel &a = h->A0;
  if (!a.val_lo) {
    BCMG_TRY(dev_alloc(reinterpret_cast<float **>(&a.val_lo), a.nnz, s));
    a.vtype_lo = kValF32;
    BCMG_TRY(convert_values(a.nnz, a.val, a.val_lo, kValF32, s));
  }
  const int coarse_type = coarse_value_type(h);
  for (auto &H : h->H) {
    for (size_t l = 0; l < H.lv.size(); ++l) {
      DevLevel &lv = H.lv[l];
      if (l == 0) {
        lv.val_lo = a.val_lo;
        lv.vtype_lo = kValF32;
        lv.own_lo = false;
      } else {
        const size_t bytes = coarse_type == kValF32 ? 4 : 2;
        BCMG_TRY(dev_alloc(reinterpret_cast<unsigned char **>(&lv.val_lo),
                           static_cast<int64_t>(bytes) * lv.nnz, s));
        lv.vtype_lo = coarse_type;
        lv.own_lo = true;
        BCMG_TRY(convert_values(lv.nnz, lv.val, lv.val_lo, coarse_type, s));
      }
      BCMG_TRY(dev_alloc(&lv.D32, lv.n, s));
      BCMG_TRY(dev_alloc(&lv.M32, lv.n, s));
      BCMG_TRY(convert_d2f(lv.n, lv.D, lv.D32, s));
      BCMG_TRY(convert_d2f(lv.n, lv.M, lv.M32, s));
      if (lv.p) {
        BCMG_TRY(dev_alloc(&lv.p32, lv.n, s));
        BCMG_TRY(convert_d2f(lv.n, lv.p, lv.p32, s));
      }
      if (lv.Prow) {
        BCMG_TRY(dev_alloc(&lv.Pval32, std::max(lv.Pnnz, 1), s));
        BCMG_TRY(dev_alloc(&lv.Rval32, std::max(lv.Pnnz, 1), s));
        BCMG_TRY(convert_d2f(lv.Pnnz, lv.Pval, lv.Pval32, s));
        BCMG_TRY(convert_d2f(lv.Pnnz, lv.Rval, lv.Rval32, s));
      }
    }
  }
  BCMG_TRY(size_buffers_t<float>(h, h->c32));
  return BCMG_OK;
}

// Sliced copies for the solve phase: the FP64 cycle reads s64 on every level,
// the mixed cycle slo; level 0 always has an FP64 copy for the FCG SpMV.
// Level 0 is shared by all hierarchies, so its copies live in h->A0.
bcmg_status prepare_solve_formats(bcmg_handle *h) {
  cudaStream_t s = h->stream;
  DevLevel &a = h->A0;
  if (!a.own64.nslices) BCMG_TRY(build_sliced(h, a.view(), kValF64, &a.own64, s));
  if (h->mixed && !a.ownlo.nslices) {
    // Values narrowed to 16 bits are the same bytes for FP32 vectors: share.
    if (a.own64.nslices && a.own64.narrowed && a.own64.vtype != kValF32)
      BCMG_TRY(sliced_alias(a.own64, kValF32, &a.ownlo, s));
    else
      BCMG_TRY(build_sliced(h, a.view(), kValF32, &a.ownlo, s));
  }
  for (auto &H : h->H) {
    for (size_t l = 0; l < H.lv.size(); ++l) {
      DevLevel &lv = H.lv[l];
      if (l == 0) {
        lv.s64 = &a.own64;
        lv.slo = h->mixed ? &a.ownlo : nullptr;
        continue;
      }
      if (h->mixed) {
        if (!lv.ownlo.nslices) BCMG_TRY(build_sliced(h, lv.view(), lv.vtype_lo, &lv.ownlo, s));
      } else {
        if (!lv.own64.nslices) BCMG_TRY(build_sliced(h, lv.view(), kValF64, &lv.own64, s));
      }
    }
  }
  return BCMG_OK;
}

bcmg_status alloc_work(bcmg_handle *h) {
  const int32_t n = h->A0.n;
  cudaStream_t s = h->stream;
  for (double **p : {&h->r, &h->v, &h->w, &h->d, &h->q, &h->b, &h->xs, &h->tmp})
    BCMG_TRY(dev_alloc(p, n, s));
  BCMG_TRY(dev_alloc(&h->partials, 4 * kRedBlocks, s));
  BCMG_TRY(dev_alloc(&h->scal, kNumScal, s));
  BCMG_CUDA(cudaMemsetAsync(h->scal, 0, sizeof(double) * kNumScal, s));
  return BCMG_OK;
}

// Bootstrap::bootstrap (src/BOOT/bootstrap.cu:46-90).  After the first
// hierarchy the inner iterations are skipped (bootstrap.cu:68-75), so with
// max_hrc >= 2 the second hierarchy comes from the same w = 1.
bcmg_status bootstrap(bcmg_handle *h) {
  const int32_t n = h->A0.n;
  cudaStream_t s = h->stream;
  double *w = nullptr;
  BCMG_TRY(dev_alloc(&w, n, s));
  BCMG_TRY(fill(w, n, 1.0, s));  // BootBuildData::initByParams, AMG.cu:442-443
  h->estimated_ratio = 1.0;
  int num_hrc = 0;
  bcmg_status st = BCMG_OK;
  while (h->estimated_ratio > h->prm.conv_ratio && num_hrc < h->prm.max_hrc) {
    h->H.emplace_back();
    st = adaptive_coarsening(h, w, h->H.back());
    if (st != BCMG_OK) break;
    ++num_hrc;
    st = size_buffers_t<double>(h, h->c64);
    if (st != BCMG_OK) break;
    if (num_hrc > 1) {
      if (h->side) st = h->side->drain();  // the inner iterations read the copies
      if (st != BCMG_OK) break;
      st = inner_iterations(h, w);
      if (st != BCMG_OK) break;
    }
  }
  dev_free(w, s);
  return st;
}

void destroy_handle(bcmg_handle *h) {
  if (!h) return;
  cudaSetDevice(h->device);
  cudaStream_t s = h->stream;
  if (h->fcg_exec) cudaGraphExecDestroy(h->fcg_exec);
  for (cudaStream_t ks : h->kc_streams) cudaStreamDestroy(ks);
  destroy_batch(h);
  for (auto &H : h->H) H.release(s);
  h->A0.own_A = true;
  h->A0.release(s);
  free_buffers_t<double>(h->c64, s);
  free_buffers_t<float>(h->c32, s);
  for (double **p : {&h->r, &h->v, &h->w, &h->d, &h->q, &h->b, &h->xs, &h->tmp,
                     &h->partials, &h->scal})
    dev_free(*p, s);
  cudaStreamSynchronize(s);
  if (h->own_stream) cudaStreamDestroy(s);
  delete h;
}

// BuildData::setMaxCoarseSize (src/AMG/AMG.cu:309-311) and
// ApplyData::setGridSweeps (src/AMG/AMG.cu:371-394).
void set_cycle_tables(bcmg_handle *h) {
  const int32_t n = h->A0.n;
  h->maxcoarsesize = static_cast<int32_t>(40 * std::pow(static_cast<double>(n), 1. / 3.));
  const int ml = std::max(0, h->prm.max_levels - 1);
  h->grid_sweeps.assign(std::max(ml, 1), 1);
  if (h->prm.cycle_type == 1) {
    for (int i = 0; i < ml; ++i)
      if (i % 2 == 0) h->grid_sweeps[i] = 2;
  } else if (h->prm.cycle_type == 2) {
    for (int i = 0; i < ml - 1; ++i) h->grid_sweeps[i] = 2;
  }
}

// After the hierarchies exist: low-precision and sliced solve copies.
bcmg_status finish_setup(bcmg_handle *h) {
  h->mixed = h->ext.precision == BCMG_PREC_MIXED;
  if (h->mixed) BCMG_TRY(prepare_mixed(h));
  g_clock.tick("mixed_copies");
  if (h->ext.sliced) BCMG_TRY(prepare_solve_formats(h));
  g_clock.tick("sliced_copies");
  BCMG_CUDA(cudaStreamSynchronize(h->stream));
  return sliced_wait_status(h->stream);
}

// Clears h->side when the setup that owns the helper returns.
struct SideScope {
  bcmg_handle *h;
  ~SideScope() { h->side = nullptr; }
};

bcmg_status setup_common(bcmg_handle *h) {
  NvtxRange range("bcmg_setup");
  const auto t0 = Clock::now();
  BCMG_TRY(csr_validate(h->A0.view(), h->stream));
  g_clock.start(h->ext.verbose >= 1, h->stream);
  set_cycle_tables(h);
  BCMG_TRY(alloc_work(h));
  // The input matrix's copy is built in line: it is bandwidth-bound work
  // that would take the SMs from the first matching sweep, and the A-norm
  // of the smooth vector reads it.
  if (h->ext.sliced) BCMG_TRY(build_sliced(h, h->A0.view(), kValF64, &h->A0.own64, h->stream));
  // Declared before the scope guard, so h->side is cleared before the
  // helper's destructor drains it.
  std::unique_ptr<SideBuilder> side;
  SideScope scope{h};
  if (h->ext.sliced && h->A0.n >= kSideBuildMinRows) {
    side = std::make_unique<SideBuilder>(h);
    h->side = side.get();
  }
  g_clock.tick("alloc");
  BCMG_TRY(bootstrap(h));
  g_clock.tick("other");
  if (side) BCMG_TRY(side->drain());
  g_clock.tick("side_copies");
  BCMG_TRY(finish_setup(h));
  h->setup_ms = ms_since(t0);
  g_clock.report("setup");
  return BCMG_OK;
}

bcmg_status new_handle(const bcmg_params *p, const bcmg_ext *ext, bcmg_handle **out) {
  if (!p || !out) return set_error(BCMG_ERR_PARAM, "null argument");
  *out = nullptr;
  BCMG_TRY(bcmg_params_check(p));
  auto h = std::make_unique<bcmg_handle>();
  h->prm = *p;
  if (ext)
    h->ext = *ext;
  else
    bcmg_ext_default(&h->ext);
  if (h->ext.precision != BCMG_PREC_FP64 && h->ext.precision != BCMG_PREC_MIXED)
    return set_error(BCMG_ERR_PARAM, "unknown precision mode %d", h->ext.precision);
  h->device = h->ext.device;
  BCMG_CUDA(cudaSetDevice(h->device));
  // Keep freed blocks in the device's default pool (the stream-ordered
  // allocator every work array comes from) instead of returning them to the
  // driver at each synchronisation: repeated setups then reuse the mappings.
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, h->device) == cudaSuccess) {
    uint64_t keep = UINT64_MAX;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  }
  if (h->ext.stream) {
    h->stream = static_cast<cudaStream_t>(h->ext.stream);
    h->own_stream = false;
  } else {
    BCMG_CUDA(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
    h->own_stream = true;
  }
  *out = h.release();
  return BCMG_OK;
}

// w = A v with the fused dots, on the sliced FP64 copy of A when present.
bcmg_status spmv_dots(bcmg_handle *h, const double *v, double *w, const double *r,
                      const double *q) {
  if (h->A0.own64.nslices)
    return sliced_fcg_spmv_dots(h->A0.own64.view(), v, w, r, q, h->partials, h->stream);
  return fcg_spmv_dots(h->A0.view(), v, w, r, q, h->partials, h->scal, h->stream);
}

// One FCG iteration (the body of the do-while, src/SOLVER/FCG.cu:497-565)
// on fixed buffers: z = v, Az = w, previous direction d, Ad = q.
bcmg_status fcg_iteration(bcmg_handle *h, cudaGraphConditionalHandle cond, bool use_cond) {
  cudaStream_t s = h->stream;
  const CsrView A = h->A0.view();
  BCMG_TRY(precond_apply(h, h->r, h->v, true, h->mixed));
  BCMG_TRY(spmv_dots(h, h->v, h->w, h->r, h->q));
  BCMG_TRY(fcg_scalars(h->partials, h->scal, false, s));
  BCMG_TRY(fcg_update(A.n, false, h->v, h->d, h->w, h->q, h->xs, h->r, h->partials, h->scal,
                      s));
  if (h->ext.replace_every > 0) {
    const SlicedView S64 = h->A0.own64.view();
    BCMG_TRY(fcg_replace(A, h->A0.own64.nslices ? &S64 : nullptr, h->b, h->xs, h->r,
                         h->partials, h->scal, h->ext.replace_every, s));
  }
  BCMG_TRY(fcg_continue(h->scal, cond, use_cond, s));
  return BCMG_OK;
}

// Captures the FCG loop once per handle: a graph whose WHILE node repeats one
// iteration until the device-side condition (k_fcg_continue) turns false,
// so a whole solve needs no host round trip per iteration.
bcmg_status build_fcg_graph(bcmg_handle *h) {
  if (h->prm.cycle_type == 3) {
    // the K-cycle's IF bodies are captured on streams of their own, one per
    // level (created here: no stream is created during a capture)
    size_t L = 0;
    for (auto &H : h->H) L = std::max(L, H.lv.size());
    while (h->kc_streams.size() < L) {
      cudaStream_t ks = nullptr;
      BCMG_CUDA(cudaStreamCreateWithFlags(&ks, cudaStreamNonBlocking));
      h->kc_streams.push_back(ks);
    }
  }
  return capture_while_loop(
      h->stream, [h](cudaGraphConditionalHandle cond) { return fcg_iteration(h, cond, true); },
      &h->fcg_exec);
}

// r = b - A x in FP64 on the input matrix, through its sliced copy when
// there is one.
bcmg_status residual64(bcmg_handle *h, const double *b, const double *x, double *r) {
  cudaStream_t s = h->stream;
  if (h->A0.own64.nslices) return sliced_residual<double>(h->A0.own64.view(), b, x, r, s);
  BCMG_TRY(copy(r, b, h->A0.n, s));
  return spmv(h->A0.view(), -1.0, x, 1.0, r, s);
}

// FCG (flexibileConjugateGradients_v3, src/SOLVER/FCG.cu:433-585) on device
// vectors h->b (rhs) and h->xs (initial guess in, solution out).
bcmg_status fcg(bcmg_handle *h, bcmg_solve_info *info) {
  const int32_t n = h->A0.n;
  cudaStream_t s = h->stream;
  double *x = h->xs, *b = h->b, *r = h->r, *v = h->v, *w = h->w, *d = h->d, *q = h->q;
  // r = b - A x0; delta0 = ||r||; ||b||   (FCG.cu:446-457)
  BCMG_TRY(residual64(h, b, x, r));
  double delta0 = 0, bnorm = 0;
  BCMG_TRY(norm2(h, r, &delta0));
  BCMG_TRY(norm2(h, b, &bnorm));
  info->iters = 0;
  info->residual = delta0;
  info->rel_residual = delta0 > 0 ? 1.0 : 0.0;
  info->converged = 0;
  if (delta0 <= DBL_EPSILON * bnorm) {
    // (a residual pass that gave up would make r meaningless)
    BCMG_TRY(sliced_wait_status(s));
    // The reference exits the process here (FCG.cu:459-462).
    info->converged = 1;
    info->rel_residual = 0.0;
    return BCMG_OK;
  }
  const double target = h->prm.rtol * delta0;
  double init[kNumScal] = {0};
  init[kTarget] = target;
  init[kItnlim] = h->prm.itnlim;
  init[kDelta0] = delta0;
  init[kBnorm] = bnorm;
  BCMG_CUDA(cudaMemcpyAsync(h->scal, init, sizeof(init), cudaMemcpyHostToDevice, s));
  pdl_fence(s);
  // First step (FCG.cu:464-495): v = B r; w = A v; x += theta v; r -= theta w;
  // d = v; q = w.
  BCMG_TRY(precond_apply(h, r, v, true, h->mixed));
  BCMG_TRY(spmv_dots(h, v, w, r, nullptr));
  BCMG_TRY(fcg_scalars(h->partials, h->scal, true, s));
  BCMG_TRY(fcg_update(n, true, v, d, w, q, x, r, h->partials, h->scal, s));
  double *hs = h->host_scal;
  const bool graphs = h->ext.use_graphs && h->ext.verbose < 2 && h->stream != nullptr;
  g_clock.tick("first_step");
  if (graphs && !h->fcg_exec && build_fcg_graph(h) != BCMG_OK) {
    clear_error();
    h->fcg_exec = nullptr;
  }
  g_clock.tick("graph_build");
  if (graphs && h->fcg_exec) {
    BCMG_CUDA(cudaGraphLaunch(h->fcg_exec, s));
    BCMG_CUDA(cudaMemcpyAsync(hs, h->scal, sizeof(double) * kNumScal, cudaMemcpyDeviceToHost,
                              s));
    BCMG_CUDA(cudaStreamSynchronize(s));
  } else {
    do {
      BCMG_TRY(fcg_iteration(h, 0, false));
      BCMG_CUDA(cudaMemcpyAsync(hs, h->scal, sizeof(double) * kNumScal,
                                cudaMemcpyDeviceToHost, s));
      BCMG_CUDA(cudaStreamSynchronize(s));
      if (h->ext.verbose > 1)
        printf("bootpcg iteration: %d  residual: %e relative residual: %e\n",
               static_cast<int>(hs[kIter]) - 1, hs[kNorm], hs[kNorm] / delta0);
    } while (hs[kNorm] > target && hs[kIter] < h->prm.itnlim && hs[kIndef] == 0.0);
  }
  g_clock.tick("fcg_loop");
  BCMG_TRY(sliced_wait_status(s));
  const double l2 = hs[kNorm];
  const int iter = static_cast<int>(hs[kIter]);
  info->iters = iter + 1;  // FCG.cu:569
  info->residual = l2;
  info->rel_residual = l2 / delta0;
  info->converged = l2 <= target ? 1 : 0;
  if (hs[kIndef] != 0.0)
    return set_error(BCMG_ERR_INDEFINITE,
                     "FCG met non-positive curvature at iteration %d (A not SPD?)", iter);
  // True residual in FP64: ||b - A x|| / ||b - A x0||.
  BCMG_TRY(residual64(h, b, x, h->tmp));
  double tr = 0;
  BCMG_TRY(norm2(h, h->tmp, &tr));
  info->true_rel_residual = tr / delta0;
  return BCMG_OK;
}

}  // namespace

// Device bytes a level holds (pointer fields that are set; shared arrays are
// counted by their owner).
size_t level_bytes(const DevLevel &l) {
  const size_t n = static_cast<size_t>(l.n), nnz = static_cast<size_t>(l.nnz);
  size_t b = 0;
  if (l.own_A && l.row) b += 4 * (n + 1) + 12 * nnz;
  for (const double *v : {l.D, l.M, l.w, l.p})
    if (v) b += 8 * n;
  if (l.agg) b += 4 * n;
  if (l.rptr) b += 4 * (static_cast<size_t>(l.nc) + 1);
  if (l.ridx) b += 4 * n;
  if (l.own_lo && l.val_lo) b += (l.vtype_lo == kValF32 ? 4 : 2) * nnz;
  for (const float *v : {l.D32, l.M32, l.p32})
    if (v) b += 4 * n;
  if (l.Prow) {  // P and R (CSR), FP32 value copies
    const size_t pn = static_cast<size_t>(l.Pnnz);
    b += 4 * (n + 1) + 4 * (static_cast<size_t>(l.nc) + 1) + 2 * 12 * pn;
    if (l.Pval32) b += 2 * 4 * pn;
  }
  return b + l.own64.bytes() + l.ownlo.bytes();
}

template <typename XT>
size_t cycle_bytes(const CycleBufs<XT> &B, size_t n0, size_t width) {
  size_t b = 0;
  for (size_t l = 0; l < B.n.size(); ++l) {
    const size_t per = static_cast<size_t>(B.n[l]) * width * sizeof(XT);
    b += per * ((B.xt[l] ? 1 : 0) + (B.res[l] ? 1 : 0));
    if (l > 0) b += per * ((B.rhs[l] ? 1 : 0) + (B.x[l] ? 1 : 0));
  }
  const XT *top[] = {B.xk, B.xadd, B.in0, B.out0};
  for (const XT *v : top)
    if (v) b += n0 * width * sizeof(XT);
  return b;
}
template size_t cycle_bytes<double>(const CycleBufs<double> &, size_t, size_t);
template size_t cycle_bytes<float>(const CycleBufs<float> &, size_t, size_t);

size_t handle_bytes(const bcmg_handle *h) {
  const size_t n = static_cast<size_t>(h->A0.n);
  size_t b = 4 * (n + 1) + 12 * static_cast<size_t>(h->A0.nnz);
  if (h->A0.val_lo) b += 4 * static_cast<size_t>(h->A0.nnz);
  b += h->A0.own64.bytes() + h->A0.ownlo.bytes();
  for (const auto &H : h->H)
    for (const auto &l : H.lv) b += level_bytes(l);
  b += cycle_bytes(h->c64, n, 1) + cycle_bytes(h->c32, n, 1);
  b += 8 * 8 * n + 8 * (4 * static_cast<size_t>(kRedBlocks) + kNumScal);
  return b + batch_bytes(h);
}

bcmg_status capture_while_loop(cudaStream_t stream,
                               const std::function<bcmg_status(cudaGraphConditionalHandle)> &body_fn,
                               cudaGraphExec_t *out) {
  *out = nullptr;
  cudaGraph_t g = nullptr;
  BCMG_CUDA(cudaGraphCreate(&g, 0));
  cudaGraphConditionalHandle cond;
  cudaError_t e = cudaGraphConditionalHandleCreate(&cond, g, 1, cudaGraphCondAssignDefault);
  if (e != cudaSuccess) {
    cudaGraphDestroy(g);
    return set_error(BCMG_ERR_CUDA, "conditional handle: %s", cudaGetErrorString(e));
  }
  // cudaGraphNodeParams has no default constructor (it holds a union); use
  // zeroed storage as the CUDA samples do with their C-style initializers.
  alignas(cudaGraphNodeParams) unsigned char np_storage[sizeof(cudaGraphNodeParams)];
  std::memset(np_storage, 0, sizeof(np_storage));
  cudaGraphNodeParams &np = *reinterpret_cast<cudaGraphNodeParams *>(np_storage);
  np.type = cudaGraphNodeTypeConditional;
  np.conditional.handle = cond;
  np.conditional.type = cudaGraphCondTypeWhile;
  np.conditional.size = 1;
  cudaGraphNode_t node;
  e = cudaGraphAddNode(&node, g, nullptr, 0, &np);
  if (e != cudaSuccess) {
    cudaGraphDestroy(g);
    return set_error(BCMG_ERR_CUDA, "conditional node: %s", cudaGetErrorString(e));
  }
  cudaGraph_t body = np.conditional.phGraph_out[0];
  e = cudaStreamBeginCaptureToGraph(stream, body, nullptr, nullptr, 0,
                                    cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) {
    cudaGraphDestroy(g);
    return set_error(BCMG_ERR_CUDA, "begin capture: %s", cudaGetErrorString(e));
  }
  bcmg_status st = body_fn(cond);
  e = cudaStreamEndCapture(stream, &body);
  if (st != BCMG_OK || e != cudaSuccess) {
    cudaGetLastError();
    cudaGraphDestroy(g);
    return st != BCMG_OK ? st
                         : set_error(BCMG_ERR_CUDA, "end capture: %s", cudaGetErrorString(e));
  }
  e = cudaGraphInstantiate(out, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) {
    *out = nullptr;
    return set_error(BCMG_ERR_CUDA, "instantiate: %s", cudaGetErrorString(e));
  }
  return BCMG_OK;
}

// ---- hierarchy files ---------------------------------------------------------
// Binary, little-endian: the magic "BCMGHRC1", the 14 settings, the input
// matrix, then per hierarchy its level data (CSR of levels >= 1, D, M, w, and
// for every level but the last the aggregates and prolongator values; R's
// member lists are rebuilt from the aggregates on load).  With smoothed
// aggregation (aggrtype 1) every level but the last also holds its smoothed
// prolongator P (nnz, then CSR row pointers, columns, values); R = P^T is
// rebuilt on load by the transpose setup uses, so it is the same bits.  Each array is an
// int64 count followed by its raw elements, in the manner of the reference's
// Vector::dump / Vector::load (src/matrix/vector.cu:468-505).
constexpr char kHrcMagic[8] = {'B', 'C', 'M', 'G', 'H', 'R', 'C', '1'};

struct FileCloser {
  void operator()(FILE *f) const {
    if (f) fclose(f);
  }
};
using File = std::unique_ptr<FILE, FileCloser>;

template <typename T>
bcmg_status put_array(FILE *f, const T *dev, int64_t count, cudaStream_t s) {
  if (fwrite(&count, sizeof(count), 1, f) != 1) return set_error(BCMG_ERR_IO, "write failed");
  if (count <= 0) return BCMG_OK;
  std::vector<T> host(static_cast<size_t>(count));
  BCMG_CUDA(cudaMemcpyAsync(host.data(), dev, sizeof(T) * count, cudaMemcpyDeviceToHost, s));
  BCMG_CUDA(cudaStreamSynchronize(s));
  if (fwrite(host.data(), sizeof(T), host.size(), f) != host.size())
    return set_error(BCMG_ERR_IO, "write failed");
  return BCMG_OK;
}

template <typename T>
bcmg_status get_array(FILE *f, T **dev, int64_t expect, cudaStream_t s) {
  int64_t count = -1;
  if (fread(&count, sizeof(count), 1, f) != 1 || count != expect)
    return set_error(BCMG_ERR_IO, "hierarchy file: array of %lld entries where %lld expected",
                     static_cast<long long>(count), static_cast<long long>(expect));
  *dev = nullptr;
  if (count <= 0) return BCMG_OK;
  std::vector<T> host(static_cast<size_t>(count));
  if (fread(host.data(), sizeof(T), host.size(), f) != host.size())
    return set_error(BCMG_ERR_IO, "hierarchy file truncated");
  BCMG_TRY(dev_alloc(dev, count, s));
  BCMG_CUDA(cudaMemcpyAsync(*dev, host.data(), sizeof(T) * count, cudaMemcpyHostToDevice, s));
  BCMG_CUDA(cudaStreamSynchronize(s));
  return BCMG_OK;
}

bcmg_status put_scalars(FILE *f, const void *p, size_t bytes) {
  return fwrite(p, 1, bytes, f) == bytes ? BCMG_OK : set_error(BCMG_ERR_IO, "write failed");
}
bcmg_status get_scalars(FILE *f, void *p, size_t bytes) {
  return fread(p, 1, bytes, f) == bytes ? BCMG_OK
                                        : set_error(BCMG_ERR_IO, "hierarchy file truncated");
}

bcmg_status save_hierarchies(const bcmg_handle *h, FILE *f) {
  cudaStream_t s = h->stream;
  BCMG_TRY(put_scalars(f, kHrcMagic, sizeof(kHrcMagic)));
  BCMG_TRY(put_scalars(f, &h->prm, sizeof(h->prm)));
  const int32_t dims[3] = {h->A0.n, h->A0.nnz, static_cast<int32_t>(h->H.size())};
  BCMG_TRY(put_scalars(f, dims, sizeof(dims)));
  BCMG_TRY(put_scalars(f, &h->estimated_ratio, sizeof(double)));
  BCMG_TRY(put_array(f, h->A0.row, h->A0.n + 1, s));
  BCMG_TRY(put_array(f, h->A0.col, h->A0.nnz, s));
  BCMG_TRY(put_array(f, h->A0.val, h->A0.nnz, s));
  for (const DevHierarchy &H : h->H) {
    const double stats[3] = {H.op_cmplx, H.op_wcmplx, H.avg_cratio};
    BCMG_TRY(put_scalars(f, stats, sizeof(stats)));
    const int32_t L = static_cast<int32_t>(H.lv.size());
    BCMG_TRY(put_scalars(f, &L, sizeof(L)));
    for (int32_t l = 0; l < L; ++l) {
      const DevLevel &lv = H.lv[l];
      const int32_t ld[3] = {lv.n, lv.nnz, lv.nc};
      BCMG_TRY(put_scalars(f, ld, sizeof(ld)));
      if (l > 0) {
        BCMG_TRY(put_array(f, lv.row, lv.n + 1, s));
        BCMG_TRY(put_array(f, lv.col, lv.nnz, s));
        BCMG_TRY(put_array(f, lv.val, lv.nnz, s));
      }
      BCMG_TRY(put_array(f, lv.D, lv.n, s));
      BCMG_TRY(put_array(f, lv.M, lv.n, s));
      BCMG_TRY(put_array(f, lv.w, lv.n, s));
      if (lv.nc > 0) {
        BCMG_TRY(put_array(f, lv.agg, lv.n, s));
        BCMG_TRY(put_array(f, lv.p, lv.n, s));
        if (h->prm.aggrtype == 1) {
          if (!lv.Prow) return set_error(BCMG_ERR_INTERNAL, "level %d has no smoothed P", l);
          BCMG_TRY(put_scalars(f, &lv.Pnnz, sizeof(lv.Pnnz)));
          BCMG_TRY(put_array(f, lv.Prow, static_cast<int64_t>(lv.n) + 1, s));
          BCMG_TRY(put_array(f, lv.Pcol, lv.Pnnz, s));
          BCMG_TRY(put_array(f, lv.Pval, lv.Pnnz, s));
        }
      }
    }
  }
  return BCMG_OK;
}

bcmg_status load_hierarchies(bcmg_handle *h, FILE *f) {
  cudaStream_t s = h->stream;
  int32_t dims[3];
  BCMG_TRY(get_scalars(f, dims, sizeof(dims)));
  BCMG_TRY(get_scalars(f, &h->estimated_ratio, sizeof(double)));
  if (dims[0] <= 0 || dims[1] < dims[0] || dims[2] < 1)
    return set_error(BCMG_ERR_IO, "hierarchy file: bad sizes");
  DevLevel &a = h->A0;
  a.n = dims[0];
  a.nnz = dims[1];
  BCMG_TRY(get_array(f, &a.row, a.n + 1, s));
  BCMG_TRY(get_array(f, &a.col, a.nnz, s));
  BCMG_TRY(get_array(f, &a.val, a.nnz, s));
  BCMG_TRY(csr_validate(a.view(), s));
  set_cycle_tables(h);
  BCMG_TRY(alloc_work(h));
  if (h->ext.sliced)
    BCMG_TRY(build_sliced(h, a.view(), kValF64, &a.own64, s));
  for (int32_t k = 0; k < dims[2]; ++k) {
    h->H.emplace_back();
    DevHierarchy &H = h->H.back();
    double stats[3];
    BCMG_TRY(get_scalars(f, stats, sizeof(stats)));
    H.op_cmplx = stats[0];
    H.op_wcmplx = stats[1];
    H.avg_cratio = stats[2];
    int32_t L = 0;
    BCMG_TRY(get_scalars(f, &L, sizeof(L)));
    if (L < 1 || L > 64) return set_error(BCMG_ERR_IO, "hierarchy file: %d levels", L);
    for (int32_t l = 0; l < L; ++l) {
      int32_t ld[3];
      BCMG_TRY(get_scalars(f, ld, sizeof(ld)));
      H.lv.emplace_back();
      DevLevel &lv = H.lv.back();
      lv.n = ld[0];
      lv.nnz = ld[1];
      lv.nc = ld[2];
      if (l == 0) {
        if (lv.n != a.n || lv.nnz != a.nnz)
          return set_error(BCMG_ERR_IO, "hierarchy file: level 0 is not the input matrix");
        lv.row = a.row;
        lv.col = a.col;
        lv.val = a.val;
        lv.own_A = false;
        if (a.own64.nslices) lv.s64 = &a.own64;
      } else {
        if (lv.n <= 0 || lv.nnz < lv.n || lv.n != H.lv[l - 1].nc)
          return set_error(BCMG_ERR_IO, "hierarchy file: bad size of level %d", l);
        BCMG_TRY(get_array(f, &lv.row, lv.n + 1, s));
        BCMG_TRY(get_array(f, &lv.col, lv.nnz, s));
        BCMG_TRY(get_array(f, &lv.val, lv.nnz, s));
        BCMG_TRY(csr_validate(lv.view(), s));
      }
      BCMG_TRY(get_array(f, &lv.D, lv.n, s));
      BCMG_TRY(get_array(f, &lv.M, lv.n, s));
      BCMG_TRY(get_array(f, &lv.w, lv.n, s));
      const bool last = l == L - 1;
      if (last != (lv.nc == 0))
        return set_error(BCMG_ERR_IO, "hierarchy file: level %d coarse size %d", l, lv.nc);
      if (!last) {
        if (lv.nc <= 0 || lv.nc > lv.n)
          return set_error(BCMG_ERR_IO, "hierarchy file: bad coarse size on level %d", l);
        BCMG_TRY(get_array(f, &lv.agg, lv.n, s));
        BCMG_TRY(get_array(f, &lv.p, lv.n, s));
        BCMG_TRY(dev_alloc(&lv.rptr, lv.nc + 1, s));
        BCMG_TRY(dev_alloc(&lv.ridx, lv.n, s));
        BCMG_TRY(transpose_agg(lv.n, lv.agg, lv.nc, lv.rptr, lv.ridx, s));
        if (h->prm.aggrtype == 1) {
          int32_t pnnz = -1;
          BCMG_TRY(get_scalars(f, &pnnz, sizeof(pnnz)));
          if (pnnz < 0 || static_cast<int64_t>(pnnz) > static_cast<int64_t>(lv.n) * lv.nc)
            return set_error(BCMG_ERR_IO, "hierarchy file: P of level %d has %d entries", l,
                             pnnz);
          lv.Pnnz = pnnz;
          BCMG_TRY(get_array(f, &lv.Prow, static_cast<int64_t>(lv.n) + 1, s));
          BCMG_TRY(get_array(f, &lv.Pcol, pnnz, s));
          BCMG_TRY(get_array(f, &lv.Pval, pnnz, s));
          BCMG_TRY(csr_validate_rect(lv.pview(), lv.nc, s));
          BCMG_TRY(dev_alloc(&lv.Rrow, static_cast<int64_t>(lv.nc) + 1, s));
          BCMG_TRY(dev_alloc(&lv.Rcol, pnnz, s));
          BCMG_TRY(dev_alloc(&lv.Rval, pnnz, s));
          BCMG_TRY(csr_transpose(lv.pview(), lv.nc, lv.Rrow, lv.Rcol, lv.Rval, s));
        }
      }
    }
    BCMG_TRY(size_buffers_t<double>(h, h->c64));
  }
  return finish_setup(h);
}

}  // namespace bcmg

using namespace bcmg;

extern "C" {

bcmg_status bcmg_setup(const bcmg_csr *A, const bcmg_params *p, const bcmg_ext *ext,
                       bcmg_handle **out) {
  clear_error();
  if (!A || !out) return set_error(BCMG_ERR_PARAM, "null argument");
  *out = nullptr;
  // Only the O(1) checks here; the entries are validated on the device after
  // the upload (csr_validate), which is far faster than a host pass.
  if (!A->row || (A->nnz > 0 && (!A->col || !A->val)))
    return set_error(BCMG_ERR_PARAM, "null CSR array");
  if (A->n <= 0 || A->n != A->m)
    return set_error(BCMG_ERR_INVALID_MATRIX, "matrix must be square with n > 0 (%d x %d)",
                     A->n, A->m);
  if (A->row[0] != 0 || A->row[A->n] != A->nnz)
    return set_error(BCMG_ERR_INVALID_MATRIX, "row pointer does not span [0, nnz]");
  bcmg_handle *h = nullptr;
  BCMG_TRY(new_handle(p, ext, &h));
  std::unique_ptr<bcmg_handle, void (*)(bcmg_handle *)> guard(h, destroy_handle);
  DevLevel &a = h->A0;
  a.n = A->n;
  a.nnz = A->nnz;
  BCMG_TRY(dev_alloc(&a.row, a.n + 1, h->stream));
  BCMG_TRY(dev_alloc(&a.col, a.nnz, h->stream));
  BCMG_TRY(dev_alloc(&a.val, a.nnz, h->stream));
  BCMG_CUDA(cudaMemcpyAsync(a.row, A->row, sizeof(int32_t) * (a.n + 1),
                            cudaMemcpyHostToDevice, h->stream));
  BCMG_CUDA(cudaMemcpyAsync(a.col, A->col, sizeof(int32_t) * a.nnz, cudaMemcpyHostToDevice,
                            h->stream));
  BCMG_CUDA(cudaMemcpyAsync(a.val, A->val, sizeof(double) * a.nnz, cudaMemcpyHostToDevice,
                            h->stream));
  BCMG_TRY(setup_common(h));
  *out = guard.release();
  return BCMG_OK;
}

bcmg_status bcmg_setup_device(int32_t n, int32_t nnz, const int32_t *d_row,
                              const int32_t *d_col, const double *d_val,
                              const bcmg_params *p, const bcmg_ext *ext, bcmg_handle **out) {
  clear_error();
  if (!d_row || !d_col || !d_val || !out || n <= 0 || nnz < n)
    return set_error(BCMG_ERR_PARAM, "bad device CSR arguments");
  *out = nullptr;
  bcmg_handle *h = nullptr;
  BCMG_TRY(new_handle(p, ext, &h));
  std::unique_ptr<bcmg_handle, void (*)(bcmg_handle *)> guard(h, destroy_handle);
  DevLevel &a = h->A0;
  a.n = n;
  a.nnz = nnz;
  BCMG_TRY(dev_alloc(&a.row, n + 1, h->stream));
  BCMG_TRY(dev_alloc(&a.col, nnz, h->stream));
  BCMG_TRY(dev_alloc(&a.val, nnz, h->stream));
  BCMG_CUDA(cudaMemcpyAsync(a.row, d_row, sizeof(int32_t) * (n + 1),
                            cudaMemcpyDeviceToDevice, h->stream));
  BCMG_CUDA(cudaMemcpyAsync(a.col, d_col, sizeof(int32_t) * nnz, cudaMemcpyDeviceToDevice,
                            h->stream));
  BCMG_CUDA(cudaMemcpyAsync(a.val, d_val, sizeof(double) * nnz, cudaMemcpyDeviceToDevice,
                            h->stream));
  BCMG_TRY(setup_common(h));
  *out = guard.release();
  return BCMG_OK;
}

bcmg_status bcmg_solve(bcmg_handle *h, const double *b, double *x, int on_device,
                       bcmg_solve_info *info) {
  clear_error();
  if (!h || !b || !x) return set_error(BCMG_ERR_PARAM, "null argument");
  bcmg_solve_info local;
  if (!info) info = &local;
  std::memset(info, 0, sizeof(*info));
  BCMG_CUDA(cudaSetDevice(h->device));
  NvtxRange range("bcmg_solve");
  const auto t0 = Clock::now();
  g_clock.start(h->ext.verbose >= 1, h->stream);
  const int32_t n = h->A0.n;
  const cudaMemcpyKind in = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  BCMG_CUDA(cudaMemcpyAsync(h->b, b, sizeof(double) * n, in, h->stream));
  BCMG_CUDA(cudaMemcpyAsync(h->xs, x, sizeof(double) * n, in, h->stream));
  pdl_fence(h->stream);  // the FCG's first kernels are programmatic launches
  bcmg_status st = fcg(h, info);
  const cudaMemcpyKind outk = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
  BCMG_CUDA(cudaMemcpyAsync(x, h->xs, sizeof(double) * n, outk, h->stream));
  BCMG_CUDA(cudaStreamSynchronize(h->stream));
  info->solve_ms = ms_since(t0);
  g_clock.tick("finish");
  g_clock.report("solve");
  info->setup_ms = h->setup_ms;
  info->num_hrc = static_cast<int>(h->H.size());
  info->estimated_ratio = h->estimated_ratio;
  return st;
}

bcmg_status bcmg_solve_legacy(const bcmg_csr *A, const bcmg_params *p, const bcmg_ext *ext,
                              const double *b, double *x, bcmg_solve_info *info) {
  if (!A || !b || !x) return set_error(BCMG_ERR_PARAM, "null argument");
  bcmg_handle *h = nullptr;
  BCMG_TRY(bcmg_setup(A, p, ext, &h));
  for (int32_t i = 0; i < A->n; ++i) x[i] = 0.0;  // Sol = 0, solver.cu:222-223
  bcmg_status st = bcmg_solve(h, b, x, 0, info);
  bcmg_destroy(h);
  return st;
}

unsigned long long bcmg_kernel_launches(void) {
  return g_kernel_launches.load(std::memory_order_relaxed);
}

bcmg_status bcmg_set_max_device_seconds(bcmg_handle *h, double seconds) {
  clear_error();
  if (!h || !(seconds > 0.0))
    return set_error(BCMG_ERR_PARAM, "need a handle and a positive bound in seconds");
  h->ext.max_device_seconds = seconds;
  const unsigned long long ns = wait_ns_of(h);
  h->A0.own64.wait_ns = h->A0.ownlo.wait_ns = ns;
  for (auto &H : h->H)
    for (auto &lv : H.lv) lv.own64.wait_ns = lv.ownlo.wait_ns = ns;
  // The captured FCG loop holds the old bound in its kernel parameters; the
  // next solve captures it again.
  if (h->fcg_exec) {
    BCMG_CUDA(cudaSetDevice(h->device));
    BCMG_CUDA(cudaStreamSynchronize(h->stream));
    cudaGraphExecDestroy(h->fcg_exec);
    h->fcg_exec = nullptr;
  }
  return BCMG_OK;
}

bcmg_status bcmg_wait_selftest(int device, double seconds) {
  clear_error();
  if (!(seconds > 0.0) || seconds > 10.0)
    return set_error(BCMG_ERR_PARAM, "bound must be in (0, 10] seconds");
  BCMG_CUDA(cudaSetDevice(device));
  cudaStream_t s = nullptr;
  BCMG_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  const bcmg_status st = wait_selftest(static_cast<unsigned long long>(seconds * 1e9), s);
  cudaStreamSynchronize(s);
  cudaStreamDestroy(s);
  return st;
}

bcmg_status bcmg_debug_fail_alloc(int64_t after) {
  g_fail_alloc_countdown.store(after < 0 ? -1 : after, std::memory_order_relaxed);
  return BCMG_OK;
}

bcmg_status bcmg_debug_alloc_stats(int64_t *live, int64_t *made) {
  if (live) *live = g_live_allocs.load(std::memory_order_relaxed);
  if (made) *made = g_made_allocs.load(std::memory_order_relaxed);
  return BCMG_OK;
}

bcmg_status bcmg_device_bytes(const bcmg_handle *h, uint64_t *bytes) {
  if (!h || !bytes) return set_error(BCMG_ERR_PARAM, "null argument");
  *bytes = handle_bytes(h);
  return BCMG_OK;
}

bcmg_status bcmg_destroy(bcmg_handle *h) {
  destroy_handle(h);
  return BCMG_OK;
}

bcmg_status bcmg_get_params(const bcmg_handle *h, bcmg_params *p) {
  if (!h || !p) return set_error(BCMG_ERR_PARAM, "null argument");
  *p = h->prm;
  return BCMG_OK;
}

bcmg_status bcmg_save(const bcmg_handle *h, const char *path) {
  clear_error();
  if (!h || !path) return set_error(BCMG_ERR_PARAM, "null argument");
  BCMG_CUDA(cudaSetDevice(h->device));
  File f(fopen(path, "wb"));
  if (!f) return set_error(BCMG_ERR_IO, "cannot open %s for writing", path);
  BCMG_TRY(save_hierarchies(h, f.get()));
  if (fflush(f.get()) != 0) return set_error(BCMG_ERR_IO, "write failed: %s", path);
  return BCMG_OK;
}

bcmg_status bcmg_load(const char *path, const bcmg_ext *ext, bcmg_handle **out) {
  clear_error();
  if (!path || !out) return set_error(BCMG_ERR_PARAM, "null argument");
  *out = nullptr;
  File f(fopen(path, "rb"));
  if (!f) return set_error(BCMG_ERR_IO, "cannot open %s", path);
  char magic[sizeof(kHrcMagic)];
  bcmg_params prm;
  if (fread(magic, 1, sizeof(magic), f.get()) != sizeof(magic) ||
      std::memcmp(magic, kHrcMagic, sizeof(magic)) != 0)
    return set_error(BCMG_ERR_IO, "%s is not a hierarchy file", path);
  if (fread(&prm, sizeof(prm), 1, f.get()) != 1)
    return set_error(BCMG_ERR_IO, "hierarchy file truncated");
  if (prm.aggrtype != 0 && prm.aggrtype != 1)
    return set_error(BCMG_ERR_IO, "%s: hierarchy file with aggrtype %d", path, prm.aggrtype);
  const auto t0 = Clock::now();
  bcmg_handle *h = nullptr;
  BCMG_TRY(new_handle(&prm, ext, &h));
  std::unique_ptr<bcmg_handle, void (*)(bcmg_handle *)> guard(h, destroy_handle);
  BCMG_TRY(load_hierarchies(h, f.get()));
  h->setup_ms = ms_since(t0);
  *out = guard.release();
  return BCMG_OK;
}

bcmg_status bcmg_set_stream(bcmg_handle *h, void *stream) {
  if (!h) return set_error(BCMG_ERR_PARAM, "null handle");
  BCMG_CUDA(cudaSetDevice(h->device));
  BCMG_CUDA(cudaStreamSynchronize(h->stream));
  if (h->own_stream) BCMG_CUDA(cudaStreamDestroy(h->stream));
  h->stream = static_cast<cudaStream_t>(stream);
  h->own_stream = false;
  return BCMG_OK;
}

bcmg_status bcmg_precond_apply(bcmg_handle *h, const double *d_r, double *d_z) {
  if (!h || !d_r || !d_z) return set_error(BCMG_ERR_PARAM, "null argument");
  BCMG_CUDA(cudaSetDevice(h->device));
  BCMG_TRY(precond_apply(h, d_r, d_z, false, h->mixed));
  BCMG_CUDA(cudaStreamSynchronize(h->stream));
  return BCMG_OK;
}

bcmg_status bcmg_hierarchy_count(const bcmg_handle *h, int *num_hrc, double *est) {
  if (!h) return set_error(BCMG_ERR_PARAM, "null handle");
  if (num_hrc) *num_hrc = static_cast<int>(h->H.size());
  if (est) *est = h->estimated_ratio;
  return BCMG_OK;
}

bcmg_status bcmg_hierarchy_info(const bcmg_handle *h, int hrc, int *num_levels,
                                double *op_cmplx, double *op_wcmplx, double *avg_cratio) {
  if (!h || hrc < 0 || hrc >= static_cast<int>(h->H.size()))
    return set_error(BCMG_ERR_PARAM, "bad hierarchy index");
  const DevHierarchy &H = h->H[hrc];
  if (num_levels) *num_levels = static_cast<int>(H.lv.size());
  if (op_cmplx) *op_cmplx = H.op_cmplx;
  if (op_wcmplx) *op_wcmplx = H.op_wcmplx;
  if (avg_cratio) *avg_cratio = H.avg_cratio;
  return BCMG_OK;
}

bcmg_status bcmg_level_info(const bcmg_handle *h, int hrc, int level, int32_t *n,
                            int32_t *nnz, int32_t *n_coarse) {
  if (!h || hrc < 0 || hrc >= static_cast<int>(h->H.size()))
    return set_error(BCMG_ERR_PARAM, "bad hierarchy index");
  const DevHierarchy &H = h->H[hrc];
  if (level < 0 || level >= static_cast<int>(H.lv.size()))
    return set_error(BCMG_ERR_PARAM, "bad level index");
  const DevLevel &l = H.lv[level];
  if (n) *n = l.n;
  if (nnz) *nnz = l.nnz;
  if (n_coarse) *n_coarse = l.nc;
  return BCMG_OK;
}

bcmg_status bcmg_level_copy(const bcmg_handle *h, int hrc, int level, int32_t *row,
                            int32_t *col, double *val, double *D, double *M, int32_t *agg,
                            double *p, double *w) {
  if (!h || hrc < 0 || hrc >= static_cast<int>(h->H.size()))
    return set_error(BCMG_ERR_PARAM, "bad hierarchy index");
  const DevHierarchy &H = h->H[hrc];
  if (level < 0 || level >= static_cast<int>(H.lv.size()))
    return set_error(BCMG_ERR_PARAM, "bad level index");
  BCMG_CUDA(cudaSetDevice(h->device));
  const DevLevel &l = H.lv[level];
  cudaStream_t s = h->stream;
  auto get = [&](void *dst, const void *src, size_t bytes) -> bcmg_status {
    if (dst && src && bytes)
      BCMG_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s));
    return BCMG_OK;
  };
  BCMG_TRY(get(row, l.row, sizeof(int32_t) * (l.n + 1)));
  BCMG_TRY(get(col, l.col, sizeof(int32_t) * l.nnz));
  BCMG_TRY(get(val, l.val, sizeof(double) * l.nnz));
  BCMG_TRY(get(D, l.D, sizeof(double) * l.n));
  BCMG_TRY(get(M, l.M, sizeof(double) * l.n));
  BCMG_TRY(get(w, l.w, sizeof(double) * l.n));
  if (l.agg) BCMG_TRY(get(agg, l.agg, sizeof(int32_t) * l.n));
  if (l.p) BCMG_TRY(get(p, l.p, sizeof(double) * l.n));
  BCMG_CUDA(cudaStreamSynchronize(s));
  return BCMG_OK;
}

bcmg_status bcmg_level_relax(bcmg_handle *h, int hrc, int level, const void *d_f, void *d_u,
                             int k) {
  clear_error();
  if (!h || hrc < 0 || hrc >= static_cast<int>(h->H.size()) || !d_f || !d_u || k < 0)
    return set_error(BCMG_ERR_PARAM, "bad arguments");
  DevHierarchy &H = h->H[hrc];
  if (level < 0 || level >= static_cast<int>(H.lv.size()))
    return set_error(BCMG_ERR_PARAM, "bad level index");
  BCMG_CUDA(cudaSetDevice(h->device));
  NvtxRange range("bcmg_level_relax");
  const DevLevel &lv = H.lv[level];
  const bool coarsest = level == static_cast<int>(H.lv.size()) - 1;
  const int type = coarsest ? h->prm.coarse_solver : h->prm.relax_type;
  if (h->mixed) {
    const float *dd = type == 0 ? Lv<float>::D(lv) : Lv<float>::M(lv);
    BCMG_TRY(relax_t<float>(Lv<float>::mat(lv), dd, static_cast<const float *>(d_f),
                            static_cast<float *>(d_u), h->c32.xt[level], k, false, h->stream));
  } else {
    const double *dd = type == 0 ? Lv<double>::D(lv) : Lv<double>::M(lv);
    BCMG_TRY(relax_t<double>(Lv<double>::mat(lv), dd, static_cast<const double *>(d_f),
                             static_cast<double *>(d_u), h->c64.xt[level], k, false,
                             h->stream));
  }
  BCMG_CUDA(cudaStreamSynchronize(h->stream));
  return sliced_wait_status(h->stream);
}

bcmg_status bcmg_level_format(const bcmg_handle *h, int hrc, int level, int64_t *slots,
                              int64_t *column_slots, int32_t *slices, int32_t *value_bytes) {
  if (!h || hrc < 0 || hrc >= static_cast<int>(h->H.size()))
    return set_error(BCMG_ERR_PARAM, "bad hierarchy index");
  const DevHierarchy &H = h->H[hrc];
  if (level < 0 || level >= static_cast<int>(H.lv.size()))
    return set_error(BCMG_ERR_PARAM, "bad level index");
  const DevLevel &lv = H.lv[level];
  const SlicedMat *S = h->mixed ? slicedlo(lv) : sliced64(lv);
  if (slots) *slots = S ? S->slots : 0;
  if (slices) *slices = S ? S->nslices : 0;
  if (value_bytes)
    *value_bytes = !S ? 0 : (S->vtype == kValF64 ? 8 : (S->vtype == kValF32 ? 4 : 2));
  if (column_slots) {
    *column_slots = 0;
    if (S && S->nslices) {
      std::vector<int4> meta(S->nslices);
      BCMG_CUDA(cudaSetDevice(h->device));
      BCMG_CUDA(cudaMemcpyAsync(meta.data(), S->meta, sizeof(int4) * S->nslices,
                                cudaMemcpyDeviceToHost, h->stream));
      BCMG_CUDA(cudaStreamSynchronize(h->stream));
      for (int32_t i = 0; i < S->nslices; ++i)
        if (!meta[i].z) *column_slots += meta[i].y;
    }
  }
  return BCMG_OK;
}

// ---- single-step entry points ------------------------------------------
bcmg_status bcmg_k_pair_aggregate(int32_t n, int32_t nnz, const int32_t *d_row,
                                  const int32_t *d_col, const double *d_val,
                                  const double *d_w, int32_t *d_agg, double *d_p,
                                  int32_t *n_coarse, double *d_W, int32_t *d_suitor,
                                  int32_t *d_match, void *stream) {
  clear_error();
  if (n <= 0 || !d_row || !d_col || !d_val || !d_w || !d_agg || !d_p || !n_coarse)
    return set_error(BCMG_ERR_PARAM, "bad arguments");
  CsrView A;
  A.n = n;
  A.nnz = nnz;
  A.row = d_row;
  A.col = d_col;
  A.val = d_val;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  BCMG_TRY(pair_aggregate(A, d_w, d_agg, d_p, n_coarse, d_W, d_suitor, d_match, s));
  BCMG_CUDA(cudaStreamSynchronize(s));
  return BCMG_OK;
}

bcmg_status bcmg_k_spgemm(int32_t n, int32_t m, int32_t x_nnz, const int32_t *d_xrow,
                          const int32_t *d_xcol, const double *d_xval, int32_t y_n,
                          int32_t y_nnz, const int32_t *d_yrow, const int32_t *d_ycol,
                          const double *d_yval, int32_t *d_crow, int32_t *c_nnz,
                          int32_t *d_ccol, double *d_cval, void *stream) {
  clear_error();
  if (n <= 0 || m <= 0 || y_n <= 0 || !d_xrow || !d_xcol || !d_xval || !d_yrow || !d_ycol ||
      !d_yval || !d_crow)
    return set_error(BCMG_ERR_PARAM, "bad arguments");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const CsrView X{n, x_nnz, d_xrow, d_xcol, d_xval};
  const CsrView Y{y_n, y_nnz, d_yrow, d_ycol, d_yval};
  int32_t *ccol = nullptr;
  double *cval = nullptr;
  int32_t cnnz = 0;
  BCMG_TRY(spgemm(X, Y, m, d_crow, &ccol, &cval, &cnnz, s));
  if (c_nnz) *c_nnz = cnnz;
  if (d_ccol && d_cval && cnnz > 0) {
    BCMG_CUDA(cudaMemcpyAsync(d_ccol, ccol, sizeof(int32_t) * cnnz, cudaMemcpyDeviceToDevice, s));
    BCMG_CUDA(cudaMemcpyAsync(d_cval, cval, sizeof(double) * cnnz, cudaMemcpyDeviceToDevice, s));
  }
  dev_free(ccol, s);
  dev_free(cval, s);
  BCMG_CUDA(cudaStreamSynchronize(s));
  return BCMG_OK;
}

bcmg_status bcmg_k_galerkin(int32_t n, int32_t nnz, const int32_t *d_row,
                            const int32_t *d_col, const double *d_val, int32_t n_coarse,
                            const int32_t *d_agg, const double *d_p, int32_t *d_crow,
                            int32_t *c_nnz, int32_t *d_ccol, double *d_cval, void *stream) {
  clear_error();
  if (n <= 0 || n_coarse <= 0 || !d_row || !d_col || !d_val || !d_agg || !d_p || !d_crow)
    return set_error(BCMG_ERR_PARAM, "bad arguments");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  CsrView A;
  A.n = n;
  A.nnz = nnz;
  A.row = d_row;
  A.col = d_col;
  A.val = d_val;
  DevBuf<int32_t> rptr, ridx;
  BCMG_TRY(rptr.alloc(n_coarse + 1, s));
  BCMG_TRY(ridx.alloc(n, s));
  BCMG_TRY(transpose_agg(n, d_agg, n_coarse, rptr.get(), ridx.get(), s));
  int32_t *ccol = nullptr;
  double *cval = nullptr;
  int32_t cnnz = 0;
  BCMG_TRY(galerkin(A, d_agg, d_p, n_coarse, rptr.get(), ridx.get(), d_crow, &ccol, &cval,
                    &cnnz, s));
  if (c_nnz) *c_nnz = cnnz;
  if (d_ccol && d_cval && cnnz > 0) {
    BCMG_CUDA(cudaMemcpyAsync(d_ccol, ccol, sizeof(int32_t) * cnnz, cudaMemcpyDeviceToDevice, s));
    BCMG_CUDA(cudaMemcpyAsync(d_cval, cval, sizeof(double) * cnnz, cudaMemcpyDeviceToDevice, s));
  }
  dev_free(ccol, s);
  dev_free(cval, s);
  BCMG_CUDA(cudaStreamSynchronize(s));
  return BCMG_OK;
}

bcmg_status bcmg_k_relax(int32_t n, int32_t nnz, const int32_t *d_row, const int32_t *d_col,
                         const double *d_val, const double *d_d, const double *d_f,
                         double *d_u, int k, void *stream) {
  clear_error();
  if (n <= 0 || !d_row || !d_col || !d_val || !d_d || !d_f || !d_u || k < 0)
    return set_error(BCMG_ERR_PARAM, "bad arguments");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  CsrView A;
  A.n = n;
  A.nnz = nnz;
  A.row = d_row;
  A.col = d_col;
  A.val = d_val;
  DevBuf<double> tmp;
  BCMG_TRY(tmp.alloc(n, s));
  BCMG_TRY(relax_t<double>(mat_f64(A), d_d, d_f, d_u, tmp.get(), k, false, s));
  BCMG_CUDA(cudaStreamSynchronize(s));
  return BCMG_OK;
}

bcmg_status bcmg_k_spmv(int32_t n, int32_t nnz, const int32_t *d_row, const int32_t *d_col,
                        const double *d_val, double alpha, const double *d_x, double beta,
                        double *d_y, void *stream) {
  clear_error();
  if (n <= 0 || !d_row || !d_col || !d_val || !d_x || !d_y)
    return set_error(BCMG_ERR_PARAM, "bad arguments");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  CsrView A;
  A.n = n;
  A.nnz = nnz;
  A.row = d_row;
  A.col = d_col;
  A.val = d_val;
  BCMG_TRY(spmv(A, alpha, d_x, beta, d_y, s));
  BCMG_CUDA(cudaStreamSynchronize(s));
  return BCMG_OK;
}

}  // extern "C"
