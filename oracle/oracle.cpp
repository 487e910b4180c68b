// oracle.cpp -- CPU FP64 restatement of BootCMatchG's alpha-AMG + FCG path.
//
// TEST INFRASTRUCTURE ONLY: the parity checker and the timed CPU baseline.
// Compiled with -ffp-contract=off so every FP64 operation is individually
// rounded; the GPU setup kernels are compiled the same way (--fmad=false),
// which makes hierarchies bit-identical on both sides.  Citations are to the
// BootCMatchG source tree.  Parity unpinned: see oracle.h.
#include "oracle.h"

#include <omp.h>

#include <algorithm>
#include <cfloat>
#include <chrono>
#include <cmath>
#include <cstring>
#include <memory>
#include <numeric>
#include <vector>

namespace {

using Vec = std::vector<double>;
using IVec = std::vector<int32_t>;

int g_threads = 0;

struct Csr {
  int32_t n = 0, m = 0;
  IVec row, col;
  Vec val;
  int32_t nnz() const { return static_cast<int32_t>(col.size()); }
};

// One level of a hierarchy.  P (level -> level+1) has one entry per fine row
// (unsmoothed aggregation): column agg[i], value p[i].  R = P^T is kept as
// the member lists of each aggregate in ascending order (rptr, ridx).
struct Level {
  std::shared_ptr<const Csr> A;
  Vec D, M, w;
  int32_t nc = 0;
  IVec agg, rptr, ridx;
  Vec p;
  // Smoothed aggregation (aggrtype 1): the smoothed prolongator and its
  // transpose replace (agg, p) and the member lists in the cycle.
  std::shared_ptr<const Csr> P, R;
};

struct Hierarchy {
  std::vector<Level> lv;
  double op_cmplx = 0, op_wcmplx = 0, avg_cratio = 0;
};

}  // namespace

struct orc_handle {
  bcmg_params prm;
  std::shared_ptr<const Csr> A0;
  std::vector<Hierarchy> H;
  double estimated_ratio = 1.0;
  int32_t maxcoarsesize = 0;
  IVec grid_sweeps;
  // cycle work buffers, per level of the deepest hierarchy
  std::vector<Vec> rhs, x, res;
  int kcycle_status = 0;  // BCMG_ERR_INDEFINITE once a K-cycle inner step broke down
};

namespace {

// ---------------------------------------------------------------------------
// Level preparation: relaxPrepare (src/AMG/matchingAggregation.cu:18-60).
// D_i = a_ii (_getDiagonal, src/matrix/CSR.cu:320-339: the loop keeps the
// last diagonal occurrence); M_i = sum_j |a_ij| in row order (_row_sum_2,
// src/matrix/CSR.cu:638-652).
void level_prep(const Csr &A, Vec &D, Vec &M) {
  D.assign(A.n, 0.0);
  M.assign(A.n, 0.0);
#pragma omp parallel for schedule(static)
  for (int32_t i = 0; i < A.n; ++i) {
    double s = 0.0;
    for (int32_t j = A.row[i]; j < A.row[i + 1]; ++j) {
      if (A.col[j] == i) D[i] = A.val[j];
      s += std::fabs(A.val[j]);
    }
    M[i] = s;
  }
}

// y = A x (sequential row sums).
void spmv(const Csr &A, const double *x, double *y) {
#pragma omp parallel for schedule(static)
  for (int32_t i = 0; i < A.n; ++i) {
    double t = 0.0;
    for (int32_t j = A.row[i]; j < A.row[i + 1]; ++j) t += A.val[j] * x[A.col[j]];
    y[i] = t;
  }
}

double dot(const double *a, const double *b, int32_t n) {
  double s = 0.0;
#pragma omp parallel for reduction(+ : s) schedule(static)
  for (int32_t i = 0; i < n; ++i) s += a[i] * b[i];
  return s;
}

// ||x||_A = sqrt(x' A x) (CSRm::vectorANorm, src/matrix/CSR.cu:360-368).
double anorm(const Csr &A, const Vec &x) {
  Vec t(A.n);
  spmv(A, x.data(), t.data());
  return std::sqrt(dot(t.data(), x.data(), A.n));
}

// ---------------------------------------------------------------------------
// Matching weights (Matching::makeAH + toMaximumProductMatrix):
//   C_i   = a_ii * w_i^2                         _makeC, matching.cu:141-162
//           (first diagonal occurrence: the loop breaks)
//   AH_ij = 1 - (2 a_ij w_i w_j) / (C_i + C_j)   _makeAH_warp, matching.cu:200-238
//           (DBL_EPSILON when C_i + C_j <= DBL_EPSILON; diagonal dropped)
//   mu    = min |AH_ij|                          find_Max_Min, matching.cu:401-431
//   W_ij  = log(|AH_ij| / (0.999 mu))            _make_w, matching.cu:387-395
// W is returned over A's own pattern with 0 on the diagonal: the matcher
// ignores weights <= 0 (suitor.cu:134), so the dropped diagonal needs no
// separate pattern.
void make_weights(const Csr &A, const Vec &w, Vec &W) {
  const int32_t n = A.n;
  Vec C(n, 0.0);
#pragma omp parallel for schedule(static)
  for (int32_t i = 0; i < n; ++i) {
    for (int32_t j = A.row[i]; j < A.row[i + 1]; ++j)
      if (A.col[j] == i) {
        C[i] = A.val[j] * (w[i] * w[i]);
        break;
      }
  }
  W.assign(A.nnz(), 0.0);
  double mu = DBL_MAX;
#pragma omp parallel for reduction(min : mu) schedule(static)
  for (int32_t i = 0; i < n; ++i) {
    for (int32_t j = A.row[i]; j < A.row[i + 1]; ++j) {
      const int32_t c = A.col[j];
      if (c == i) continue;
      const double norm = C[i] + C[c];
      double ah;
      if (norm > DBL_EPSILON) {
        const double wt = w[i] * w[c];
        ah = 1.0 - ((2.0 * A.val[j]) * wt) / norm;
      } else {
        ah = DBL_EPSILON;
      }
      W[j] = ah;
      mu = std::min(mu, std::fabs(ah));
    }
  }
  const double den = 0.999 * mu;
#pragma omp parallel for schedule(static)
  for (int32_t i = 0; i < n; ++i)
    for (int32_t j = A.row[i]; j < A.row[i + 1]; ++j) {
      if (A.col[j] == i) continue;
      W[j] = std::log(std::fabs(W[j]) / den);
    }
}

// Offer (weight, proposer) at a receiver; the receiver keeps the larger one,
// ties broken by the higher proposer id (suitor.cu:158).  An edge is usable
// only if its weight is > 0 (suitor.cu:134); NaN weights are never usable.
inline bool beats(double w, int32_t x, double cw, int32_t cid) {
  return w > cw || (w == cw && x > cid);
}

// Suitor matching (kernel_for_matching, suitor.cu:242-392; find_Candidate
// :118-214; set_suitor :49-114).  A proposer x offers to the neighbour y of
// largest (W_xy, y) whose current offer it beats (ties to the higher id,
// suitor.cu:144-145,197-203); y keeps the best offer and the displaced
// proposer searches again.  Offers only grow, so this is Gale-Shapley with
// strict preferences and its outcome does not depend on the processing
// order: the race-free reading of the reference's kernel.
void suitor_match(const Csr &A, const Vec &W, IVec &s) {
  const int32_t n = A.n;
  Vec ow(n, 0.0);
  s.assign(n, -1);
  for (int32_t v = 0; v < n; ++v) {
    int32_t cur = v;
    while (true) {
      int32_t by = -1;
      double bw = 0.0;
      for (int32_t e = A.row[cur]; e < A.row[cur + 1]; ++e) {
        const int32_t y = A.col[e];
        const double we = W[e];
        if (y == cur || !(we > 0.0)) continue;
        if (!beats(we, cur, ow[y], s[y])) continue;
        if (by < 0 || we > bw || (we == bw && y > by)) {
          by = y;
          bw = we;
        }
      }
      if (by < 0) break;
      const int32_t prev = s[by];
      s[by] = cur;
      ow[by] = bw;
      if (prev < 0) break;
      cur = prev;
    }
  }
}

// unsymFix (src/AMG/unsymMatching.cu:58-71).  Pass 1 (_setSymPair, :32-50):
// mutual suitors are matched.  Pass 2 (_setUnsymPair, :3-30): v with suitor
// u < v, both unmatched, claims u then itself with CAS and rolls back if v
// was claimed meanwhile.  The reference's pass 2 is racy; this resolves it
// as if all threads ran each step in lockstep (a valid interleaving): v gets
// u iff u is free after pass 1 and no other claimer targets v.  With a
// symmetric W the suitor array is already symmetric and pass 2 is a no-op.
void unsym_fix(const IVec &s, IVec &m) {
  const int32_t n = static_cast<int32_t>(s.size());
  m.assign(n, -1);
  for (int32_t v = 0; v < n; ++v) {
    const int32_t u = s[v];
    if (u >= 0 && s[u] == v) m[v] = u;
  }
  std::vector<char> claimer(n, 0), targeted(n, 0);
  for (int32_t v = 0; v < n; ++v) {
    const int32_t u = s[v];
    if (u >= 0 && u < v && m[v] == -1) claimer[v] = 1;
  }
  for (int32_t v = 0; v < n; ++v)
    if (claimer[v]) targeted[s[v]] = 1;
  IVec m2 = m;
  for (int32_t v = 0; v < n; ++v) {
    if (!claimer[v]) continue;
    const int32_t u = s[v];
    if (m[u] == -1 && !targeted[v]) {
      m2[v] = u;
      m2[u] = v;
    }
  }
  m.swap(m2);
}

// Pairwise aggregation (_aggregate_symmetric, matchingAggregation.cu:92-137).
// Matched pair {v < u}: p = w / ||(w_v, w_u)||_2 when the norm exceeds
// DBL_EPSILON, master v.  Otherwise each vertex is its own aggregate with
// p = w / |w| (good single) or 0 (|w| <= DBL_EPSILON, bad single).
// Numbering: the reference hands out coarse indices with atomicAdd (order
// not reproducible); here aggregates are numbered by ascending master
// vertex, i.e. the atomicAdds taken in thread order.
void aggregate(const IVec &m, const Vec &w, IVec &agg, Vec &p, int32_t &nc) {
  const int32_t n = static_cast<int32_t>(m.size());
  agg.assign(n, -1);
  p.assign(n, 0.0);
  std::vector<char> master(n, 0);
  std::vector<char> paired(n, 0);
#pragma omp parallel for schedule(static)
  for (int32_t v = 0; v < n; ++v) {
    const int32_t u = m[v];
    if (u >= 0) {
      const int32_t a = std::min(u, v), b = std::max(u, v);
      const double norm = std::sqrt(w[a] * w[a] + w[b] * w[b]);
      if (norm > DBL_EPSILON) {
        paired[v] = 1;
        if (v < u) master[v] = 1;
        p[v] = w[v] / norm;
        continue;
      }
    }
    master[v] = 1;
    p[v] = std::fabs(w[v]) > DBL_EPSILON ? w[v] / std::fabs(w[v]) : 0.0;
  }
  int32_t c = 0;
  for (int32_t v = 0; v < n; ++v)
    if (master[v]) agg[v] = c++;
  for (int32_t v = 0; v < n; ++v)
    if (paired[v] && !master[v]) agg[v] = agg[m[v]];
  nc = c;
}

// R = P^T as aggregate member lists, ascending (CSRm::T via csr2csc,
// src/matrix/CSR.cu:272-285, gives sorted rows).
void transpose_p(const IVec &agg, int32_t nc, IVec &rptr, IVec &ridx) {
  const int32_t n = static_cast<int32_t>(agg.size());
  rptr.assign(nc + 1, 0);
  for (int32_t i = 0; i < n; ++i) rptr[agg[i] + 1]++;
  for (int32_t I = 0; I < nc; ++I) rptr[I + 1] += rptr[I];
  ridx.assign(n, 0);
  IVec fill(rptr.begin(), rptr.end() - 1);
  for (int32_t i = 0; i < n; ++i) ridx[fill[agg[i]]++] = i;
}

// Galerkin product A_c = P^T A P (matchingAggregation.cu:239-244, computed
// there as R (A P) by two nsparse hash SpGEMMs with FP64 atomics).  The
// structure is the structural product -- explicit zeros stay, as in the
// hash SpGEMM -- with sorted columns.  Values: terms (p_i p_j) a_ij over
// i in I, j in J, summed from the first term in ascending
// (min(i,j), max(i,j), i) order; for an exactly symmetric A this order is
// the same for (I,J) and (J,I), so A_c is exactly symmetric.
struct Term {
  int32_t J, mn, mx, i;
  double t;
};

void galerkin(const Csr &A, const IVec &agg, const Vec &p, int32_t nc,
              const IVec &rptr, const IVec &ridx, Csr &C) {
  C.n = C.m = nc;
  C.row.assign(nc + 1, 0);
  std::vector<IVec> cols(nc);
  std::vector<Vec> vals(nc);
#pragma omp parallel
  {
    std::vector<Term> terms;
#pragma omp for schedule(dynamic, 256)
    for (int32_t I = 0; I < nc; ++I) {
      terms.clear();
      for (int32_t k = rptr[I]; k < rptr[I + 1]; ++k) {
        const int32_t i = ridx[k];
        for (int32_t e = A.row[i]; e < A.row[i + 1]; ++e) {
          const int32_t j = A.col[e];
          terms.push_back({agg[j], std::min(i, j), std::max(i, j), i,
                           (p[i] * p[j]) * A.val[e]});
        }
      }
      std::sort(terms.begin(), terms.end(), [](const Term &a, const Term &b) {
        if (a.J != b.J) return a.J < b.J;
        if (a.mn != b.mn) return a.mn < b.mn;
        if (a.mx != b.mx) return a.mx < b.mx;
        return a.i < b.i;
      });
      IVec &cc = cols[I];
      Vec &cv = vals[I];
      for (size_t t = 0; t < terms.size(); ++t) {
        if (t == 0 || terms[t].J != terms[t - 1].J) {
          cc.push_back(terms[t].J);
          cv.push_back(terms[t].t);
        } else {
          cv.back() = cv.back() + terms[t].t;
        }
      }
    }
  }
  for (int32_t I = 0; I < nc; ++I) C.row[I + 1] = C.row[I] + static_cast<int32_t>(cols[I].size());
  C.col.resize(C.row[nc]);
  C.val.resize(C.row[nc]);
#pragma omp parallel for schedule(static)
  for (int32_t I = 0; I < nc; ++I) {
    std::copy(cols[I].begin(), cols[I].end(), C.col.begin() + C.row[I]);
    std::copy(vals[I].begin(), vals[I].end(), C.val.begin() + C.row[I]);
  }
}

// w_c = R w (matchingAggregation.cu:253): members summed in ascending order.
void restrict_vec(const IVec &rptr, const IVec &ridx, const Vec &p, const double *x,
                  double *y, int32_t nc) {
#pragma omp parallel for schedule(static)
  for (int32_t I = 0; I < nc; ++I) {
    double s = 0.0;
    bool first = true;
    for (int32_t k = rptr[I]; k < rptr[I + 1]; ++k) {
      const int32_t i = ridx[k];
      const double t = p[i] * x[i];
      s = first ? t : s + t;
      first = false;
    }
    y[I] = s;
  }
}

// One matching + aggregation sweep (matchingPairAggregation,
// matchingAggregation.cu:181-208, with Matching::suitor, matching.cu:476-502).
void pair_aggregate(const Csr &A, const Vec &w, IVec &agg, Vec &p, int32_t &nc,
                    Vec *Wout, IVec *sout, IVec *mout) {
  Vec W;
  make_weights(A, w, W);
  IVec s, m;
  suitor_match(A, W, s);
  unsym_fix(s, m);
  aggregate(m, w, agg, p, nc);
  if (Wout) Wout->swap(W);
  if (sout) sout->swap(s);
  if (mout) mout->swap(m);
}

constexpr int kFtcoarseInc = 100;       // FTCOARSE_INC, matchingAggregation.cu:12
constexpr double kCoarseRatio = 1.2;    // COARSERATIO_THRSLD, matchingAggregation.cu:13

// matchingAggregation (matchingAggregation.cu:211-295): aggrsweeps pairwise
// sweeps composed into one prolongator; returns the coarse matrix, updates
// w to the coarse smooth vector and ftcoarse.
std::shared_ptr<Csr> matching_aggregation(const orc_handle &h, const Csr &A, Vec &w,
                                          int &ftcoarse, IVec &agg, Vec &p,
                                          int32_t &nc) {
  std::shared_ptr<const Csr> Ai_;
  const Csr *cur = &A;
  Vec wi_ = w;
  std::shared_ptr<Csr> Ai;
  for (int sweep = 0; sweep < h.prm.aggrsweeps; ++sweep) {
    IVec ag;
    Vec pv;
    int32_t nci = 0;
    pair_aggregate(*cur, wi_, ag, pv, nci, nullptr, nullptr, nullptr);
    IVec rptr, ridx;
    transpose_p(ag, nci, rptr, ridx);
    Ai = std::make_shared<Csr>();
    galerkin(*cur, ag, pv, nci, rptr, ridx, *Ai);
    Vec wi(nci);
    restrict_vec(rptr, ridx, pv, wi_.data(), wi.data(), nci);
    const double size_precoarse = cur->n;
    const double size_coarse = Ai->n;
    const double coarse_ratio = size_precoarse / size_coarse;
    if (sweep == 0) {
      agg.swap(ag);
      p.swap(pv);
    } else {
      // P = P * P_i: each row keeps one entry (matchingAggregation.cu:264).
      for (size_t i = 0; i < agg.size(); ++i) {
        const int32_t a = agg[i];
        p[i] = p[i] * pv[a];
        agg[i] = ag[a];
      }
    }
    nc = nci;
    wi_.swap(wi);
    if (coarse_ratio <= kCoarseRatio) ftcoarse = kFtcoarseInc;
    if (size_coarse <= static_cast<double>(ftcoarse * h.maxcoarsesize)) break;
    Ai_ = Ai;
    cur = Ai_.get();
  }
  w.swap(wi_);
  return Ai;
}

// C = X Y in the canonical order: row i's terms x_ik y_kj are generated by
// k in X's row order, then by Y's row order; a stable sort by column groups
// them and each column's terms are summed in generation order from the
// first term (the GPU kernel follows the same order, so C is bit-identical).
std::shared_ptr<Csr> spgemm(const Csr &X, const Csr &Y) {
  auto C = std::make_shared<Csr>();
  C->n = X.n;
  C->m = Y.m;
  C->row.assign(X.n + 1, 0);
  std::vector<IVec> cols(X.n);
  std::vector<Vec> vals(X.n);
#pragma omp parallel for schedule(dynamic, 256)
  for (int32_t i = 0; i < X.n; ++i) {
    std::vector<std::pair<int32_t, double>> t;
    for (int32_t a = X.row[i]; a < X.row[i + 1]; ++a) {
      const int32_t k = X.col[a];
      const double x = X.val[a];
      for (int32_t b = Y.row[k]; b < Y.row[k + 1]; ++b) t.emplace_back(Y.col[b], x * Y.val[b]);
    }
    std::stable_sort(t.begin(), t.end(),
                     [](const std::pair<int32_t, double> &u,
                        const std::pair<int32_t, double> &v) { return u.first < v.first; });
    for (size_t q = 0; q < t.size();) {
      double s = t[q].second;
      size_t e = q + 1;
      for (; e < t.size() && t[e].first == t[q].first; ++e) s = s + t[e].second;
      cols[i].push_back(t[q].first);
      vals[i].push_back(s);
      q = e;
    }
  }
  for (int32_t i = 0; i < X.n; ++i) C->row[i + 1] = C->row[i] + static_cast<int32_t>(cols[i].size());
  C->col.reserve(C->row[X.n]);
  C->val.reserve(C->row[X.n]);
  for (int32_t i = 0; i < X.n; ++i) {
    C->col.insert(C->col.end(), cols[i].begin(), cols[i].end());
    C->val.insert(C->val.end(), vals[i].begin(), vals[i].end());
  }
  return C;
}

// A^T with rows in increasing column order of A (csr2csc).
std::shared_ptr<Csr> transpose_csr(const Csr &A) {
  auto T = std::make_shared<Csr>();
  T->n = A.m;
  T->m = A.n;
  T->row.assign(A.m + 1, 0);
  for (int32_t c : A.col) ++T->row[c + 1];
  for (int32_t i = 0; i < A.m; ++i) T->row[i + 1] += T->row[i];
  T->col.resize(A.nnz());
  T->val.resize(A.nnz());
  IVec cur(T->row.begin(), T->row.end() - 1);
  for (int32_t i = 0; i < A.n; ++i)
    for (int32_t j = A.row[i]; j < A.row[i + 1]; ++j) {
      const int32_t q = cur[A.col[j]]++;
      T->col[q] = i;
      T->val[q] = A.val[j];
    }
  return T;
}

// Smoothed aggregation (adaptiveCoarsening, matchingAggregation.cu:353-390),
// applied to the built hierarchy: for each level j,
//   A_s = D_j^{-1} A_j (CSRm::matrixVectorScaling, CSR.cu:519-545),
//   omega = 4 / (3 ||A_s||_inf) (CSRm::infinityNorm, which the reference
//           stubs with assert(false), CSR.cu:402-417: the max absolute row sum),
//   S = I - omega A_s (applyOmega, matchingAggregation.cu:63-88),
//   P_j = S P_j, R_j = P_j^T, A_{j+1} = (R_j A_j) P_j, and relaxPrepare.
void smooth_hierarchy(Hierarchy &H) {
  const int L = static_cast<int>(H.lv.size());
  for (int j = 0; j + 1 < L; ++j) {
    Level &lv = H.lv[j];
    const Csr &A = *lv.A;
    Csr S = A;
    double inf = 0.0;
    for (int32_t i = 0; i < A.n; ++i) {
      double rs = 0.0;
      for (int32_t e = A.row[i]; e < A.row[i + 1]; ++e) {
        S.val[e] = A.val[e] / lv.D[i];
        rs = rs + std::fabs(S.val[e]);
      }
      inf = std::max(inf, rs);
    }
    const double omega = 4.0 / (3.0 * inf);
    for (int32_t i = 0; i < A.n; ++i)
      for (int32_t e = A.row[i]; e < A.row[i + 1]; ++e) {
        S.val[e] = -omega * S.val[e];
        if (A.col[e] == i) S.val[e] = S.val[e] + 1.0;
      }
    Csr Pt;
    Pt.n = A.n;
    Pt.m = lv.nc;
    Pt.row.resize(A.n + 1);
    std::iota(Pt.row.begin(), Pt.row.end(), 0);
    Pt.col = lv.agg;
    Pt.val = lv.p;
    lv.P = spgemm(S, Pt);
    lv.R = transpose_csr(*lv.P);
    auto RA = spgemm(*lv.R, A);
    auto Ac = spgemm(*RA, *lv.P);
    Level &c = H.lv[j + 1];
    c.A = Ac;
    level_prep(*Ac, c.D, c.M);
  }
}

// adaptiveCoarsening (matchingAggregation.cu:298-423).
Hierarchy adaptive_coarsening(const orc_handle &h, const Vec &w_in) {
  Hierarchy H;
  const int maxlevels = h.prm.max_levels;
  Vec w = w_in;
  const double normw = anorm(*h.A0, w);
  Level l0;
  l0.A = h.A0;
  level_prep(*h.A0, l0.D, l0.M);
  l0.w = w;
  H.lv.push_back(std::move(l0));
  int ftcoarse = 1;
  double avcoarseratio = 0.0;
  int level = 0;
  if (normw > DBL_EPSILON) {
    for (level = 1; level < maxlevels;) {
      Level &fine = H.lv[level - 1];
      Level nl;
      nl.A = matching_aggregation(h, *fine.A, w, ftcoarse, fine.agg, fine.p, fine.nc);
      transpose_p(fine.agg, fine.nc, fine.rptr, fine.ridx);
      level_prep(*nl.A, nl.D, nl.M);
      nl.w = w;
      const double size_coarse = nl.A->n;
      const double coarse_ratio = fine.A->n / size_coarse;
      avcoarseratio += coarse_ratio;
      H.lv.push_back(std::move(nl));
      ++level;
      if (size_coarse <= static_cast<double>(ftcoarse * h.maxcoarsesize)) break;
    }
  } else {
    // The reference asserts here (finalize_level with 0 levels); a single
    // level (smoother-only preconditioner) is used instead.
    level = 1;
  }
  if (h.prm.aggrtype == 1) smooth_hierarchy(H);
  double nnz0 = H.lv[0].A->nnz(), c = 0, cw = 0;
  for (size_t i = 0; i < H.lv.size(); ++i) {
    c += H.lv[i].A->nnz();
    cw += std::pow(2.0, static_cast<double>(i)) * H.lv[i].A->nnz();
  }
  H.op_cmplx = c / nnz0;
  H.op_wcmplx = cw / nnz0;
  H.avg_cratio = level > 1 ? avcoarseratio / (level - 1) : 0.0;
  return H;
}

// k unweighted Jacobi / l1-Jacobi sweeps (relax + jacobi_adaptive_miniwarp +
// _jacobi_it<0,MW>, src/AMG/relaxation.cu:176-285,357-377):
// u_i <- ((-(A u)_i + f_i) / d_i) + u_i.
void relax(const Csr &A, const Vec &d, const double *f, double *u, int k, Vec &tmp) {
  tmp.resize(A.n);
  for (int s = 0; s < k; ++s) {
#pragma omp parallel for schedule(static)
    for (int32_t i = 0; i < A.n; ++i) {
      double t = 0.0;
      for (int32_t j = A.row[i]; j < A.row[i + 1]; ++j) t += A.val[j] * u[A.col[j]];
      tmp[i] = ((-t + f[i]) / d[i]) + u[i];
    }
    std::memcpy(u, tmp.data(), sizeof(double) * A.n);
  }
}

// Grid-sweep table (ApplyData::setGridSweeps, src/AMG/AMG.cu:371-394).
IVec grid_sweeps(int cycle_type, int max_levels) {
  int ml = std::max(0, max_levels - 1);
  IVec g(std::max(ml, 1), 1);
  if (cycle_type == 1) {
    for (int i = 0; i < ml; ++i)
      if (i % 2 == 0) g[i] = 2;
  } else if (cycle_type == 2) {
    for (int i = 0; i < ml - 1; ++i) g[i] = 2;
  }
  return g;
}

void cycle(orc_handle &h, int k, int l);

// Relative reduction at which the K-cycle stops after its first inner step
// (RTOL, src/SOLVER/GAMG_cycle.cu:5).
constexpr double kKcycleRtol = 0.25;

// inneritkcycle (src/SOLVER/FCG.cu:633-723): two flexible-CG steps on the
// coarse level c (0-based) preconditioned by the cycle from that level
// (preconditionApplyK, FCG.cu:590-628, on fresh zero iterates); the result
// replaces x[c].  rhs[c] holds the right-hand side on entry.
void kcycle_inner(orc_handle &h, int k, int c) {
  const Csr &A = *h.H[k].lv[c].A;
  const int32_t n = A.n;
  Vec w(h.rhs[c].begin(), h.rhs[c].begin() + n);
  Vec d0(n), d1(n), v(n), v1(n), xk(n, 0.0);
  auto precond_k = [&](const Vec &r, Vec &d) {
    std::copy(r.begin(), r.end(), h.rhs[c].begin());
    std::fill(h.x[c].begin(), h.x[c].begin() + n, 0.0);
    cycle(h, k, c + 1);
    std::copy(h.x[c].begin(), h.x[c].begin() + n, d.begin());
  };
  auto axpy = [&](double a, const Vec &x, Vec &y) {
    for (int32_t i = 0; i < n; ++i) y[i] = a * x[i] + y[i];
  };
  const double delta0 = std::sqrt(dot(w.data(), w.data(), n));
  precond_k(w, d0);
  const double delta_old = dot(w.data(), d0.data(), n);
  spmv(A, d0.data(), v.data());
  const double tau = dot(d0.data(), v.data(), n);
  if (!(delta_old > 0.0) || !(tau > 0.0)) {
    // The reference exits the process here (FCG.cu:662-665, 676-679).
    h.kcycle_status = BCMG_ERR_INDEFINITE;
    std::fill(h.x[c].begin(), h.x[c].begin() + n, 0.0);
    return;
  }
  double alpha = delta_old / tau;
  axpy(-alpha, v, w);
  const double l2 = std::sqrt(dot(w.data(), w.data(), n));
  if (l2 <= kKcycleRtol * delta0) {
    axpy(alpha, d0, xk);
  } else {
    precond_k(w, d1);
    spmv(A, d1.data(), v1.data());
    const double tau1 = dot(d1.data(), v.data(), n);
    const double tau2 = dot(d1.data(), v1.data(), n);
    const double tau3 = dot(d1.data(), w.data(), n);
    const double tau4 = tau2 - (tau1 * tau1) / tau;
    alpha = alpha - (tau1 * tau3) / (tau * tau4);
    axpy(alpha, d0, xk);
    alpha = tau3 / tau4;
    axpy(alpha, d1, xk);
  }
  std::copy(xk.begin(), xk.end(), h.x[c].begin());
}

// GAMG_cycle (src/SOLVER/GAMG_cycle.cu:25-140), l is 1-based as there.
void cycle(orc_handle &h, int k, int l) {
  Hierarchy &H = h.H[k];
  const int L = static_cast<int>(H.lv.size());
  const bcmg_params &p = h.prm;
  Vec tmp;
  if (l == L) {
    Level &lv = H.lv[l - 1];
    relax(*lv.A, p.coarse_solver == 0 ? lv.D : lv.M, h.rhs[l - 1].data(),
          h.x[l - 1].data(), p.relaxnumber_coarse, tmp);
    return;
  }
  Level &lv = H.lv[l - 1];
  const Vec &d = p.relax_type == 0 ? lv.D : lv.M;
  const int32_t n = lv.A->n;
  relax(*lv.A, d, h.rhs[l - 1].data(), h.x[l - 1].data(), p.prerelax_sweeps, tmp);
  // Res = Rhs - A X (CSRVector_product_adaptive_miniwarp OP2, GAMG_cycle.cu:57-67)
  Vec &res = h.res[l - 1];
  spmv(*lv.A, h.x[l - 1].data(), res.data());
#pragma omp parallel for schedule(static)
  for (int32_t i = 0; i < n; ++i) res[i] = h.rhs[l - 1][i] - res[i];
  // Rhs_l = R Res (GAMG_cycle.cu:74-79)
  if (lv.R)
    spmv(*lv.R, res.data(), h.rhs[l].data());  // Rhs_l = R Res (GAMG_cycle.cu:74-79)
  else
    restrict_vec(lv.rptr, lv.ridx, lv.p, res.data(), h.rhs[l].data(), lv.nc);
  std::fill(h.x[l].begin(), h.x[l].begin() + lv.nc, 0.0);
  if (p.cycle_type == 3) {
    // K-cycle (GAMG_cycle.cu:88-100): the coarsest level is one cycle,
    // any other coarse level two inner flexible-CG steps.
    if (l == L - 1) cycle(h, k, l + 1);
    else kcycle_inner(h, k, l);
  } else {
    for (int i = 1; i <= h.grid_sweeps[l - 1]; ++i) {
      cycle(h, k, l + 1);
      if (l == L - 1) break;
    }
  }
  // X += P X_c (_CSR_vector_mul_prolongator, src/matrix/CSR.cu:965-976; the
  // general SpMV with beta = 1 for a smoothed P, GAMG_cycle.cu:116-117)
  double *xf = h.x[l - 1].data();
  const double *xc = h.x[l].data();
  if (lv.P) {
    const Csr &P = *lv.P;
#pragma omp parallel for schedule(static)
    for (int32_t i = 0; i < n; ++i) {
      double t = 0.0;
      for (int32_t e = P.row[i]; e < P.row[i + 1]; ++e) t += P.val[e] * xc[P.col[e]];
      xf[i] = xf[i] + t;
    }
  } else {
#pragma omp parallel for schedule(static)
    for (int32_t i = 0; i < n; ++i) xf[i] += lv.p[i] * xc[lv.agg[i]];
  }
  relax(*lv.A, d, h.rhs[l - 1].data(), xf, p.postrelax_sweeps, tmp);
}

// preconditionApply (src/SOLVER/FCG.cu:112-187).
void precond_apply(orc_handle &h, const double *rhs, double *x) {
  const int32_t n = h.A0->n;
  const int nh = static_cast<int>(h.H.size());
  auto run = [&](int k, const double *xin) {
    std::memcpy(h.rhs[0].data(), rhs, sizeof(double) * n);
    std::memcpy(h.x[0].data(), xin, sizeof(double) * n);
    cycle(h, k, 1);
  };
  if (h.prm.solver_type == 0) {
    for (int k = 0; k < nh; ++k) {
      run(k, x);
      std::memcpy(x, h.x[0].data(), sizeof(double) * n);
    }
  } else if (h.prm.solver_type == 1) {
    for (int k = 0; k < nh; ++k) {
      run(k, x);
      std::memcpy(x, h.x[0].data(), sizeof(double) * n);
    }
    for (int k = nh - 1; k >= 0; --k) {
      run(k, x);
      std::memcpy(x, h.x[0].data(), sizeof(double) * n);
    }
  } else {
    Vec xadd(n, 0.0);
    for (int k = 0; k < nh; ++k) {
      run(k, x);
      for (int32_t i = 0; i < n; ++i) xadd[i] += h.x[0][i];
    }
    const double alpha = 1.0 / static_cast<double>(nh);
    for (int32_t i = 0; i < n; ++i) x[i] = xadd[i] * alpha;
  }
}

void size_buffers(orc_handle &h) {
  size_t L = 0;
  for (auto &H : h.H) L = std::max(L, H.lv.size());
  h.rhs.resize(L);
  h.x.resize(L);
  h.res.resize(L);
  for (size_t l = 0; l < L; ++l) {
    int32_t nmax = 0;
    for (auto &H : h.H)
      if (l < H.lv.size()) nmax = std::max(nmax, H.lv[l].A->n);
    h.rhs[l].assign(nmax, 0.0);
    h.x[l].assign(nmax, 0.0);
    h.res[l].assign(nmax, 0.0);
  }
}

// Bootstrap::innerIterations (src/BOOT/bootstrap.cu:5-44).
void inner_iterations(orc_handle &h, Vec &w) {
  const Csr &A = *h.A0;
  Vec x(A.n, 1.0), rhs(A.n, 0.0);
  double normold = anorm(A, x), normnew = normold, conv = 1.0;
  const int solver_it = 15;  // BootBuildData::initDefault, AMG.cu:407
  for (int i = 1; i <= solver_it; ++i) {
    precond_apply(h, rhs.data(), x.data());
    normnew = anorm(A, x);
    conv = normnew / normold;
    normold = normnew;
  }
  const double alpha = 1.0 / normnew;
  for (int32_t i = 0; i < A.n; ++i) w[i] = x[i] * alpha;
  h.estimated_ratio = conv;
}

// Bootstrap::bootstrap (src/BOOT/bootstrap.cu:46-90).  After the first
// hierarchy the inner iterations are skipped (bootstrap.cu:68-75), so the
// second hierarchy is built from the same w = 1.
void bootstrap(orc_handle &h) {
  Vec w(h.A0->n, 1.0);  // BootBuildData::initByParams, AMG.cu:442-443
  h.estimated_ratio = 1.0;
  int num_hrc = 0;
  while (h.estimated_ratio > h.prm.conv_ratio && num_hrc < h.prm.max_hrc) {
    h.H.push_back(adaptive_coarsening(h, w));
    ++num_hrc;
    size_buffers(h);
    if (num_hrc > 1) inner_iterations(h, w);
  }
}

Csr from_bcmg(const bcmg_csr *A) {
  Csr c;
  c.n = A->n;
  c.m = A->m;
  c.row.assign(A->row, A->row + A->n + 1);
  c.col.assign(A->col, A->col + A->nnz);
  c.val.assign(A->val, A->val + A->nnz);
  return c;
}

Csr wrap(int32_t n, int32_t nnz, const int32_t *row, const int32_t *col,
         const double *val) {
  Csr c;
  c.n = c.m = n;
  c.row.assign(row, row + n + 1);
  c.col.assign(col, col + nnz);
  c.val.assign(val, val + nnz);
  return c;
}

// flexibileConjugateGradients_v3 (src/SOLVER/FCG.cu:433-585).
int fcg(orc_handle &h, const double *b, double *x, int itnlim, bcmg_solve_info *info,
        bool honour_exit) {
  const Csr &A = *h.A0;
  const int32_t n = A.n;
  Vec v(n, 0.0), w(n), r(n), d(n), q(n);
  spmv(A, x, w.data());
  for (int32_t i = 0; i < n; ++i) r[i] = b[i] - w[i];
  const double delta0 = std::sqrt(dot(r.data(), r.data(), n));
  const double rhs_norm = std::sqrt(dot(b, b, n));
  if (honour_exit && delta0 <= DBL_EPSILON * rhs_norm) {
    info->iters = 0;
    info->converged = 1;
    info->residual = delta0;
    info->rel_residual = 0.0;
    return BCMG_OK;
  }
  h.kcycle_status = 0;
  precond_apply(h, r.data(), v.data());
  if (h.kcycle_status) return h.kcycle_status;
  spmv(A, v.data(), w.data());
  double alpha = dot(r.data(), v.data(), n);
  double beta = dot(w.data(), v.data(), n);
  double delta = beta;
  double theta = alpha / delta;
  double gamma;
  for (int32_t i = 0; i < n; ++i) {
    x[i] += theta * v[i];
    r[i] -= theta * w[i];
  }
  double l2 = std::sqrt(dot(r.data(), r.data(), n));
  d = v;
  q = w;
  int iter = 0;
  int status = BCMG_OK;
  do {
    const int idx = iter % 2;
    Vec &z = idx == 0 ? v : d;   // current preconditioned residual
    Vec &az = idx == 0 ? w : q;  // A z
    Vec &zp = idx == 0 ? d : v;  // previous direction
    Vec &azp = idx == 0 ? q : w;
    std::fill(z.begin(), z.end(), 0.0);
    precond_apply(h, r.data(), z.data());
    if (h.kcycle_status) {
      status = h.kcycle_status;
      break;
    }
    spmv(A, z.data(), az.data());
    alpha = dot(r.data(), z.data(), n);
    beta = dot(az.data(), z.data(), n);
    gamma = dot(azp.data(), z.data(), n);
    double theta2;
    const double nd = beta - (gamma * gamma) / delta;
    if (nd > 0.0) {
      theta = gamma / delta;
      delta = nd;
      theta2 = alpha / delta;
    } else if (alpha == 0.0 && gamma == 0.0) {
      // Exact previous step (r = 0, z = 0): the reference divides 0 by 0
      // here (FCG.cu:531-534); treat the iteration as a no-op.
      theta = 0.0;
      theta2 = 0.0;
    } else {
      theta = gamma / delta;
      delta = nd;
      theta2 = alpha / delta;
      status = BCMG_ERR_INDEFINITE;
    }
#pragma omp parallel for schedule(static)
    for (int32_t i = 0; i < n; ++i) {
      const double zi = -theta * zp[i] + z[i];
      z[i] = zi;
      x[i] = theta2 * zi + x[i];
      const double ai = -theta * azp[i] + az[i];
      az[i] = ai;
      r[i] = -theta2 * ai + r[i];
    }
    l2 = std::sqrt(dot(r.data(), r.data(), n));
    ++iter;
    if (status != BCMG_OK) break;
  } while (l2 > h.prm.rtol * delta0 && iter < itnlim);
  info->iters = iter + 1;
  info->residual = l2;
  info->rel_residual = delta0 > 0 ? l2 / delta0 : 0.0;
  info->converged = l2 <= h.prm.rtol * delta0;
  return status;
}

}  // namespace

extern "C" {

// BuildData::setMaxCoarseSize (src/AMG/AMG.cu:309-311).
int32_t orc_max_coarse_size(int32_t n) {
  return static_cast<int32_t>(40 * std::pow(static_cast<double>(n), 1. / 3.));
}

int orc_grid_sweeps(int cycle_type, int max_levels, int32_t *out) {
  const IVec g = grid_sweeps(cycle_type, max_levels);
  const int k = std::max(0, max_levels - 1);
  for (int i = 0; i < k; ++i) out[i] = g[i];
  return k;
}

void orc_set_threads(int nthreads) {
  g_threads = nthreads;
  if (nthreads > 0) omp_set_num_threads(nthreads);
}

int orc_get_threads(void) { return omp_get_max_threads(); }

int orc_setup(const bcmg_csr *A, const bcmg_params *p, orc_handle **out) {
  if (!A || !p || !out) return BCMG_ERR_PARAM;
  if (p->aggrtype != 0 && p->aggrtype != 1) return BCMG_ERR_UNSUPPORTED;
  auto h = std::make_unique<orc_handle>();
  h->prm = *p;
  h->A0 = std::make_shared<Csr>(from_bcmg(A));
  h->maxcoarsesize = orc_max_coarse_size(A->n);
  h->grid_sweeps = grid_sweeps(p->cycle_type, p->max_levels);
  bootstrap(*h);
  *out = h.release();
  return BCMG_OK;
}

int orc_setup_from_w(const bcmg_csr *A, const bcmg_params *p, const double *w,
                     orc_handle **out) {
  if (!A || !p || !w || !out) return BCMG_ERR_PARAM;
  auto h = std::make_unique<orc_handle>();
  h->prm = *p;
  h->A0 = std::make_shared<Csr>(from_bcmg(A));
  h->maxcoarsesize = orc_max_coarse_size(A->n);
  h->grid_sweeps = grid_sweeps(p->cycle_type, p->max_levels);
  Vec wv(w, w + A->n);
  h->H.push_back(adaptive_coarsening(*h, wv));
  size_buffers(*h);
  *out = h.release();
  return BCMG_OK;
}

int orc_solve(orc_handle *h, const double *b, double *x, bcmg_solve_info *info) {
  if (!h || !b || !x || !info) return BCMG_ERR_PARAM;
  std::memset(info, 0, sizeof(*info));
  auto t0 = std::chrono::steady_clock::now();
  int st = fcg(*h, b, x, h->prm.itnlim, info, true);
  auto t1 = std::chrono::steady_clock::now();
  info->solve_ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
  info->num_hrc = static_cast<int>(h->H.size());
  info->estimated_ratio = h->estimated_ratio;
  Vec ax(h->A0->n);
  spmv(*h->A0, x, ax.data());
  double rr = 0, bb = 0;
  for (int32_t i = 0; i < h->A0->n; ++i) {
    rr += (b[i] - ax[i]) * (b[i] - ax[i]);
    bb += b[i] * b[i];
  }
  info->true_rel_residual = bb > 0 ? std::sqrt(rr / bb) : 0.0;
  return st;
}

int orc_fcg_sample(orc_handle *h, const double *b, double *x, int iters, double *seconds) {
  bcmg_solve_info info;
  std::memset(&info, 0, sizeof(info));
  auto t0 = std::chrono::steady_clock::now();
  int st = fcg(*h, b, x, iters, &info, false);
  auto t1 = std::chrono::steady_clock::now();
  if (seconds) *seconds = std::chrono::duration<double>(t1 - t0).count();
  return st;
}

int orc_precond_apply(orc_handle *h, const double *r, double *z) {
  if (!h) return BCMG_ERR_PARAM;
  precond_apply(*h, r, z);
  return BCMG_OK;
}

void orc_destroy(orc_handle *h) { delete h; }

int orc_hierarchy_count(const orc_handle *h, int *num_hrc, double *est_ratio) {
  if (!h) return BCMG_ERR_PARAM;
  if (num_hrc) *num_hrc = static_cast<int>(h->H.size());
  if (est_ratio) *est_ratio = h->estimated_ratio;
  return BCMG_OK;
}

int orc_hierarchy_info(const orc_handle *h, int hrc, int *num_levels, double *op_cmplx,
                       double *op_wcmplx, double *avg_cratio) {
  if (!h || hrc < 0 || hrc >= static_cast<int>(h->H.size())) return BCMG_ERR_PARAM;
  const Hierarchy &H = h->H[hrc];
  if (num_levels) *num_levels = static_cast<int>(H.lv.size());
  if (op_cmplx) *op_cmplx = H.op_cmplx;
  if (op_wcmplx) *op_wcmplx = H.op_wcmplx;
  if (avg_cratio) *avg_cratio = H.avg_cratio;
  return BCMG_OK;
}

int orc_level_info(const orc_handle *h, int hrc, int level, int32_t *n, int32_t *nnz,
                   int32_t *n_coarse) {
  if (!h || hrc < 0 || hrc >= static_cast<int>(h->H.size())) return BCMG_ERR_PARAM;
  const Hierarchy &H = h->H[hrc];
  if (level < 0 || level >= static_cast<int>(H.lv.size())) return BCMG_ERR_PARAM;
  const Level &lv = H.lv[level];
  if (n) *n = lv.A->n;
  if (nnz) *nnz = lv.A->nnz();
  if (n_coarse) *n_coarse = lv.nc;
  return BCMG_OK;
}

int orc_level_copy(const orc_handle *h, int hrc, int level, int32_t *row, int32_t *col,
                   double *val, double *D, double *M, int32_t *agg, double *p,
                   double *w) {
  if (!h || hrc < 0 || hrc >= static_cast<int>(h->H.size())) return BCMG_ERR_PARAM;
  const Hierarchy &H = h->H[hrc];
  if (level < 0 || level >= static_cast<int>(H.lv.size())) return BCMG_ERR_PARAM;
  const Level &lv = H.lv[level];
  const Csr &A = *lv.A;
  if (row) std::copy(A.row.begin(), A.row.end(), row);
  if (col) std::copy(A.col.begin(), A.col.end(), col);
  if (val) std::copy(A.val.begin(), A.val.end(), val);
  if (D) std::copy(lv.D.begin(), lv.D.end(), D);
  if (M) std::copy(lv.M.begin(), lv.M.end(), M);
  if (w) std::copy(lv.w.begin(), lv.w.end(), w);
  if (agg && !lv.agg.empty()) std::copy(lv.agg.begin(), lv.agg.end(), agg);
  if (p && !lv.p.empty()) std::copy(lv.p.begin(), lv.p.end(), p);
  return BCMG_OK;
}

int orc_pair_aggregate(int32_t n, int32_t nnz, const int32_t *row, const int32_t *col,
                       const double *val, const double *w, int32_t *agg, double *p,
                       int32_t *n_coarse, double *W, int32_t *suitor, int32_t *match) {
  Csr A = wrap(n, nnz, row, col, val);
  Vec wv(w, w + n), pv, Wv;
  IVec ag, s, m;
  int32_t nc = 0;
  pair_aggregate(A, wv, ag, pv, nc, &Wv, &s, &m);
  if (agg) std::copy(ag.begin(), ag.end(), agg);
  if (p) std::copy(pv.begin(), pv.end(), p);
  if (n_coarse) *n_coarse = nc;
  if (W) std::copy(Wv.begin(), Wv.end(), W);
  if (suitor) std::copy(s.begin(), s.end(), suitor);
  if (match) std::copy(m.begin(), m.end(), match);
  return BCMG_OK;
}

int orc_galerkin(int32_t n, int32_t nnz, const int32_t *row, const int32_t *col,
                 const double *val, int32_t n_coarse, const int32_t *agg, const double *p,
                 int32_t *crow, int32_t *c_nnz, int32_t *ccol, double *cval) {
  Csr A = wrap(n, nnz, row, col, val);
  IVec ag(agg, agg + n), rptr, ridx;
  Vec pv(p, p + n);
  transpose_p(ag, n_coarse, rptr, ridx);
  Csr C;
  galerkin(A, ag, pv, n_coarse, rptr, ridx, C);
  if (crow) std::copy(C.row.begin(), C.row.end(), crow);
  if (c_nnz) *c_nnz = C.nnz();
  if (ccol) std::copy(C.col.begin(), C.col.end(), ccol);
  if (cval) std::copy(C.val.begin(), C.val.end(), cval);
  return BCMG_OK;
}

// C = X Y in the canonical order of spgemm (X: n rows; Y: yn rows, m columns).
int orc_spgemm(int32_t n, int32_t xnnz, const int32_t *xrow, const int32_t *xcol,
               const double *xval, int32_t yn, int32_t m, int32_t ynnz, const int32_t *yrow,
               const int32_t *ycol, const double *yval, int32_t *crow, int32_t *c_nnz,
               int32_t *ccol, double *cval) {
  Csr X = wrap(n, xnnz, xrow, xcol, xval);
  Csr Y = wrap(yn, ynnz, yrow, ycol, yval);
  Y.m = m;
  auto C = spgemm(X, Y);
  if (crow) std::copy(C->row.begin(), C->row.end(), crow);
  if (c_nnz) *c_nnz = C->nnz();
  if (ccol) std::copy(C->col.begin(), C->col.end(), ccol);
  if (cval) std::copy(C->val.begin(), C->val.end(), cval);
  return BCMG_OK;
}

int orc_relax(int32_t n, const int32_t *row, const int32_t *col, const double *val,
              const double *d, const double *f, double *u, int k) {
  Csr A = wrap(n, row[n], row, col, val);
  Vec dv(d, d + n), tmp;
  relax(A, dv, f, u, k, tmp);
  return BCMG_OK;
}

int orc_spmv(int32_t n, const int32_t *row, const int32_t *col, const double *val,
             double alpha, const double *x, double beta, double *y) {
  for (int32_t i = 0; i < n; ++i) {
    double t = 0.0;
    for (int32_t j = row[i]; j < row[i + 1]; ++j) t += val[j] * x[col[j]];
    y[i] = alpha * t + (beta != 0.0 ? beta * y[i] : 0.0);
  }
  return BCMG_OK;
}

int orc_greedy_match(int32_t n, const int32_t *row, const int32_t *col, const double *W,
                     int32_t *match) {
  struct E {
    double w;
    int32_t hi, lo;
  };
  std::vector<E> edges;
  for (int32_t i = 0; i < n; ++i)
    for (int32_t j = row[i]; j < row[i + 1]; ++j) {
      const int32_t c = col[j];
      if (c > i && W[j] > 0.0) edges.push_back({W[j], c, i});
    }
  std::sort(edges.begin(), edges.end(), [](const E &a, const E &b) {
    if (a.w != b.w) return a.w > b.w;
    if (a.hi != b.hi) return a.hi > b.hi;
    return a.lo > b.lo;
  });
  for (int32_t i = 0; i < n; ++i) match[i] = -1;
  for (const E &e : edges)
    if (match[e.hi] < 0 && match[e.lo] < 0) {
      match[e.hi] = e.lo;
      match[e.lo] = e.hi;
    }
  return BCMG_OK;
}

}  // extern "C"
