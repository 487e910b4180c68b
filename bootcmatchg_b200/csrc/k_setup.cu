// Setup kernels: level preparation, matching weights, suitor matching,
// unsymFix, pairwise aggregation, P^T member lists, Galerkin product and
// w restriction.
//
// Built with --fmad=false: every FP64 operation here is individually rounded
// so that the hierarchy is bit-identical to the CPU oracle's (which is built
// with -ffp-contract=off and follows the same canonical orders).  All
// reductions whose order could vary are either exact (min, integer sums) or
// run in a fixed order, so setup is deterministic run to run.
#include <cfloat>
#include <climits>
#include <cmath>
#include <cstring>

#include "common.cuh"
#include "kernels.h"
#include "scan.cuh"

namespace bcmg {
namespace {

// ---------------------------------------------------------------------------
// relaxPrepare (src/AMG/matchingAggregation.cu:18-60): D_i = a_ii (last
// occurrence, _getDiagonal src/matrix/CSR.cu:320-339) and
// M_i = sum_j |a_ij| in row order (_row_sum_2, src/matrix/CSR.cu:638-652).
__global__ void k_level_prep(int32_t n, const int32_t *__restrict__ row,
                             const int32_t *__restrict__ col,
                             const double *__restrict__ val, double *D, double *M) {
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double d = 0.0, s = 0.0;
  for (int32_t j = row[i]; j < row[i + 1]; ++j) {
    const double a = val[j];
    if (col[j] == i) d = a;
    s = s + fabs(a);
  }
  D[i] = d;
  M[i] = s;
}

// C_i = a_ii * w_i^2 from the first diagonal occurrence (_makeC,
// src/AMG/matching.cu:141-162; pow(w,2) is the exactly rounded square).
__global__ void k_make_C(int32_t n, const int32_t *__restrict__ row,
                         const int32_t *__restrict__ col,
                         const double *__restrict__ val, const double *__restrict__ w,
                         double *C) {
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double c = 0.0;
  for (int32_t j = row[i]; j < row[i + 1]; ++j)
    if (col[j] == i) {
      c = val[j] * (w[i] * w[i]);
      break;
    }
  C[i] = c;
}

// AH_ij = 1 - (2 a_ij w_i w_j) / (C_i + C_j), or DBL_EPSILON when the
// denominator is <= DBL_EPSILON (_makeAH_warp, src/AMG/matching.cu:200-238).
__device__ __forceinline__ double ah_value(double a, double ci, double cj, double wi,
                                           double wj) {
  const double norm = ci + cj;
  if (norm > DBL_EPSILON) {
    const double wt = wi * wj;
    return 1.0 - ((2.0 * a) * wt) / norm;
  }
  return DBL_EPSILON;
}

template <int G>
__device__ __forceinline__ unsigned group_mask() {
  if (G == 32) return 0xffffffffu;
  return ((1u << (G & 31)) - 1u) << ((threadIdx.x & 31) & ~(G - 1));
}

// min |AH| over off-diagonal entries (find_Max_Min with AbsMin,
// src/AMG/matching.cu:319-329,401-431).  Grid-stride over rows, block
// reduction, one atomicMin per block: non-negative doubles order like their
// bit patterns, so the global min is an integer atomicMin (exact, order-free).
// A group of G lanes takes kMinRows rows at a time with the loads of each
// stage issued for all of them together (the pass is bound by the latency of
// the gathers of C and w, not by bandwidth).
constexpr int kMinRows = 2;

template <int G>
__global__ void __launch_bounds__(256)
    k_ah_min(int32_t n, const int32_t *__restrict__ row, const int32_t *__restrict__ col,
             const double *__restrict__ val, const double *__restrict__ w,
             const double *__restrict__ C, unsigned long long *min_bits) {
  __shared__ double wmin[8];
  const int lane = threadIdx.x % G;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x / G;
  double m = DBL_MAX;
  for (int64_t g0 = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) / G; g0 < n;
       g0 += kMinRows * stride) {
    int32_t i[kMinRows], b[kMinRows], e[kMinRows], c[kMinRows];
    double ci[kMinRows], wi[kMinRows], a[kMinRows], cc[kMinRows], wc[kMinRows];
#pragma unroll
    for (int u = 0; u < kMinRows; ++u) {
      const int64_t r = g0 + u * stride;
      i[u] = r < n ? static_cast<int32_t>(r) : -1;
      b[u] = e[u] = 0;
      ci[u] = wi[u] = 0.0;
      if (i[u] >= 0) {
        b[u] = row[i[u]];
        e[u] = row[i[u] + 1];
        ci[u] = C[i[u]];
        wi[u] = w[i[u]];
      }
    }
#pragma unroll
    for (int u = 0; u < kMinRows; ++u) {
      const int32_t j = b[u] + lane;
      c[u] = j < e[u] ? col[j] : -1;
      a[u] = j < e[u] ? val[j] : 0.0;
    }
#pragma unroll
    for (int u = 0; u < kMinRows; ++u) {
      cc[u] = wc[u] = 0.0;
      if (c[u] >= 0) {
        cc[u] = C[c[u]];
        wc[u] = w[c[u]];
      }
    }
#pragma unroll
    for (int u = 0; u < kMinRows; ++u) {
      if (c[u] >= 0 && c[u] != i[u]) {
        const double ah = fabs(ah_value(a[u], ci[u], cc[u], wi[u], wc[u]));
        if (ah < m) m = ah;
      }
      // entries past the first G of a long row
      for (int32_t j = b[u] + lane + G; j < e[u]; j += G) {
        const int32_t cj = col[j];
        if (cj == i[u]) continue;
        const double ah = fabs(ah_value(val[j], ci[u], C[cj], wi[u], w[cj]));
        if (ah < m) m = ah;
      }
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmin(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) wmin[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int k = 1; k < static_cast<int>(blockDim.x >> 5); ++k) m = fmin(m, wmin[k]);
    if (m < DBL_MAX)
      atomicMin(min_bits, static_cast<unsigned long long>(__double_as_longlong(m)));
  }
}

// W_ij = log(|AH_ij| / (0.999 mu)) (_make_w with MAXIMUM_PRODUCT_MATRIX_OP 1,
// src/AMG/matching.cu:387-395) is computed inside the preference sort
// (match_weight), so W is never stored unless a caller asks for it.

// Suitor matching (kernel_for_matching, src/AMG/suitor.cu:242-392).
//
// Preferences are static: proposer x ranks its neighbours y by (W_xy, y)
// descending (find_Candidate, suitor.cu:118-214, ties to the higher id), so
// each row is first sorted into that order (k_sort_prefs).  A proposer offers
// to the first neighbour in its sorted row whose current offer it beats; a
// receiver keeps the best offer under (weight, proposer id) (suitor.cu:158).
// Offers only increase, so a neighbour a proposer once could not beat (or was
// displaced from) stays unbeatable: each proposer resumes its scan where it
// stopped (next[]), and all proposals together read each row about once.
// With symmetric weights (every SPD input: W is bitwise symmetric when A is)
// an offer is the proposer's position in the receiver's own sorted row and a
// single atomicMin tests and installs it (k_suitor_sym).  Otherwise an offer
// is one 64-bit word (sorted position << 32 | proposer); the position
// recovers the immutable weight, so a CAS replaces the reference's per-vertex
// spin locks (suitor.cu:19-38,69-110).  A displaced proposer is
// taken over by the displacing thread (set_suitor, suitor.cu:89-93).  The
// final state is the proposer-optimal (Gale-Shapley) one, independent of the
// interleaving.  next[] is written without synchronisation: any value a
// thread can observe is a valid resume point (it never skips a neighbour
// that could still be beaten), so a stale read only costs a rescan.

// Position-ordered preference: a before b.
__device__ __forceinline__ bool pref_before(double wa, int32_t ya, double wb, int32_t yb) {
  return wa > wb || (wa == wb && ya > yb);
}

constexpr int kSortCapLong = 4096;  // entries per block (shared memory sort)
constexpr int kSortWarps = 4;
constexpr int kSortRegMax = 128;    // longest row sorted in registers (4 per lane)

// Within a row the columns are strictly increasing, so comparing original
// offsets t orders entries exactly as comparing their columns: the sort keys
// are (W, t) and ties go to the larger t (the higher column id).

// The matching weight of entry e = (i, c) (k_make_W formula); -1 marks an
// entry the matcher never uses (the diagonal, W <= 0, NaN).  W_out, when
// given, receives W over A's pattern with 0 on the diagonal.
__device__ __forceinline__ double match_weight(int32_t i, int32_t e, double ci, double wi,
                                               const int32_t *__restrict__ col,
                                               const double *__restrict__ val,
                                               const double *__restrict__ w,
                                               const double *__restrict__ C, double den,
                                               double *W_out) {
  const int32_t c = col[e];
  if (c == i) {
    if (W_out) W_out[e] = 0.0;
    return -1.0;
  }
  const double x = log(fabs(ah_value(val[e], ci, C[c], wi, w[c])) / den);
  if (W_out) W_out[e] = x;
  return x > 0.0 ? x : -1.0;
}

// Writes one sorted entry: scol/sW at sorted position pos, and the inverse
// permutation inv[b + t] = pos.
__device__ __forceinline__ void put_sorted(int32_t b, int pos, int t, double wv,
                                           const int32_t *__restrict__ col, double *sW,
                                           int32_t *scol, int32_t *inv) {
  sW[b + pos] = wv;
  scol[b + pos] = col[b + t];
  inv[b + t] = pos;
}

// Bitonic sort of 32*E (weight, offset) pairs held E per lane (position
// e*32 + lane) into preference order.
template <int E>
__device__ __forceinline__ void warp_bitonic(double (&wv)[E], int32_t (&tv)[E], int lane) {
#pragma unroll
  for (int k = 2; k <= 32 * E; k <<= 1) {
#pragma unroll
    for (int j = k >> 1; j > 0; j >>= 1) {
      if (j >= 32) {
#pragma unroll
        for (int e = 0; e < E; ++e) {
          const int f = e ^ (j >> 5);
          if (f > e) {
            const bool asc = ((e * 32 + lane) & k) == 0;
            const bool pb = pref_before(wv[f], tv[f], wv[e], tv[e]);
            if (asc ? pb : !pb) {
              const double tw = wv[e];
              wv[e] = wv[f];
              wv[f] = tw;
              const int32_t tt = tv[e];
              tv[e] = tv[f];
              tv[f] = tt;
            }
          }
        }
      } else {
#pragma unroll
        for (int e = 0; e < E; ++e) {
          const int p = e * 32 + lane;
          const double pw = __shfl_xor_sync(0xffffffffu, wv[e], j);
          const int32_t pt = __shfl_xor_sync(0xffffffffu, tv[e], j);
          const bool lower = (p & j) == 0;
          const bool asc = (p & k) == 0;
          const bool pb = pref_before(pw, pt, wv[e], tv[e]);  // partner ranks first
          if ((lower == asc) ? pb : !pb) {
            wv[e] = pw;
            tv[e] = pt;
          }
        }
      }
    }
  }
}

// A row's weights in registers (entry t at lane t % 32, register t / 32);
// -1 and offset -1 past the row's end.
template <int E>
__device__ __forceinline__ void row_weights(int32_t i, int32_t b, int T, double ci, double wi,
                                            const int32_t *__restrict__ col,
                                            const double *__restrict__ val,
                                            const double *__restrict__ w,
                                            const double *__restrict__ C, double den,
                                            double *W_out, double (&wv)[E], int32_t (&tv)[E],
                                            int lane) {
#pragma unroll
  for (int e = 0; e < E; ++e) {
    const int t = e * 32 + lane;
    wv[e] = -1.0;
    tv[e] = -1;
    if (t < T) {
      wv[e] = match_weight(i, b + t, ci, wi, col, val, w, C, den, W_out);
      tv[e] = t;
    }
  }
}

// Orders one row from its weights in registers and writes sW, scol, inv and
// ucnt.
template <int E>
__device__ __forceinline__ void order_row(int32_t i, int32_t b, int T, double (&wv)[E],
                                          int32_t (&tv)[E], const int32_t *__restrict__ col,
                                          double *sW, int32_t *scol, int32_t *inv,
                                          int32_t *ucnt, int lane) {
  int nu = 0;
#pragma unroll
  for (int e = 0; e < E; ++e) nu += wv[e] > 0.0 ? 1 : 0;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) nu += __shfl_xor_sync(0xffffffffu, nu, o);
  if (E == 1) {
    // All usable weights equal (a constant-coefficient stencil under w = 1):
    // the order is usable entries by offset descending, then the rest by
    // offset descending — positions from two ballots, no sort.
    const bool usable = wv[0] > 0.0;
    const unsigned U = __ballot_sync(0xffffffffu, usable);
    const unsigned Vd = __ballot_sync(0xffffffffu, tv[0] >= 0);
    const double wref = __shfl_sync(0xffffffffu, wv[0], U ? __ffs(U) - 1 : 0);
    if (__all_sync(0xffffffffu, !usable || wv[0] == wref)) {
      if (lane < T) {
        const unsigned above = static_cast<unsigned>((0xffffffffull << (lane + 1)) & 0xffffffffull);
        const int pos = usable ? __popc(U & above) : __popc(U) + __popc(Vd & ~U & above);
        put_sorted(b, pos, lane, wv[0], col, sW, scol, inv);
      }
      if (lane == 0) ucnt[i] = nu;
      return;
    }
  }
  warp_bitonic<E>(wv, tv, lane);
#pragma unroll
  for (int e = 0; e < E; ++e) {
    const int pos = e * 32 + lane;
    if (pos < T) put_sorted(b, pos, tv[e], wv[e], col, sW, scol, inv);
  }
  if (lane == 0) ucnt[i] = nu;
}

template <int E>
__device__ __forceinline__ void sort_row_regs(int32_t i, int32_t b, int T, double ci, double wi,
                                              const int32_t *__restrict__ col,
                                              const double *__restrict__ val,
                                              const double *__restrict__ w,
                                              const double *__restrict__ C, double den,
                                              double *W_out, double *sW, int32_t *scol,
                                              int32_t *inv, int32_t *ucnt, int lane) {
  double wv[E];
  int32_t tv[E];
  row_weights<E>(i, b, T, ci, wi, col, val, w, C, den, W_out, wv, tv, lane);
  order_row<E>(i, b, T, wv, tv, col, sW, scol, inv, ucnt, lane);
}

// Computes each row's matching weights and sorts the row into preference
// order: sW, scol, the inverse permutation inv (original offset -> sorted
// position) and the number of usable entries per row (ucnt).  One warp per
// kSortRowsPerWarp consecutive rows, in registers: when both rows have at
// most 32 entries their weights (and the gathers behind them) are computed
// before either is ordered, so the two rows' dependent loads overlap (the
// pass is latency-bound).  Longer rows are queued: up to kSortRegMax entries
// for k_sort_prefs_mid (2 or 4 entries per lane), beyond that for
// k_sort_prefs_long.  Keeping the multi-register sorts out of this kernel
// keeps its register count, and so the warps it has in flight, at what the
// rows of at most 32 entries need.
constexpr int kSortRowsPerWarp = 2;

__device__ __forceinline__ void sort_one_row(int32_t i, const int32_t *__restrict__ row,
                                             const int32_t *__restrict__ col,
                                             const double *__restrict__ val,
                                             const double *__restrict__ w,
                                             const double *__restrict__ C, double den,
                                             double *W_out, double *sW, int32_t *scol,
                                             int32_t *inv, int32_t *ucnt, int32_t *mid_rows,
                                             int32_t *n_mid, int32_t *long_rows,
                                             int32_t *n_long, int lane) {
  const int32_t b = row[i], T = row[i + 1] - b;
  if (T > kSortRegMax) {
    if (lane == 0) long_rows[atomicAdd(n_long, 1)] = i;
    return;
  }
  if (T > 32) {
    if (lane == 0) mid_rows[atomicAdd(n_mid, 1)] = i;
    return;
  }
  sort_row_regs<1>(i, b, T, C[i], w[i], col, val, w, C, den, W_out, sW, scol, inv, ucnt, lane);
}

// The queued rows of 33..kSortRegMax entries, one warp per row (warps take
// queue entries q, q + all warps, ...).
__global__ void __launch_bounds__(kSortWarps * 32)
    k_sort_prefs_mid(const int32_t *__restrict__ mid_rows, const int32_t *__restrict__ n_mid,
                     const int32_t *__restrict__ row, const int32_t *__restrict__ col,
                     const double *__restrict__ val, const double *__restrict__ w,
                     const double *__restrict__ C,
                     const unsigned long long *__restrict__ min_bits, double *W_out,
                     double *sW, int32_t *scol, int32_t *inv, int32_t *ucnt) {
  const int lane = threadIdx.x & 31;
  const int32_t nq = *n_mid;
  const int32_t warps = static_cast<int32_t>(gridDim.x) * kSortWarps;
  const double den = 0.999 * __longlong_as_double(static_cast<long long>(*min_bits));
  for (int32_t q = blockIdx.x * kSortWarps + (threadIdx.x >> 5); q < nq; q += warps) {
    const int32_t i = mid_rows[q];
    const int32_t b = row[i], T = row[i + 1] - b;
    const double ci = C[i], wi = w[i];
    if (T <= 64)
      sort_row_regs<2>(i, b, T, ci, wi, col, val, w, C, den, W_out, sW, scol, inv, ucnt, lane);
    else
      sort_row_regs<4>(i, b, T, ci, wi, col, val, w, C, den, W_out, sW, scol, inv, ucnt, lane);
  }
}

__global__ void __launch_bounds__(kSortWarps * 32)
    k_sort_prefs(int32_t n, const int32_t *__restrict__ row, const int32_t *__restrict__ col,
                 const double *__restrict__ val, const double *__restrict__ w,
                 const double *__restrict__ C,
                 const unsigned long long *__restrict__ min_bits, double *W_out, double *sW,
                 int32_t *scol, int32_t *inv, int32_t *ucnt, int32_t *mid_rows,
                 int32_t *n_mid, int32_t *long_rows, int32_t *n_long) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int32_t i0 = (blockIdx.x * kSortWarps + wid) * kSortRowsPerWarp;
  if (i0 >= n) return;
  const double den = 0.999 * __longlong_as_double(static_cast<long long>(*min_bits));
  const int32_t i1 = i0 + 1;
  const int32_t b0 = row[i0], e0 = row[i0 + 1];
  const int32_t e1 = i1 < n ? row[i1 + 1] : e0;
  const int T0 = e0 - b0, T1 = e1 - e0;
  if (i1 < n && T0 <= 32 && T1 <= 32) {
    const double ci0 = C[i0], wi0 = w[i0], ci1 = C[i1], wi1 = w[i1];
    double w0[1], w1[1];
    int32_t t0[1], t1[1];
    row_weights<1>(i0, b0, T0, ci0, wi0, col, val, w, C, den, W_out, w0, t0, lane);
    row_weights<1>(i1, e0, T1, ci1, wi1, col, val, w, C, den, W_out, w1, t1, lane);
    order_row<1>(i0, b0, T0, w0, t0, col, sW, scol, inv, ucnt, lane);
    order_row<1>(i1, e0, T1, w1, t1, col, sW, scol, inv, ucnt, lane);
    return;
  }
  sort_one_row(i0, row, col, val, w, C, den, W_out, sW, scol, inv, ucnt, mid_rows, n_mid,
               long_rows, n_long, lane);
  if (i1 < n)
    sort_one_row(i1, row, col, val, w, C, den, W_out, sW, scol, inv, ucnt, mid_rows, n_mid,
                 long_rows, n_long, lane);
}

// Same for the queued long rows, one block per row in shared memory: each
// block takes queue entries blockIdx.x, blockIdx.x + gridDim.x, ...
__global__ void __launch_bounds__(256)
    k_sort_prefs_long(const int32_t *__restrict__ long_rows, const int32_t *__restrict__ n_long,
                      const int32_t *__restrict__ row, const int32_t *__restrict__ col,
                      const double *__restrict__ val, const double *__restrict__ w,
                      const double *__restrict__ C,
                      const unsigned long long *__restrict__ min_bits, double *W_out,
                      double *sW, int32_t *scol, int32_t *inv, int32_t *ucnt, int *err) {
  extern __shared__ __align__(16) unsigned char sort_dyn[];
  __shared__ int nu_sh;
  double *ws = reinterpret_cast<double *>(sort_dyn);
  int32_t *ts = reinterpret_cast<int32_t *>(sort_dyn + sizeof(double) * kSortCapLong);
  const double den = 0.999 * __longlong_as_double(static_cast<long long>(*min_bits));
  for (int32_t q = blockIdx.x; q < *n_long; q += gridDim.x) {
    const int32_t i = long_rows[q];
    const int32_t b = row[i], T = row[i + 1] - b;
    if (T > kSortCapLong) {
      if (threadIdx.x == 0) atomicExch(err, 2);
      return;
    }
    if (threadIdx.x == 0) nu_sh = 0;
    __syncthreads();
    const double ci = C[i], wi = w[i];
    int P2 = 64;
    while (P2 < T) P2 <<= 1;
    int nu = 0;
    for (int t = threadIdx.x; t < P2; t += blockDim.x) {
      if (t < T) {
        ws[t] = match_weight(i, b + t, ci, wi, col, val, w, C, den, W_out);
        ts[t] = t;
        nu += ws[t] > 0.0 ? 1 : 0;
      } else {
        ws[t] = -1.0;
        ts[t] = -1;
      }
    }
    atomicAdd(&nu_sh, nu);
    __syncthreads();
    for (int k = 2; k <= P2; k <<= 1)
      for (int j = k >> 1; j > 0; j >>= 1) {
        for (int t = threadIdx.x; t < P2 / 2; t += blockDim.x) {
          const int i0 = ((t & ~(j - 1)) << 1) | (t & (j - 1)), i1 = i0 + j;  // j = 2^m
          const bool asc = (i0 & k) == 0;
          const bool swap = asc ? pref_before(ws[i1], ts[i1], ws[i0], ts[i0])
                                : pref_before(ws[i0], ts[i0], ws[i1], ts[i1]);
          if (swap) {
            const double tw = ws[i0];
            ws[i0] = ws[i1];
            ws[i1] = tw;
            const int32_t tt = ts[i0];
            ts[i0] = ts[i1];
            ts[i1] = tt;
          }
        }
        __syncthreads();
      }
    for (int t = threadIdx.x; t < T; t += blockDim.x)
      put_sorted(b, t, ts[t], ws[t], col, sW, scol, inv);
    if (threadIdx.x == 0) ucnt[i] = nu_sh;
    __syncthreads();
  }
}

// Symmetric weights: receiver y ranks proposers x by (W_xy, x) descending,
// which for W_xy = W_yx is y's own preference order, so an offer can be the
// proposer's position in y's sorted row.  For sorted usable entry k of row x
// pointing to y, E[k] packs what a proposal through it needs in one word:
// bits 0-31 y, bits 32-62 the index of x's entry in y's sorted row (row[y]
// plus the position; offers at one receiver compare like these indices), bit
// 63 set when k is x's last usable entry.  Any usable entry whose transposed
// entry is missing or carries a different weight (bit for bit) sets *nonsym,
// and the general matcher runs instead.
constexpr unsigned long long kLastEntry = 1ull << 63;

// One group of G lanes takes kKeyRows receiver rows at a time (one measured
// best: the full grid keeps more warps resident than interleaved rows with
// their registers do).  Usability comes from the sorted position
// (pa < ucnt[y]); the symmetry test compares the two values bit for bit,
// which is the same as comparing the two weights (both are computed from
// them by the same commutative expression).
constexpr int kKeyRows = 1;

template <int G>
__device__ __forceinline__ void sym_key_entry(int32_t y, int32_t by, int32_t ey, int32_t a,
                                              int32_t x, int32_t pa, double va,
                                              const int32_t *__restrict__ row,
                                              const int32_t *__restrict__ col,
                                              const double *__restrict__ val,
                                              const int32_t *__restrict__ inv,
                                              const int32_t *__restrict__ ucnt,
                                              unsigned long long *E, int *nonsym) {
  // the entry (x, y): first the mirrored position (a symmetric stencil row
  // of the same length holds y at index len - 1 - (a - by)), else a binary
  // search of y in row x (columns increasing)
  const int32_t bx = row[x], ex = row[x + 1];
  const int32_t ux = ucnt[x];
  int32_t lo = bx, hi = ex - 1;
  const int32_t guess = hi - (a - by);
  if (hi - lo == ey - 1 - by && col[guess] == y) {
    lo = hi = guess;
  } else {
    while (lo < hi) {
      const int32_t mid = (lo + hi) >> 1;
      if (col[mid] < y) lo = mid + 1;
      else hi = mid;
    }
  }
  if (lo > hi || col[lo] != y ||
      __double_as_longlong(val[lo]) != __double_as_longlong(va)) {
    atomicExch(nonsym, 1);
    return;
  }
  const int32_t pb = inv[lo];
  E[bx + pb] = (pb == ux - 1 ? kLastEntry : 0ull) |
               (static_cast<unsigned long long>(static_cast<uint32_t>(by + pa)) << 32) |
               static_cast<uint32_t>(y);
}

template <int G>
__global__ void __launch_bounds__(256)
    k_sym_keys(int32_t n, const int32_t *__restrict__ row, const int32_t *__restrict__ col,
               const double *__restrict__ val, const int32_t *__restrict__ inv,
               const int32_t *__restrict__ ucnt, unsigned long long *E, int *nonsym) {
  const int lane = threadIdx.x % G;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x / G;
  for (int64_t g0 = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) / G; g0 < n;
       g0 += kKeyRows * stride) {
    int32_t y[kKeyRows], by[kKeyRows], ey[kKeyRows], uy[kKeyRows];
    int32_t a[kKeyRows], x[kKeyRows], pa[kKeyRows];
    int32_t bx[kKeyRows], ex[kKeyRows], ux[kKeyRows], g[kKeyRows];
    double va[kKeyRows];
    bool ok[kKeyRows];
#pragma unroll
    for (int u = 0; u < kKeyRows; ++u) {
      const int64_t r = g0 + u * stride;
      y[u] = r < n ? static_cast<int32_t>(r) : -1;
      by[u] = ey[u] = uy[u] = 0;
      if (y[u] >= 0) {
        by[u] = row[y[u]];
        ey[u] = row[y[u] + 1];
        uy[u] = ucnt[y[u]];
      }
    }
#pragma unroll
    for (int u = 0; u < kKeyRows; ++u) {
      a[u] = by[u] + lane;
      x[u] = -1;
      pa[u] = 0;
      va[u] = 0.0;
      if (a[u] < ey[u]) {
        x[u] = col[a[u]];
        pa[u] = inv[a[u]];
        va[u] = val[a[u]];
      }
      ok[u] = x[u] >= 0 && x[u] != y[u] && pa[u] < uy[u];
    }
#pragma unroll
    for (int u = 0; u < kKeyRows; ++u) {
      bx[u] = ex[u] = ux[u] = 0;
      if (ok[u]) {
        bx[u] = row[x[u]];
        ex[u] = row[x[u] + 1];
        ux[u] = ucnt[x[u]];
      }
    }
    // the mirrored-position guess for every row at once
#pragma unroll
    for (int u = 0; u < kKeyRows; ++u) {
      g[u] = -1;
      if (ok[u] && ex[u] - 1 - bx[u] == ey[u] - 1 - by[u]) {
        const int32_t guess = ex[u] - 1 - (a[u] - by[u]);
        if (col[guess] == y[u] &&
            __double_as_longlong(val[guess]) == __double_as_longlong(va[u]))
          g[u] = guess;
      }
    }
#pragma unroll
    for (int u = 0; u < kKeyRows; ++u) {
      if (ok[u]) {
        if (g[u] >= 0) {
          const int32_t pb = inv[g[u]];
          E[bx[u] + pb] =
              (pb == ux[u] - 1 ? kLastEntry : 0ull) |
              (static_cast<unsigned long long>(static_cast<uint32_t>(by[u] + pa[u])) << 32) |
              static_cast<uint32_t>(y[u]);
        } else {
          sym_key_entry<G>(y[u], by[u], ey[u], a[u], x[u], pa[u], va[u], row, col, val, inv,
                           ucnt, E, nonsym);
        }
      }
      // entries past the first G of a long row
      for (int32_t aa = by[u] + lane + G; aa < ey[u]; aa += G) {
        const int32_t xx = col[aa];
        const int32_t pp = inv[aa];
        if (xx == y[u] || pp >= uy[u]) continue;
        sym_key_entry<G>(y[u], by[u], ey[u], aa, xx, pp, val[aa], row, col, val, inv, ucnt, E,
                         nonsym);
      }
    }
  }
}

// Suitor with symmetric weights.  offer[y] = (index of the current suitor's
// entry in y's sorted row) << 32 | (the suitor's own sorted entry index k of
// that proposal, bit 31 set if k is its last usable entry), kNoOffer if
// none.  The high half orders offers (smaller is better, unique per
// proposer), so one 64-bit atomicMin tests and installs an offer and returns
// the displaced one; the low half says where the displaced proposer resumes
// (k + 1, its candidates before k having rejected it for good), so taking a
// displaced proposer over costs one load of E[k + 1] and no per-vertex state.
// Proposer v starts at its first sorted entry; the thread's next candidate is
// loaded while the atomic is in flight.  Threads take the proposers from the
// highest id down: on tied weights a receiver prefers the higher proposer,
// so the winners tend to arrive first and fewer offers are displaced (the
// final state does not depend on the order).  Exits at once when *nonsym is
// set.
__global__ void __launch_bounds__(256)
    k_suitor_sym(int32_t n, const int32_t *__restrict__ row, const int32_t *__restrict__ ucnt,
                 const unsigned long long *__restrict__ E, unsigned long long *offer,
                 int64_t limit, const int *__restrict__ nonsym, int *err) {
  const int32_t gid = blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= n || *nonsym) return;
  const int32_t v = n - 1 - gid;
  if (ucnt[v] <= 0) return;
  uint32_t k = static_cast<uint32_t>(row[v]);
  unsigned long long ek = E[k];
  int64_t steps = 0;
  while (true) {
    if (++steps > limit) {
      atomicExch(err, 1);
      return;
    }
    const bool last = (ek & kLastEntry) != 0;
    const uint32_t y = static_cast<uint32_t>(ek);
    const unsigned long long mine = (ek & 0x7fffffff00000000ull) | k |
                                    (last ? 0x80000000ull : 0ull);
    unsigned long long en = 0;
    if (!last) en = E[k + 1];  // in flight with the atomic
    const unsigned long long old = atomicMin(offer + y, mine);
    if (old > mine) {
      if (old == kNoOffer) return;
      if (old & 0x80000000ull) return;  // the displaced proposer has no candidate left
      k = static_cast<uint32_t>(old & 0x7fffffffull) + 1u;
      ek = E[k];
      continue;
    }
    if (last) return;
    ++k;
    ek = en;
  }
}

// One thread per initial proposer; `limit` bounds the steps of a thread
// (advances, successful and failed CASes); on overrun *err is raised.  Used
// when the weights are not symmetric (exits at once otherwise).
__global__ void __launch_bounds__(256)
    k_suitor(int32_t n, const int32_t *__restrict__ row, const int32_t *__restrict__ scol,
             const double *__restrict__ sW, int32_t *next, unsigned long long *offer,
             int64_t limit, const int *__restrict__ nonsym, int *err) {
  const int32_t gid = blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= n || !*nonsym) return;
  volatile unsigned long long *voffer = offer;
  volatile int32_t *vnext = next;
  int32_t cur = gid;
  int64_t steps = 0;
  while (true) {
    int32_t k = vnext[cur];
    const int32_t e = row[cur + 1];
    unsigned long long won = kNoOffer;
    bool found = false;
    while (k < e) {
      if (++steps > limit) {
        atomicExch(err, 1);
        return;
      }
      const double wk = sW[k];
      if (!(wk > 0.0)) {
        k = e;
        break;
      }
      const int32_t y = scol[k];
      const unsigned long long o = voffer[y];
      double cw = 0.0;
      int32_t cid = -1;
      if (o != kNoOffer) {
        cw = sW[static_cast<int32_t>(o >> 32)];
        cid = static_cast<int32_t>(o & 0xffffffffull);
      }
      if (wk > cw || (wk == cw && cur > cid)) {
        const unsigned long long mine =
            (static_cast<unsigned long long>(static_cast<uint32_t>(k)) << 32) |
            static_cast<uint32_t>(cur);
        if (atomicCAS(offer + y, o, mine) == o) {
          won = o;
          found = true;
          break;
        }
        continue;  // the offer changed: test the same neighbour again
      }
      ++k;
    }
    vnext[cur] = found ? k + 1 : e;
    if (!found || won == kNoOffer) return;
    cur = static_cast<int32_t>(won & 0xffffffffull);  // the displaced proposer
  }
}

// Resume points at each row's start; no offers yet.
__global__ void k_init_match(int32_t n, const int32_t *__restrict__ row, int32_t *next,
                             unsigned long long *offer) {
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  next[i] = row[i];
  offer[i] = kNoOffer;
}

// Suitor array from whichever matcher ran: the general matcher keeps the
// proposer in the offer's low 32 bits; the symmetric one keeps the index of
// the proposer's entry in the receiver's own sorted row in the high half,
// whose column is the proposer.
__global__ void k_offer_to_suitor(int32_t n, const unsigned long long *__restrict__ offer,
                                  const int32_t *__restrict__ scol,
                                  const int *__restrict__ nonsym, int32_t *s) {
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const unsigned long long o = offer[i];
  if (o == kNoOffer) {
    s[i] = -1;
    return;
  }
  s[i] = *nonsym ? static_cast<int32_t>(o & 0xffffffffull) : scol[o >> 32];
}

// unsymFix pass 1 (_setSymPair, src/AMG/unsymMatching.cu:32-50).
__global__ void k_sym_pairs(int32_t n, const int32_t *__restrict__ s, int32_t *m) {
  const int32_t v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= n) return;
  const int32_t u = s[v];
  m[v] = (u >= 0 && s[u] == v) ? u : -1;
}

// unsymFix pass 2 (_setUnsymPair, src/AMG/unsymMatching.cu:3-30) resolved as
// if every thread took each CAS step in lockstep: claimer v (suitor u < v,
// v unmatched) gets u iff u is unmatched and no other claimer targets v.
__global__ void k_unsym_targets(int32_t n, const int32_t *__restrict__ s,
                                const int32_t *__restrict__ m, int32_t *targeted) {
  const int32_t v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= n) return;
  const int32_t u = s[v];
  if (u >= 0 && u < v && m[v] == -1) targeted[u] = 1;
}

__global__ void k_unsym_pairs(int32_t n, const int32_t *__restrict__ s,
                              const int32_t *__restrict__ m,
                              const int32_t *__restrict__ targeted, int32_t *m2) {
  const int32_t v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= n) return;
  const int32_t u = s[v];
  if (u >= 0 && u < v && m[v] == -1 && m[u] == -1 && !targeted[v]) {
    m2[v] = u;
    m2[u] = v;
  }
}

// _aggregate_symmetric (src/AMG/matchingAggregation.cu:92-137), first half:
// prolongator values and "is aggregate master" flags.
__global__ void k_agg_flags(int32_t n, const int32_t *__restrict__ m,
                            const double *__restrict__ w, int32_t *master, double *p) {
  const int32_t v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= n) return;
  const int32_t u = m[v];
  const double wv = w[v];
  if (u >= 0) {
    const int32_t a = min(u, v), b = max(u, v);
    const double wa = w[a], wb = w[b];
    const double norm = sqrt(wa * wa + wb * wb);
    if (norm > DBL_EPSILON) {
      master[v] = v < u ? 1 : 0;
      p[v] = wv / norm;
      return;
    }
  }
  master[v] = 1;
  p[v] = fabs(wv) > DBL_EPSILON ? wv / fabs(wv) : 0.0;
}

// Second half: coarse index = rank of the aggregate's master (the reference
// numbers with atomicAdd; this is that numbering in thread order).
__global__ void k_agg_assign(int32_t n, const int32_t *__restrict__ m,
                             const int32_t *__restrict__ master,
                             const int32_t *__restrict__ rank, int32_t *agg) {
  const int32_t v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= n) return;
  agg[v] = master[v] ? rank[v] : rank[m[v]];
}

// Aggregate sizes; an out-of-range coarse index raises *err and is skipped.
__global__ void k_count_agg(int32_t n, const int32_t *__restrict__ agg, int32_t nc,
                            int32_t *cnt, int *err) {
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int32_t I = agg[i];
  if (I < 0 || I >= nc) {
    atomicExch(err, 1);
    return;
  }
  atomicAdd(cnt + I, 1);
}

__global__ void k_fill_agg(int32_t n, const int32_t *__restrict__ agg, int32_t nc,
                           const int32_t *__restrict__ rptr, int32_t *cursor,
                           int32_t *ridx) {
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int32_t I = agg[i];
  if (I < 0 || I >= nc) return;
  ridx[rptr[I] + atomicAdd(cursor + I, 1)] = i;
}

// Members of each aggregate in ascending order (CSRm::T via csr2csc gives
// sorted rows, src/matrix/CSR.cu:272-285).
__global__ void k_sort_segments(int32_t nc, const int32_t *__restrict__ rptr,
                                int32_t *ridx) {
  const int32_t I = blockIdx.x * blockDim.x + threadIdx.x;
  if (I >= nc) return;
  const int32_t b = rptr[I], e = rptr[I + 1];
  for (int32_t k = b + 1; k < e; ++k) {
    const int32_t x = ridx[k];
    int32_t j = k - 1;
    while (j >= b && ridx[j] > x) {
      ridx[j + 1] = ridx[j];
      --j;
    }
    ridx[j + 1] = x;
  }
}

// ---------------------------------------------------------------------------
// Galerkin product A_c = P^T A P for one-entry-per-row P.  The reference
// forms R (A P) with two nsparse hash SpGEMMs whose FP64 shared-memory
// atomics sum in a nondeterministic order
// (kernel_spgemm_hash_d.cu:631-1027).  Here each coarse row I is built by a
// team (a warp, or a whole block for long rows): it gathers the terms
// (p_i p_j) a_ij of its members i, sorts them by coarse column J, and sums
// each J-run in ascending (min(i,j), max(i,j), i) order starting from the
// first term.  That order is symmetric in (i,j), so an exactly symmetric A
// gives an exactly symmetric A_c; the structure is the structural product
// (explicit zeros kept), columns ascending, as nsparse produces.
constexpr int kGalCap = 256;       // terms per warp team
constexpr int kGalCapLong = 4096;  // terms per block team
constexpr int kGalMaxRun = 16;     // terms per (I,J): |I| * |J|
constexpr int kGalWarpsPerBlock = 4;
constexpr int kGalLongThreads = 256;

struct GalSmem {
  unsigned long long *key;
  double *tv;
  int32_t *ti;
  int32_t *tj;
  int32_t *heads;  // first position of each run (gal_emit)
};

__device__ __forceinline__ GalSmem gal_smem(unsigned char *base, int cap) {
  GalSmem s;
  s.key = reinterpret_cast<unsigned long long *>(base);
  s.tv = reinterpret_cast<double *>(base + sizeof(unsigned long long) * cap);
  s.ti = reinterpret_cast<int32_t *>(base + 16 * cap);
  s.tj = reinterpret_cast<int32_t *>(base + 20 * cap);
  s.heads = reinterpret_cast<int32_t *>(base + 24 * cap);
  return s;
}
constexpr int kGalBytesPerTerm = 28;

template <int TEAM>
__device__ __forceinline__ void team_sync() {
  if (TEAM == 32)
    __syncwarp();
  else
    __syncthreads();
}

// Gathers the terms of coarse row I and sorts them by (J, gather position).
// Returns the term count, or -1 when it exceeds cap.
template <int TEAM>
__device__ int gal_gather(int32_t I, const int32_t *__restrict__ row,
                          const int32_t *__restrict__ col,
                          const double *__restrict__ val,
                          const int32_t *__restrict__ agg,
                          const double *__restrict__ p,
                          const int32_t *__restrict__ rptr,
                          const int32_t *__restrict__ ridx, GalSmem sm, int cap,
                          int tid) {
  const int32_t kb = rptr[I], ke = rptr[I + 1];
  int T = 0;
  for (int32_t k = kb; k < ke; ++k) {
    const int32_t i = ridx[k];
    T += row[i + 1] - row[i];
  }
  if (T > cap) return -1;
  int base = 0;
  for (int32_t k = kb; k < ke; ++k) {
    const int32_t i = ridx[k];
    const int32_t b = row[i];
    const int len = row[i + 1] - b;
    const double pi = p[i];
    for (int t = tid; t < len; t += TEAM) {
      const int32_t e = b + t;
      const int32_t j = col[e];
      const int pos = base + t;
      sm.key[pos] = (static_cast<unsigned long long>(static_cast<uint32_t>(agg[j])) << 32) |
                    static_cast<uint32_t>(pos);
      sm.tv[pos] = (pi * p[j]) * val[e];
      sm.ti[pos] = i;
      sm.tj[pos] = j;
    }
    base += len;
  }
  int P2 = 1;
  while (P2 < T) P2 <<= 1;
  for (int t = T + tid; t < P2; t += TEAM) sm.key[t] = ~0ull;
  team_sync<TEAM>();
  // Bitonic sort of P2 keys (all distinct below T).
  for (int k = 2; k <= P2; k <<= 1) {
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int t = tid; t < P2 / 2; t += TEAM) {
        const int i0 = ((t & ~(j - 1)) << 1) | (t & (j - 1));  // j = 2^m
        const int i1 = i0 + j;
        const bool asc = (i0 & k) == 0;
        const unsigned long long a = sm.key[i0], b = sm.key[i1];
        if ((a > b) == asc) {
          sm.key[i0] = b;
          sm.key[i1] = a;
        }
      }
      team_sync<TEAM>();
    }
  }
  return T;
}

__device__ __forceinline__ bool gal_head(const GalSmem &sm, int k) {
  return k == 0 || (sm.key[k] >> 32) != (sm.key[k - 1] >> 32);
}

// Sums the run of len terms starting at sorted position k; returns false if
// the run is longer than kGalMaxRun.
// Canonical-order compare-exchange of two run terms (a before b after it).
__device__ __forceinline__ void gal_cx(int &ia, int32_t &mna, int32_t &mxa, int32_t &ta, int &ib,
                                       int32_t &mnb, int32_t &mxb, int32_t &tb) {
  const bool greater = mna > mnb || (mna == mnb && (mxa > mxb || (mxa == mxb && ta > tb)));
  if (greater) {
    int t0 = ia; ia = ib; ib = t0;
    int32_t t1 = mna; mna = mnb; mnb = t1;
    t1 = mxa; mxa = mxb; mxb = t1;
    t1 = ta; ta = tb; tb = t1;
  }
}

__device__ bool gal_run_sum(const GalSmem &sm, int k, int len, int32_t *J, double *sum) {
  const unsigned long long jj = sm.key[k] >> 32;
  if (len <= 4) {
    // Runs of at most four terms (pairwise aggregates: |I| |J| <= 4): a
    // four-input sorting network on (min(i,j), max(i,j), i) in registers;
    // absent terms carry INT_MAX keys and sort last.
    int id[4];
    int32_t mn[4], mx[4], ti[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const bool ok = q < len;
      id[q] = ok ? static_cast<int>(sm.key[k + q] & 0xffffffffull) : 0;
      const int32_t a = ok ? sm.ti[id[q]] : INT_MAX, b = ok ? sm.tj[id[q]] : INT_MAX;
      ti[q] = a;
      mn[q] = min(a, b);
      mx[q] = max(a, b);
    }
    gal_cx(id[0], mn[0], mx[0], ti[0], id[1], mn[1], mx[1], ti[1]);
    gal_cx(id[2], mn[2], mx[2], ti[2], id[3], mn[3], mx[3], ti[3]);
    gal_cx(id[0], mn[0], mx[0], ti[0], id[2], mn[2], mx[2], ti[2]);
    gal_cx(id[1], mn[1], mx[1], ti[1], id[3], mn[3], mx[3], ti[3]);
    gal_cx(id[1], mn[1], mx[1], ti[1], id[2], mn[2], mx[2], ti[2]);
    double s = sm.tv[id[0]];
#pragma unroll
    for (int q = 1; q < 4; ++q)
      if (q < len) s = s + sm.tv[id[q]];
    *J = static_cast<int32_t>(jj);
    *sum = s;
    return true;
  }
  if (len > kGalMaxRun) return false;
  int idx[kGalMaxRun];
  const int r = len;
  for (int q = 0; q < r; ++q) idx[q] = static_cast<int>(sm.key[k + q] & 0xffffffffull);
  // Insertion sort of the run by (min(i,j), max(i,j), i).
  for (int a = 1; a < r; ++a) {
    const int x = idx[a];
    const int32_t xi = sm.ti[x], xj = sm.tj[x];
    const int32_t xmn = min(xi, xj), xmx = max(xi, xj);
    int b = a - 1;
    while (b >= 0) {
      const int y = idx[b];
      const int32_t yi = sm.ti[y], yj = sm.tj[y];
      const int32_t ymn = min(yi, yj), ymx = max(yi, yj);
      const bool greater = ymn > xmn || (ymn == xmn && (ymx > xmx || (ymx == xmx && yi > xi)));
      if (!greater) break;
      idx[b + 1] = idx[b];
      --b;
    }
    idx[b + 1] = x;
  }
  double s = sm.tv[idx[0]];
  for (int a = 1; a < r; ++a) s = s + sm.tv[idx[a]];
  *J = static_cast<int32_t>(jj);
  *sum = s;
  return true;
}

// Term count of each coarse row: the summed lengths of its members' rows.
__global__ void k_gal_terms(int32_t nc, const int32_t *__restrict__ row,
                            const int32_t *__restrict__ rptr,
                            const int32_t *__restrict__ ridx, int32_t *tcount) {
  const int32_t I = blockIdx.x * blockDim.x + threadIdx.x;
  if (I >= nc) return;
  int32_t t = 0;
  for (int32_t k = rptr[I]; k < rptr[I + 1]; ++k) {
    const int32_t i = ridx[k];
    t += row[i + 1] - row[i];
  }
  tcount[I] = t;
}

// Writes the runs of a sorted coarse row: (J, sum) at tJ/tV[base + rank] and
// the number of runs in runs[I].  Run by one warp: the run heads are listed
// first, then each lane sums whole runs.
__device__ void gal_emit(const GalSmem &sm, int T, int32_t I, int64_t base, int32_t *tJ,
                         double *tV, int32_t *runs, int *err, int lane) {
  int nr = 0;
  for (int b0 = 0; b0 < T; b0 += 32) {
    const int k = b0 + lane;
    const bool h = k < T && gal_head(sm, k);
    const unsigned hm = __ballot_sync(0xffffffffu, h);
    if (h) sm.heads[nr + __popc(hm & ((1u << lane) - 1u))] = k;
    nr += __popc(hm);
  }
  __syncwarp();
  for (int r = lane; r < nr; r += 32) {
    const int k = sm.heads[r];
    const int len = (r + 1 < nr ? sm.heads[r + 1] : T) - k;
    int32_t J;
    double sum;
    if (gal_run_sum(sm, k, len, &J, &sum)) {
      tJ[base + r] = J;
      tV[base + r] = sum;
    } else {
      atomicExch(err, 2);
    }
  }
  if (lane == 0) runs[I] = nr;
}

// Sort-and-reduce pass, one warp per coarse row, over the rows queued by
// k_gal_rows_reg (grid-stride); rows over kGalCap terms are queued for
// k_gal_rows_long.
__global__ void __launch_bounds__(kGalWarpsPerBlock * 32)
    k_gal_rows(const int32_t *__restrict__ queue, const int32_t *__restrict__ n_queue,
               const int32_t *__restrict__ row, const int32_t *__restrict__ col,
               const double *__restrict__ val, const int32_t *__restrict__ agg,
               const double *__restrict__ p, const int32_t *__restrict__ rptr,
               const int32_t *__restrict__ ridx, const int32_t *__restrict__ tpos,
               int32_t *tJ, double *tV, int32_t *runs, int32_t *long_rows, int32_t *n_long,
               int *err) {
  extern __shared__ __align__(16) unsigned char gal_dyn[];
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  GalSmem sm = gal_smem(gal_dyn + static_cast<size_t>(wid) * kGalCap * kGalBytesPerTerm,
                        kGalCap);
  const int32_t nq = *n_queue;
  for (int32_t q = blockIdx.x * kGalWarpsPerBlock + wid; q < nq;
       q += gridDim.x * kGalWarpsPerBlock) {
    const int32_t I = queue[q];
    const int T = gal_gather<32>(I, row, col, val, agg, p, rptr, ridx, sm, kGalCap, lane);
    if (T < 0) {
      if (lane == 0) long_rows[atomicAdd(n_long, 1)] = I;
      continue;
    }
    gal_emit(sm, T, I, tpos[I], tJ, tV, runs, err, lane);
    __syncwarp();
  }
}

// Coarse rows of at most kGalRegTerms terms, one warp per row with the terms
// in registers, two per lane (slot t = lane + 32 r): keys J << 6 | t (J below
// 2^26) go through a 64-key bitonic network of shuffles, the terms' values
// and fine (i, j) wait in shared memory by slot, and the lane at each run head
// sums its run in the canonical order.  Same output as k_gal_rows, at a
// fraction of its instructions; longer rows, and aggregates of more than 32
// members, are queued for it.
constexpr int kGalRegTerms = 64;
constexpr int kGalRegWarps = 8;
struct GalRegSmem {
  double v[kGalRegTerms];
  int32_t ti[kGalRegTerms];
  int32_t tj[kGalRegTerms];
  int32_t sidx[kGalRegTerms];
};

__global__ void __launch_bounds__(kGalRegWarps * 32)
    k_gal_rows_reg(int32_t nc, const int32_t *__restrict__ row,
                   const int32_t *__restrict__ col, const double *__restrict__ val,
                   const int32_t *__restrict__ agg, const double *__restrict__ p,
                   const int32_t *__restrict__ rptr, const int32_t *__restrict__ ridx,
                   const int32_t *__restrict__ tpos, int32_t *tJ, double *tV,
                   int32_t *runs, int32_t *mid_rows, int32_t *n_mid, int *err) {
  __shared__ GalRegSmem smem[kGalRegWarps];
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int32_t I = blockIdx.x * kGalRegWarps + wid;
  if (I >= nc) return;
  GalRegSmem &sm = smem[wid];
  const int32_t kb = rptr[I];
  const int M = rptr[I + 1] - kb;
  // Members (ascending): row start, length, p, and the exclusive prefix of
  // the lengths (each member's first slot).
  int32_t mi = 0, mb = 0, ml = 0;
  double mp = 0.0;
  if (lane < M) {
    mi = ridx[kb + lane];
    mb = row[mi];
    ml = row[mi + 1] - mb;
    mp = p[mi];
  }
  int32_t incl = ml;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int32_t y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  const int32_t T = __shfl_sync(0xffffffffu, incl, 31);
  if (M > 32 || T > kGalRegTerms) {
    if (lane == 0) mid_rows[atomicAdd(n_mid, 1)] = I;
    return;
  }
  const int32_t first = incl - ml;
  uint32_t key[2];
#pragma unroll
  for (int r = 0; r < 2; ++r) {
    const int t = lane + 32 * r;
    // the member holding slot t: the last one whose first slot is <= t
    int m = 0;
    for (int q = 1; q < M; ++q)
      if (__shfl_sync(0xffffffffu, first, q) <= t) m = q;
    const int32_t b = __shfl_sync(0xffffffffu, mb, m);
    const int32_t f = __shfl_sync(0xffffffffu, first, m);
    const int32_t i = __shfl_sync(0xffffffffu, mi, m);
    const double pi = __shfl_sync(0xffffffffu, mp, m);
    key[r] = 0xffffffffu;
    if (t < T) {
      const int32_t e = b + (t - f);
      const int32_t j = col[e];
      sm.v[t] = (pi * p[j]) * val[e];
      sm.ti[t] = i;
      sm.tj[t] = j;
      key[r] = (static_cast<uint32_t>(agg[j]) << 6) | static_cast<uint32_t>(t);
    }
  }
  // Ascending bitonic sort of the 64 keys (position lane + 32 r).
#pragma unroll
  for (int k = 2; k <= 64; k <<= 1) {
#pragma unroll
    for (int j = k >> 1; j > 0; j >>= 1) {
      if (j == 32) {
        const uint32_t a = key[0], b = key[1];
        key[0] = min(a, b);
        key[1] = max(a, b);
      } else {
#pragma unroll
        for (int r = 0; r < 2; ++r) {
          const uint32_t o = __shfl_xor_sync(0xffffffffu, key[r], j);
          const int pos = lane + 32 * r;
          const bool lower = (pos & j) == 0;
          const bool asc = (pos & k) == 0;
          key[r] = (lower == asc) ? min(key[r], o) : max(key[r], o);
        }
      }
    }
  }
#pragma unroll
  for (int r = 0; r < 2; ++r)
    if (lane + 32 * r < T) sm.sidx[lane + 32 * r] = static_cast<int32_t>(key[r] & 63u);
  __syncwarp();
  // Run heads and their ranks.
  const uint32_t J0 = key[0] >> 6, J1 = key[1] >> 6;
  const uint32_t up0 = __shfl_up_sync(0xffffffffu, J0, 1);
  const uint32_t up1 = __shfl_up_sync(0xffffffffu, J1, 1);
  const uint32_t last0 = __shfl_sync(0xffffffffu, J0, 31);
  const bool h0 = lane < T && (lane == 0 || J0 != up0);
  const bool h1 = lane + 32 < T && J1 != (lane == 0 ? last0 : up1);
  const unsigned b0 = __ballot_sync(0xffffffffu, h0), b1 = __ballot_sync(0xffffffffu, h1);
  const unsigned long long H = static_cast<unsigned long long>(b0) |
                               (static_cast<unsigned long long>(b1) << 32);
  const int nr = __popcll(H);
  const int64_t base = tpos[I];
#pragma unroll
  for (int r = 0; r < 2; ++r) {
    if (!(r == 0 ? h0 : h1)) continue;
    const int q = lane + 32 * r;
    const unsigned long long after = q < 63 ? (H >> (q + 1)) : 0ull;
    const int len = (after ? q + 1 + __ffsll(static_cast<long long>(after)) - 1 : T) - q;
    const int rank = __popcll(H & ((1ull << q) - 1ull));
    int32_t Jv = static_cast<int32_t>(r == 0 ? J0 : J1);
    double sum = 0.0;
    if (len <= 4) {
      int id[4];
      int32_t mn[4], mx[4], ti[4];
#pragma unroll
      for (int a = 0; a < 4; ++a) {
        const bool ok = a < len;
        id[a] = ok ? sm.sidx[q + a] : 0;
        const int32_t x = ok ? sm.ti[id[a]] : INT_MAX, y = ok ? sm.tj[id[a]] : INT_MAX;
        ti[a] = x;
        mn[a] = min(x, y);
        mx[a] = max(x, y);
      }
      gal_cx(id[0], mn[0], mx[0], ti[0], id[1], mn[1], mx[1], ti[1]);
      gal_cx(id[2], mn[2], mx[2], ti[2], id[3], mn[3], mx[3], ti[3]);
      gal_cx(id[0], mn[0], mx[0], ti[0], id[2], mn[2], mx[2], ti[2]);
      gal_cx(id[1], mn[1], mx[1], ti[1], id[3], mn[3], mx[3], ti[3]);
      gal_cx(id[1], mn[1], mx[1], ti[1], id[2], mn[2], mx[2], ti[2]);
      sum = sm.v[id[0]];
#pragma unroll
      for (int a = 1; a < 4; ++a)
        if (a < len) sum = sum + sm.v[id[a]];
    } else if (len <= kGalMaxRun) {
      int idx[kGalMaxRun];
      for (int a = 0; a < len; ++a) idx[a] = sm.sidx[q + a];
      for (int a = 1; a < len; ++a) {  // insertion sort by (min, max, i)
        const int x = idx[a];
        const int32_t xi = sm.ti[x], xj = sm.tj[x];
        const int32_t xmn = min(xi, xj), xmx = max(xi, xj);
        int c = a - 1;
        while (c >= 0) {
          const int y = idx[c];
          const int32_t yi = sm.ti[y], yj = sm.tj[y];
          const int32_t ymn = min(yi, yj), ymx = max(yi, yj);
          if (!(ymn > xmn || (ymn == xmn && (ymx > xmx || (ymx == xmx && yi > xi))))) break;
          idx[c + 1] = idx[c];
          --c;
        }
        idx[c + 1] = x;
      }
      sum = sm.v[idx[0]];
      for (int a = 1; a < len; ++a) sum = sum + sm.v[idx[a]];
    } else {
      atomicExch(err, 2);
      continue;
    }
    tJ[base + rank] = Jv;
    tV[base + rank] = sum;
  }
  if (lane == 0) runs[I] = nr;
}

// The queued long rows, one block per row (grid-stride over the queue).
__global__ void __launch_bounds__(kGalLongThreads)
    k_gal_rows_long(const int32_t *__restrict__ long_rows, const int32_t *__restrict__ n_long,
                    const int32_t *__restrict__ row, const int32_t *__restrict__ col,
                    const double *__restrict__ val, const int32_t *__restrict__ agg,
                    const double *__restrict__ p, const int32_t *__restrict__ rptr,
                    const int32_t *__restrict__ ridx, const int32_t *__restrict__ tpos,
                    int32_t *tJ, double *tV, int32_t *runs, int *err) {
  extern __shared__ __align__(16) unsigned char gal_dyn[];
  GalSmem sm = gal_smem(gal_dyn, kGalCapLong);
  for (int32_t q = blockIdx.x; q < *n_long; q += gridDim.x) {
    const int32_t I = long_rows[q];
    const int T = gal_gather<kGalLongThreads>(I, row, col, val, agg, p, rptr, ridx, sm,
                                              kGalCapLong, threadIdx.x);
    if (T < 0) {
      if (threadIdx.x == 0) atomicExch(err, 3);
      return;
    }
    if (threadIdx.x < 32) gal_emit(sm, T, I, tpos[I], tJ, tV, runs, err, threadIdx.x);
    __syncthreads();
  }
}

// ---- general SpGEMM C = X Y (smoothed aggregation) --------------------------
// Canonical order: C_ij sums the terms x_ik y_kj in X's row order, from the
// first term.  Every Y row has distinct columns, so column j gets at most one
// term per X entry, and this equals summing each column's run of the
// generation-ordered term list after a stable sort by column.
// Rows run in three tiers by their distinct column count U: a warp with a
// shared-memory hash set of kSpWarpHash slots, a block with kSpBlockHash
// slots, a block with a table in global memory.  A set is used up to half
// full.  The symbolic pass counts U (sending a row on to the next tier when
// its set would pass half full); the numeric pass rebuilds the set, sorts its
// columns, stores each column's rank in the set and accumulates one value per
// rank, X entry by X entry.

constexpr int kSpWarpHash = 1024;  // warp tier: U <= 512
constexpr int kSpWarpsPerBlock = 4;
constexpr int kSpBlockHash = 4096;  // block tier: U <= 2048
constexpr int kSpThreads = 256;

// The numeric pass takes a row's X entries in chunks of at most CA entries
// whose Y rows hold at most SB terms in all: their (rank, value) pairs are
// computed in parallel into shared memory, then added X entry by X entry.
template <int CA, int SB>
struct SpStage {
  double x[CA];
  double v[SB];
  int b0[CA];
  int len[CA];
  int off[CA + 1];
  int r[SB];
};
using SpStageWarp = SpStage<64, 192>;
using SpStageBlock = SpStage<256, 2048>;
constexpr size_t kSpStageWarpBytes = (sizeof(SpStageWarp) + 15) & ~size_t(15);
constexpr size_t kSpStageBlockBytes = (sizeof(SpStageBlock) + 15) & ~size_t(15);

struct SpTable {
  double *acc;          // hc/2 values, by rank
  int *key;             // hc slots, -1 = empty
  int *rank;            // hc slots
  int *cols;            // hc/2 sorted columns
  int *count;           // distinct columns inserted
  unsigned char *seen;  // hc/2 flags: acc holds a first term
  int hc;
};

__host__ __device__ constexpr size_t sp_table_bytes(int hc) {
  return (static_cast<size_t>(14) * hc + 16 + hc / 2 + 15) & ~static_cast<size_t>(15);
}

__device__ __forceinline__ SpTable sp_table(unsigned char *base, int hc) {
  SpTable t;
  t.hc = hc;
  t.acc = reinterpret_cast<double *>(base);
  t.key = reinterpret_cast<int *>(base + 4 * static_cast<size_t>(hc));
  t.rank = reinterpret_cast<int *>(base + 8 * static_cast<size_t>(hc));
  t.cols = reinterpret_cast<int *>(base + 12 * static_cast<size_t>(hc));
  t.count = reinterpret_cast<int *>(base + 14 * static_cast<size_t>(hc));
  t.seen = base + 14 * static_cast<size_t>(hc) + 16;
  return t;
}

__device__ __forceinline__ unsigned sp_hash(int key, int hc) {
  return (static_cast<unsigned>(key) * 2654435761u) & static_cast<unsigned>(hc - 1);
}

__device__ __forceinline__ int sp_find(const SpTable &t, int key) {
  unsigned h = sp_hash(key, t.hc);
  for (int probe = 0; probe < t.hc; ++probe) {
    if (t.key[h] == key) return static_cast<int>(h);
    h = (h + 1) & static_cast<unsigned>(t.hc - 1);
  }
  return 0;  // unreachable: the key was inserted
}

// Inserts the columns of row i of X Y into t; returns their number, or -1 if
// the set would pass half full.  Ends with the team synchronised.
template <int TEAM>
__device__ int sp_collect(const SpTable &t, int32_t i, const int32_t *__restrict__ xrow,
                          const int32_t *__restrict__ xcol, const int32_t *__restrict__ yrow,
                          const int32_t *__restrict__ ycol, int tid) {
  for (int q = tid; q < t.hc; q += TEAM) t.key[q] = -1;
  if (tid == 0) *t.count = 0;
  team_sync<TEAM>();
  const int limit = t.hc / 2;
  volatile int *cnt = t.count;
  constexpr int kWarps = TEAM / 32;
  const int lane = tid & 31;
  for (int32_t a = xrow[i] + tid / 32; a < xrow[i + 1]; a += kWarps) {
    const int32_t k = xcol[a];
    const int32_t b0 = yrow[k], len = yrow[k + 1] - b0;
    for (int32_t q = lane; q < len; q += 32) {
      if (*cnt > limit) break;  // (at most TEAM keys past the limit)
      const int j = ycol[b0 + q];
      unsigned h = sp_hash(j, t.hc);
      for (int probe = 0; probe < t.hc; ++probe) {
        const int prev = atomicCAS(t.key + h, -1, j);
        if (prev == -1) {
          atomicAdd(t.count, 1);
          break;
        }
        if (prev == j) break;
        h = (h + 1) & static_cast<unsigned>(t.hc - 1);
      }
    }
  }
  team_sync<TEAM>();
  const int U = *cnt;
  team_sync<TEAM>();
  return U > limit ? -1 : U;
}

// Row i's sorted columns and values into ccol/cval from `base`; t holds the
// row's set (sp_collect), U its size, st is the team's staging area.
template <int TEAM, int CA, int SB>
__device__ void sp_numeric(const SpTable &t, SpStage<CA, SB> &st, int32_t i, int U,
                           const int32_t *__restrict__ xrow, const int32_t *__restrict__ xcol,
                           const double *__restrict__ xval, const int32_t *__restrict__ yrow,
                           const int32_t *__restrict__ ycol, const double *__restrict__ yval,
                           int32_t base, int32_t *ccol, double *cval, int tid) {
  static_assert(CA % 32 == 0, "chunk of X entries in whole warps");
  if (tid == 0) *t.count = 0;
  team_sync<TEAM>();
  for (int q = tid; q < t.hc; q += TEAM) {
    const int j = t.key[q];
    if (j >= 0) t.cols[atomicAdd(t.count, 1)] = j;
  }
  int P2 = 1;
  while (P2 < U) P2 <<= 1;
  for (int q = U + tid; q < P2; q += TEAM) t.cols[q] = INT_MAX;
  team_sync<TEAM>();
  for (int k = 2; k <= P2; k <<= 1) {
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int q = tid; q < P2 / 2; q += TEAM) {
        const int i0 = ((q & ~(j - 1)) << 1) | (q & (j - 1));  // j = 2^m
        const int i1 = i0 + j;
        const bool asc = (i0 & k) == 0;
        const int u = t.cols[i0], v = t.cols[i1];
        if ((u > v) == asc) {
          t.cols[i0] = v;
          t.cols[i1] = u;
        }
      }
      team_sync<TEAM>();
    }
  }
  for (int r = tid; r < U; r += TEAM) {
    const int j = t.cols[r];
    t.rank[sp_find(t, j)] = r;
    t.seen[r] = 0;
    ccol[base + r] = j;
  }
  team_sync<TEAM>();
  const int32_t a_end = xrow[i + 1];
  for (int32_t a0 = xrow[i]; a0 < a_end;) {
    const int na = a_end - a0 < CA ? static_cast<int>(a_end - a0) : CA;
    for (int u = tid; u < na; u += TEAM) {
      const int32_t k = xcol[a0 + u];
      const int32_t b = yrow[k];
      st.b0[u] = b;
      st.len[u] = yrow[k + 1] - b;
      st.x[u] = xval[a0 + u];
    }
    team_sync<TEAM>();
    if (tid < 32) {  // st.off = exclusive scan of min(len, SB + 1)
      constexpr int kPer = CA / 32;
      int loc[kPer];
      int sum = 0;
#pragma unroll
      for (int p = 0; p < kPer; ++p) {
        const int u = tid * kPer + p;
        loc[p] = u < na ? min(st.len[u], SB + 1) : 0;
        sum += loc[p];
      }
      int incl = sum;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, incl, o);
        if (tid >= o) incl += y;
      }
      int run = incl - sum;
#pragma unroll
      for (int p = 0; p < kPer; ++p) {
        st.off[tid * kPer + p] = run;
        run += loc[p];
      }
      if (tid == 31) st.off[CA] = incl;
    }
    team_sync<TEAM>();
    if (st.off[1] > SB) {  // one Y row over the stage: added directly
      const int32_t b0 = st.b0[0], len = st.len[0];
      const double x = st.x[0];
      for (int32_t q = tid; q < len; q += TEAM) {
        const int r = t.rank[sp_find(t, ycol[b0 + q])];
        const double v = x * yval[b0 + q];
        t.acc[r] = t.seen[r] ? t.acc[r] + v : v;
        t.seen[r] = 1;
      }
      team_sync<TEAM>();
      a0 += 1;
      continue;
    }
    int nfit = 1;  // the most X entries whose terms fit the stage
    {
      int lo = 1, hi = na;
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (st.off[mid] <= SB) lo = mid;
        else hi = mid - 1;
      }
      nfit = lo;
    }
    const int total = st.off[nfit];
    for (int e = tid; e < total; e += TEAM) {
      int lo = 0, hi = nfit - 1;  // the X entry whose terms hold e
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (st.off[mid] <= e) lo = mid;
        else hi = mid - 1;
      }
      const int32_t b = st.b0[lo] + (e - st.off[lo]);
      st.r[e] = t.rank[sp_find(t, ycol[b])];
      st.v[e] = st.x[lo] * yval[b];
    }
    team_sync<TEAM>();
    for (int u = 0; u < nfit; ++u) {
      for (int e = st.off[u] + tid; e < st.off[u + 1]; e += TEAM) {
        const int r = st.r[e];
        const double v = st.v[e];
        t.acc[r] = t.seen[r] ? t.acc[r] + v : v;
        t.seen[r] = 1;
      }
      team_sync<TEAM>();
    }
    a0 += nfit;
  }
  for (int r = tid; r < U; r += TEAM) cval[base + r] = t.acc[r];
  team_sync<TEAM>();
}

__global__ void k_sp_max_terms(int32_t n, const int32_t *__restrict__ xrow,
                               const int32_t *__restrict__ xcol,
                               const int32_t *__restrict__ yrow, unsigned long long *max_terms) {
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int64_t t = 0;
  for (int32_t a = xrow[i]; a < xrow[i + 1]; ++a) {
    const int32_t k = xcol[a];
    t += yrow[k + 1] - yrow[k];
  }
  atomicMax(max_terms, static_cast<unsigned long long>(t));
}

// Symbolic pass, warp tier, every row: ucount[i] = U; rows over the warp
// set go to `next` with tier[i] = 1.
__global__ void __launch_bounds__(kSpWarpsPerBlock * 32)
    k_sp_count_warp(int32_t n, const int32_t *__restrict__ xrow, const int32_t *__restrict__ xcol,
                    const int32_t *__restrict__ yrow, const int32_t *__restrict__ ycol,
                    int32_t *ucount, unsigned char *tier, int32_t *next, int32_t *n_next) {
  extern __shared__ __align__(16) unsigned char sp_dyn[];
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int32_t i = blockIdx.x * kSpWarpsPerBlock + wid;
  if (i >= n) return;
  const SpTable t = sp_table(sp_dyn + wid * sp_table_bytes(kSpWarpHash), kSpWarpHash);
  const int U = sp_collect<32>(t, i, xrow, xcol, yrow, ycol, lane);
  if (lane == 0) {
    ucount[i] = U < 0 ? 0 : U;
    tier[i] = U < 0 ? 1 : 0;
    if (U < 0) next[atomicAdd(n_next, 1)] = i;
  }
}

// Symbolic pass, block tiers, over rows[0..*n_rows): the table in shared
// memory (gtab null, kSpBlockHash slots) or in this block's slice of gtab
// (ghc slots, sized for every row).  Rows over the set go to `next` with
// tier[i] = tier_here + 1, or raise err when there is no next tier.
// A global table's size for one row: a power of two, at least 64, at least
// twice `bound` (+2), at most ghc.
__device__ __forceinline__ int sp_row_hc(int64_t bound, int ghc) {
  int64_t c = 64;
  while (c < 2 * bound + 2 && c < ghc) c <<= 1;
  return static_cast<int>(c);
}

// Terms of row i of X Y (team-wide; ends synchronised).
__device__ int64_t sp_row_terms(int32_t i, const int32_t *__restrict__ xrow,
                                const int32_t *__restrict__ xcol,
                                const int32_t *__restrict__ yrow, unsigned long long *acc) {
  if (threadIdx.x == 0) *acc = 0;
  __syncthreads();
  unsigned long long t = 0;
  for (int32_t a = xrow[i] + threadIdx.x; a < xrow[i + 1]; a += blockDim.x) {
    const int32_t k = xcol[a];
    t += static_cast<unsigned long long>(yrow[k + 1] - yrow[k]);
  }
  atomicAdd(acc, t);
  __syncthreads();
  const int64_t T = static_cast<int64_t>(*acc);
  __syncthreads();
  return T;
}

__global__ void __launch_bounds__(kSpThreads)
    k_sp_count_block(const int32_t *__restrict__ rows, const int32_t *__restrict__ n_rows,
                     const int32_t *__restrict__ xrow, const int32_t *__restrict__ xcol,
                     const int32_t *__restrict__ yrow, const int32_t *__restrict__ ycol,
                     int32_t m, int32_t *ucount, unsigned char *tier, int32_t *next,
                     int32_t *n_next, unsigned char *gtab, int ghc, int tier_here, int *err) {
  extern __shared__ __align__(16) unsigned char sp_dyn[];
  __shared__ unsigned long long terms;
  for (int32_t q = blockIdx.x; q < *n_rows; q += gridDim.x) {
    const int32_t i = rows[q];
    SpTable t;
    if (gtab) {
      const int64_t T = sp_row_terms(i, xrow, xcol, yrow, &terms);
      t = sp_table(gtab + blockIdx.x * sp_table_bytes(ghc), sp_row_hc(T < m ? T : m, ghc));
    } else {
      t = sp_table(sp_dyn, kSpBlockHash);
    }
    const int U = sp_collect<kSpThreads>(t, i, xrow, xcol, yrow, ycol, threadIdx.x);
    if (threadIdx.x == 0) {
      ucount[i] = U < 0 ? 0 : U;
      if (U < 0) {
        if (next) {
          tier[i] = static_cast<unsigned char>(tier_here + 1);
          next[atomicAdd(n_next, 1)] = i;
        } else {
          atomicExch(err, 1);
        }
      }
    }
  }
}

// Numeric pass, warp tier (rows with tier 0).
__global__ void __launch_bounds__(kSpWarpsPerBlock * 32)
    k_sp_fill_warp(int32_t n, const int32_t *__restrict__ xrow, const int32_t *__restrict__ xcol,
                   const double *__restrict__ xval, const int32_t *__restrict__ yrow,
                   const int32_t *__restrict__ ycol, const double *__restrict__ yval,
                   const unsigned char *__restrict__ tier, const int32_t *__restrict__ crow,
                   int32_t *ccol, double *cval) {
  extern __shared__ __align__(16) unsigned char sp_dyn[];
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int32_t i = blockIdx.x * kSpWarpsPerBlock + wid;
  if (i >= n || tier[i] != 0) return;
  unsigned char *mine = sp_dyn + wid * (sp_table_bytes(kSpWarpHash) + kSpStageWarpBytes);
  const SpTable t = sp_table(mine, kSpWarpHash);
  SpStageWarp &st = *reinterpret_cast<SpStageWarp *>(mine + sp_table_bytes(kSpWarpHash));
  const int U = sp_collect<32>(t, i, xrow, xcol, yrow, ycol, lane);
  sp_numeric<32>(t, st, i, U, xrow, xcol, xval, yrow, ycol, yval, crow[i], ccol, cval, lane);
}

// Numeric pass, block tiers: rows of rows[0..*n_rows) with tier[i] ==
// tier_here, tables as in k_sp_count_block.
__global__ void __launch_bounds__(kSpThreads)
    k_sp_fill_block(const int32_t *__restrict__ rows, const int32_t *__restrict__ n_rows,
                    const int32_t *__restrict__ xrow, const int32_t *__restrict__ xcol,
                    const double *__restrict__ xval, const int32_t *__restrict__ yrow,
                    const int32_t *__restrict__ ycol, const double *__restrict__ yval,
                    const unsigned char *__restrict__ tier, const int32_t *__restrict__ crow,
                    int32_t *ccol, double *cval, unsigned char *gtab, int ghc, int tier_here) {
  extern __shared__ __align__(16) unsigned char sp_dyn[];
  SpStageBlock &st = *reinterpret_cast<SpStageBlock *>(sp_dyn);
  for (int32_t q = blockIdx.x; q < *n_rows; q += gridDim.x) {
    const int32_t i = rows[q];
    if (tier[i] != tier_here) continue;
    const SpTable t =
        gtab ? sp_table(gtab + blockIdx.x * sp_table_bytes(ghc), sp_row_hc(crow[i + 1] - crow[i], ghc))
             : sp_table(sp_dyn + kSpStageBlockBytes, kSpBlockHash);
    const int U = sp_collect<kSpThreads>(t, i, xrow, xcol, yrow, ycol, threadIdx.x);
    sp_numeric<kSpThreads>(t, st, i, U, xrow, xcol, xval, yrow, ycol, yval, crow[i], ccol, cval,
                           threadIdx.x);
  }
}

// CSR transpose: counts, a scan, unordered fill, then each row sorted by
// column (= source row) so the result is canonical.
__global__ void k_tr_count(int32_t nnz, const int32_t *__restrict__ col, int32_t m,
                           int32_t *cnt, int *err) {
  const int32_t e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nnz) return;
  const int32_t c = col[e];
  if (c < 0 || c >= m) {
    atomicExch(err, 1);
    return;
  }
  atomicAdd(cnt + c, 1);
}

__global__ void k_tr_fill(int32_t n, const int32_t *__restrict__ row,
                          const int32_t *__restrict__ col, const double *__restrict__ val,
                          int32_t m, const int32_t *__restrict__ trow, int32_t *cursor,
                          int32_t *tcol, double *tval) {
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  for (int32_t e = row[i]; e < row[i + 1]; ++e) {
    const int32_t c = col[e];
    if (c < 0 || c >= m) continue;
    const int32_t q = trow[c] + atomicAdd(cursor + c, 1);
    tcol[q] = i;
    tval[q] = val[e];
  }
}

// Sorts key[0..n) ascending with its payload, team-wide: a bitonic network
// whose comparators all point up (each merge starts by comparing mirrored
// positions), so positions n..P2 act as +infinity and are never touched.
template <int TEAM>
__device__ void sort_up_pairs(int32_t *key, double *val, int n, int tid) {
  int P2 = 1;
  while (P2 < n) P2 <<= 1;
  for (int k = 2; k <= P2; k <<= 1) {
    const int h = k >> 1;
    for (int t = tid; t < P2 / 2; t += TEAM) {
      const int i = (t / h) * k + (t % h);
      const int j = i ^ (k - 1);
      if (j < n && key[i] > key[j]) {
        const int32_t tk = key[i];
        key[i] = key[j];
        key[j] = tk;
        const double tv = val[i];
        val[i] = val[j];
        val[j] = tv;
      }
    }
    team_sync<TEAM>();
    for (int d = k >> 2; d > 0; d >>= 1) {
      for (int t = tid; t < P2 / 2; t += TEAM) {
        const int i = (t / d) * 2 * d + (t % d);
        const int j = i + d;
        if (j < n && key[i] > key[j]) {
          const int32_t tk = key[i];
          key[i] = key[j];
          key[j] = tk;
          const double tv = val[i];
          val[i] = val[j];
          val[j] = tv;
        }
      }
      team_sync<TEAM>();
    }
  }
}

constexpr int kTrThreads = 256;
constexpr int kTrSmem = 8192;  // rows up to this length sort in shared memory

// Sorts every row of the transpose by column (= source row), a block per
// row: in shared memory up to kTrSmem entries, in place beyond.
__global__ void __launch_bounds__(kTrThreads)
    k_tr_sort(int32_t m, const int32_t *__restrict__ trow, int32_t *tcol, double *tval) {
  extern __shared__ __align__(16) unsigned char tr_dyn[];
  double *sv = reinterpret_cast<double *>(tr_dyn);
  int32_t *sk = reinterpret_cast<int32_t *>(tr_dyn + sizeof(double) * kTrSmem);
  for (int32_t r = blockIdx.x; r < m; r += gridDim.x) {
    const int32_t b = trow[r];
    const int len = trow[r + 1] - b;
    if (len <= 1) continue;
    if (len <= kTrSmem) {
      for (int q = threadIdx.x; q < len; q += kTrThreads) {
        sk[q] = tcol[b + q];
        sv[q] = tval[b + q];
      }
      __syncthreads();
      sort_up_pairs<kTrThreads>(sk, sv, len, threadIdx.x);
      for (int q = threadIdx.x; q < len; q += kTrThreads) {
        tcol[b + q] = sk[q];
        tval[b + q] = sv[q];
      }
      __syncthreads();
    } else {
      sort_up_pairs<kTrThreads>(tcol + b, tval + b, len, threadIdx.x);
    }
  }
}

// Smoothing operator S = I - omega D^{-1} A, in two passes:
// k_smooth_scale writes s = a / d_i and the max absolute row sum (the
// infinity norm, exact max on non-negative doubles via their bits);
// k_smooth_omega then applies s = -omega s (+1 on the diagonal).
__global__ void k_smooth_scale(int32_t n, const int32_t *__restrict__ row,
                               const double *__restrict__ val, const double *__restrict__ D,
                               double *sval, unsigned long long *inf_bits) {
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double rs = 0.0;
  for (int32_t e = row[i]; e < row[i + 1]; ++e) {
    const double t = val[e] / D[i];
    sval[e] = t;
    rs = rs + fabs(t);
  }
  atomicMax(inf_bits, static_cast<unsigned long long>(__double_as_longlong(rs)));
}

__global__ void k_smooth_omega(int32_t n, const int32_t *__restrict__ row,
                               const int32_t *__restrict__ col, double omega, double *sval) {
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  for (int32_t e = row[i]; e < row[i + 1]; ++e) {
    double t = -omega * sval[e];
    if (col[e] == i) t = t + 1.0;
    sval[e] = t;
  }
}

__global__ void k_iota(int32_t n, int32_t *x) {
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i <= n) x[i] = i;
}

// Moves each row's runs from its term-sized slot to its final CSR position.
__global__ void k_gal_compact(int32_t nc, const int32_t *__restrict__ tpos,
                              const int32_t *__restrict__ crow,
                              const int32_t *__restrict__ tJ, const double *__restrict__ tV,
                              int32_t *ccol, double *cval) {
  const int lane = threadIdx.x & 31;
  const int32_t I = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (I >= nc) return;
  const int32_t src = tpos[I], dst = crow[I], len = crow[I + 1] - crow[I];
  for (int32_t k = lane; k < len; k += 32) {
    ccol[dst + k] = tJ[src + k];
    cval[dst + k] = tV[src + k];
  }
}

// y[I] = sum over members i of I (ascending) of p_i x_i, from the first term.
__global__ void k_restrict_exact(int32_t nc, const int32_t *__restrict__ rptr,
                                 const int32_t *__restrict__ ridx,
                                 const double *__restrict__ p,
                                 const double *__restrict__ x, double *y) {
  const int32_t I = blockIdx.x * blockDim.x + threadIdx.x;
  if (I >= nc) return;
  const int32_t b = rptr[I], e = rptr[I + 1];
  double s = 0.0;
  for (int32_t k = b; k < e; ++k) {
    const int32_t i = ridx[k];
    const double t = p[i] * x[i];
    s = (k == b) ? t : s + t;
  }
  y[I] = s;
}

// P = P * P_i (matchingAggregation.cu:264): one entry per row stays one entry.
__global__ void k_compose(int32_t n, int32_t *agg, double *p,
                          const int32_t *__restrict__ agg2,
                          const double *__restrict__ p2) {
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int32_t a = agg[i];
  p[i] = p[i] * p2[a];
  agg[i] = agg2[a];
}

template <int G>
bcmg_status launch_min(const CsrView &A, const double *w, const double *C,
                       unsigned long long *min_bits, cudaStream_t s) {
  const int threads = 256;
  const int blocks = ceil_div(static_cast<int64_t>(A.n) * G, threads);
  launch(k_ah_min<G>, std::min(blocks, 64 * kNumSM), threads, 0, s, A.n, A.row, A.col, A.val,
         w, C, min_bits);
  BCMG_LAUNCH_CHECK();
  return BCMG_OK;
}

}  // namespace

// ---------------------------------------------------------------------------
bcmg_status level_prep(const CsrView &A, double *D, double *M, cudaStream_t s) {
  if (A.n <= 0) return BCMG_OK;
  launch(k_level_prep, ceil_div(A.n, 256), 256, 0, s, A.n, A.row, A.col, A.val, D, M);
  BCMG_LAUNCH_CHECK();
  return BCMG_OK;
}

// matchingPairAggregation (src/AMG/matchingAggregation.cu:181-208) with
// Matching::suitor (src/AMG/matching.cu:476-502).
bcmg_status pair_aggregate(const CsrView &A, const double *w, int32_t *agg, double *p,
                           int32_t *nc_out, double *W_out, int32_t *s_out,
                           int32_t *m_out, cudaStream_t s, int64_t step_limit) {
  const int32_t n = A.n;
  if (n <= 0) {
    *nc_out = 0;
    return BCMG_OK;
  }
  const int T = 256;
  const int nb = ceil_div(n, T);
  DevBuf<double> C;
  DevBuf<unsigned long long> offer, minb;
  DevBuf<int32_t> sv, mv, m2, tgt, master, rank, tmp, total;
  DevBuf<int> err;
  BCMG_TRY(C.alloc(n, s));
  BCMG_TRY(offer.alloc(n, s));
  BCMG_TRY(minb.alloc(1, s));
  BCMG_TRY(sv.alloc(n, s));
  BCMG_TRY(mv.alloc(n, s));
  BCMG_TRY(m2.alloc(n, s));
  BCMG_TRY(tgt.alloc(n, s));
  BCMG_TRY(master.alloc(n, s));
  BCMG_TRY(rank.alloc(n, s));
  BCMG_TRY(tmp.alloc(scan_tmp_size(n), s));
  BCMG_TRY(total.alloc(1, s));
  BCMG_TRY(err.alloc(1, s));

  // Weights.
  launch(k_make_C, nb, T, 0, s, n, A.row, A.col, A.val, w, C.get());
  const unsigned long long dbl_max_bits = 0x7FEFFFFFFFFFFFFFull;
  BCMG_CUDA(cudaMemcpyAsync(minb.get(), &dbl_max_bits, sizeof(dbl_max_bits),
                            cudaMemcpyHostToDevice, s));
  const int G = group_for(A.nnz, n);
  switch (G) {
    case 4: BCMG_TRY(launch_min<4>(A, w, C.get(), minb.get(), s)); break;
    case 8: BCMG_TRY(launch_min<8>(A, w, C.get(), minb.get(), s)); break;
    case 16: BCMG_TRY(launch_min<16>(A, w, C.get(), minb.get(), s)); break;
    default: BCMG_TRY(launch_min<32>(A, w, C.get(), minb.get(), s)); break;
  }

  phase_tick("weights");
  // Preference-sorted rows, then the suitor proposals.
  DevBuf<double> sW;
  DevBuf<int32_t> scol, inv, ucnt, next, long_rows, mid_rows, n_queued;
  DevBuf<unsigned long long> E;
  DevBuf<int> nonsym;
  BCMG_TRY(sW.alloc(A.nnz, s));
  BCMG_TRY(scol.alloc(A.nnz, s));
  BCMG_TRY(inv.alloc(A.nnz, s));
  BCMG_TRY(E.alloc(A.nnz, s));
  BCMG_TRY(ucnt.alloc(n, s));
  BCMG_TRY(next.alloc(n, s));
  BCMG_TRY(long_rows.alloc(n, s));
  BCMG_TRY(mid_rows.alloc(n, s));
  BCMG_TRY(n_queued.alloc(2, s));  // [0] rows queued for the long sort, [1] for the mid sort
  BCMG_TRY(nonsym.alloc(1, s));
  int32_t *n_long = n_queued.get(), *n_mid = n_queued.get() + 1;
  BCMG_CUDA(cudaMemsetAsync(n_queued.get(), 0, 2 * sizeof(int32_t), s));
  BCMG_CUDA(cudaMemsetAsync(err.get(), 0, sizeof(int), s));
  BCMG_CUDA(cudaMemsetAsync(nonsym.get(), 0, sizeof(int), s));
  launch(k_sort_prefs, ceil_div(n, kSortWarps * kSortRowsPerWarp), kSortWarps * 32, 0, s, n,
         A.row, A.col, A.val,
         w, C.get(), minb.get(), W_out, sW.get(), scol.get(), inv.get(), ucnt.get(),
         mid_rows.get(), n_mid, long_rows.get(), n_long);
  // Rows of 33..kSortRegMax entries: a grid of a few warps per SM walks the
  // queue (its length stays on the device).
  launch(k_sort_prefs_mid, std::min(ceil_div(n, kSortWarps), 4 * kNumSM), kSortWarps * 32, 0,
         s, mid_rows.get(), n_mid, A.row, A.col, A.val, w, C.get(), minb.get(), W_out,
         sW.get(), scol.get(), inv.get(), ucnt.get());
  {
    const size_t smem = (sizeof(double) + sizeof(int32_t)) * kSortCapLong;
    BCMG_CUDA(cudaFuncSetAttribute(k_sort_prefs_long,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   static_cast<int>(smem)));
    launch(k_sort_prefs_long, std::min(n, kNumSM), 256, smem, s, long_rows.get(),
           n_long, A.row, A.col, A.val, w, C.get(), minb.get(), W_out, sW.get(),
           scol.get(), inv.get(), ucnt.get(), err.get());
    BCMG_LAUNCH_CHECK();
  }
  // every lane group its kKeyRows rows
  auto key_blocks = [&](int g) {
    return ceil_div(static_cast<int64_t>(n) * g, static_cast<int64_t>(T) * kKeyRows);
  };
  switch (G) {
    case 4: launch(k_sym_keys<4>, key_blocks(4), T, 0, s, n, A.row, A.col, A.val, inv.get(), ucnt.get(), E.get(), nonsym.get()); break;
    case 8: launch(k_sym_keys<8>, key_blocks(8), T, 0, s, n, A.row, A.col, A.val, inv.get(), ucnt.get(), E.get(), nonsym.get()); break;
    case 16: launch(k_sym_keys<16>, key_blocks(16), T, 0, s, n, A.row, A.col, A.val, inv.get(), ucnt.get(), E.get(), nonsym.get()); break;
    default: launch(k_sym_keys<32>, key_blocks(32), T, 0, s, n, A.row, A.col, A.val, inv.get(), ucnt.get(), E.get(), nonsym.get()); break;
  }
  BCMG_LAUNCH_CHECK();
  phase_tick("sort_prefs");
  // Both matchers are launched; the one that does not apply (by *nonsym)
  // returns at once, so no host round trip decides between them.
  launch(k_init_match, nb, T, 0, s, n, A.row, next.get(), offer.get());
  const int64_t limit =
      step_limit > 0 ? step_limit : 8 * static_cast<int64_t>(A.nnz) + 1024;
  launch(k_suitor_sym, nb, T, 0, s, n, A.row, ucnt.get(), E.get(), offer.get(), limit,
         nonsym.get(), err.get());
  launch(k_suitor, nb, T, 0, s, n, A.row, scol.get(), sW.get(), next.get(), offer.get(), limit,
         nonsym.get(), err.get());
  BCMG_LAUNCH_CHECK();
  launch(k_offer_to_suitor, nb, T, 0, s, n, offer.get(), scol.get(), nonsym.get(), sv.get());
  phase_tick("suitor");

  // unsymFix.
  launch(k_sym_pairs, nb, T, 0, s, n, sv.get(), mv.get());
  BCMG_CUDA(cudaMemsetAsync(tgt.get(), 0, sizeof(int32_t) * n, s));
  launch(k_unsym_targets, nb, T, 0, s, n, sv.get(), mv.get(), tgt.get());
  BCMG_CUDA(cudaMemcpyAsync(m2.get(), mv.get(), sizeof(int32_t) * n,
                            cudaMemcpyDeviceToDevice, s));
  launch(k_unsym_pairs, nb, T, 0, s, n, sv.get(), mv.get(), tgt.get(), m2.get());

  // Aggregation and canonical numbering.
  launch(k_agg_flags, nb, T, 0, s, n, m2.get(), w, master.get(), p);
  BCMG_LAUNCH_CHECK();
  BCMG_TRY(exclusive_scan(master.get(), rank.get(), n, total.get(), tmp.get(), s));
  launch(k_agg_assign, nb, T, 0, s, n, m2.get(), master.get(), rank.get(), agg);
  BCMG_LAUNCH_CHECK();
  if (s_out)
    BCMG_CUDA(cudaMemcpyAsync(s_out, sv.get(), sizeof(int32_t) * n,
                              cudaMemcpyDeviceToDevice, s));
  if (m_out)
    BCMG_CUDA(cudaMemcpyAsync(m_out, m2.get(), sizeof(int32_t) * n,
                              cudaMemcpyDeviceToDevice, s));
  int h_err = 0;
  int32_t h_nc = 0;
  BCMG_CUDA(cudaMemcpyAsync(&h_err, err.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
  BCMG_CUDA(cudaMemcpyAsync(&h_nc, total.get(), sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  BCMG_CUDA(cudaStreamSynchronize(s));
  if (h_err == 2)
    return set_error(BCMG_ERR_UNSUPPORTED, "a row has more than %d entries", kSortCapLong);
  if (h_err)
    return set_error(BCMG_ERR_DEVICE_TIMEOUT,
                     "suitor matching exceeded its iteration bound (n=%d, nnz=%d)", n,
                     A.nnz);
  *nc_out = h_nc;
  return BCMG_OK;
}

bcmg_status transpose_agg(int32_t n, const int32_t *agg, int32_t nc, int32_t *rptr,
                          int32_t *ridx, cudaStream_t s) {
  if (nc <= 0) return BCMG_OK;
  DevBuf<int32_t> cursor, tmp;
  DevBuf<int> err;
  BCMG_TRY(cursor.alloc(nc, s));
  BCMG_TRY(tmp.alloc(scan_tmp_size(nc), s));
  BCMG_TRY(err.alloc(1, s));
  BCMG_CUDA(cudaMemsetAsync(rptr, 0, sizeof(int32_t) * (nc + 1), s));
  BCMG_CUDA(cudaMemsetAsync(cursor.get(), 0, sizeof(int32_t) * nc, s));
  BCMG_CUDA(cudaMemsetAsync(err.get(), 0, sizeof(int), s));
  launch(k_count_agg, ceil_div(n, 256), 256, 0, s, n, agg, nc, rptr, err.get());
  BCMG_LAUNCH_CHECK();
  BCMG_TRY(exclusive_scan(rptr, rptr, nc, rptr + nc, tmp.get(), s));
  launch(k_fill_agg, ceil_div(n, 256), 256, 0, s, n, agg, nc, rptr, cursor.get(), ridx);
  launch(k_sort_segments, ceil_div(nc, 256), 256, 0, s, nc, rptr, ridx);
  BCMG_LAUNCH_CHECK();
  int h_err = 0;
  BCMG_CUDA(cudaMemcpyAsync(&h_err, err.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
  BCMG_CUDA(cudaStreamSynchronize(s));
  if (h_err)
    return set_error(BCMG_ERR_PARAM, "aggregate index outside [0, %d)", nc);
  return BCMG_OK;
}

// Galerkin product (matchingAggregation.cu:239-244): A_c in CSR, ccol/cval
// allocated here on stream s.
bcmg_status galerkin(const CsrView &A, const int32_t *agg, const double *p, int32_t nc,
                     const int32_t *rptr, const int32_t *ridx, int32_t *crow,
                     int32_t **ccol_out, double **cval_out, int32_t *cnnz, cudaStream_t s) {
  *ccol_out = nullptr;
  *cval_out = nullptr;
  *cnnz = 0;
  if (nc <= 0) return BCMG_OK;
  DevBuf<int32_t> tpos, tJ, long_rows, n_long, mid_rows, n_mid, tmp;
  DevBuf<double> tV;
  DevBuf<int> err;
  BCMG_TRY(tpos.alloc(nc + 1, s));
  BCMG_TRY(tJ.alloc(std::max<int32_t>(A.nnz, 1), s));
  BCMG_TRY(tV.alloc(std::max<int32_t>(A.nnz, 1), s));
  BCMG_TRY(long_rows.alloc(nc, s));
  BCMG_TRY(n_long.alloc(1, s));
  BCMG_TRY(mid_rows.alloc(static_cast<int64_t>(nc) + 1, s));  // (iota writes nc + 1)
  BCMG_TRY(n_mid.alloc(1, s));
  BCMG_TRY(err.alloc(1, s));
  BCMG_TRY(tmp.alloc(scan_tmp_size(nc), s));
  BCMG_CUDA(cudaMemsetAsync(n_long.get(), 0, sizeof(int32_t), s));
  BCMG_CUDA(cudaMemsetAsync(n_mid.get(), 0, sizeof(int32_t), s));
  BCMG_CUDA(cudaMemsetAsync(err.get(), 0, sizeof(int), s));
  launch(k_gal_terms, ceil_div(nc, 256), 256, 0, s, nc, A.row, rptr, ridx, tpos.get());
  BCMG_TRY(exclusive_scan(tpos.get(), tpos.get(), nc, tpos.get() + nc, tmp.get(), s));
  phase_tick("gal_terms");
  const size_t smem_warp = static_cast<size_t>(kGalWarpsPerBlock) * kGalCap * kGalBytesPerTerm;
  const size_t smem_long = static_cast<size_t>(kGalCapLong) * kGalBytesPerTerm;
  BCMG_CUDA(cudaFuncSetAttribute(k_gal_rows_long, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(smem_long)));
  if (nc < (1 << 26)) {
    // Short rows in registers; the rest queued for the shared-memory sort.
    launch(k_gal_rows_reg, ceil_div(nc, kGalRegWarps), kGalRegWarps * 32, 0, s, nc, A.row,
           A.col, A.val, agg, p, rptr, ridx, tpos.get(), tJ.get(), tV.get(), crow,
           mid_rows.get(), n_mid.get(), err.get());
  } else {
    BCMG_TRY(iota(nc, mid_rows.get(), s));
    BCMG_CUDA(cudaMemcpyAsync(n_mid.get(), &nc, sizeof(int32_t), cudaMemcpyHostToDevice, s));
  }
  launch(k_gal_rows, std::min(ceil_div(nc, kGalWarpsPerBlock), 16 * kNumSM),
         kGalWarpsPerBlock * 32, smem_warp, s, mid_rows.get(), n_mid.get(), A.row, A.col, A.val,
         agg, p, rptr, ridx, tpos.get(), tJ.get(), tV.get(), crow, long_rows.get(),
         n_long.get(), err.get());
  launch(k_gal_rows_long, std::min(nc, kNumSM), kGalLongThreads, smem_long, s, long_rows.get(),
         n_long.get(), A.row, A.col, A.val, agg, p, rptr, ridx, tpos.get(), tJ.get(), tV.get(),
         crow, err.get());
  BCMG_LAUNCH_CHECK();
  phase_tick("gal_rows");
  // crow holds the run counts: scan them into row pointers.
  BCMG_TRY(exclusive_scan(crow, crow, nc, crow + nc, tmp.get(), s));
  int h_err = 0;
  int32_t h_nnz = 0;
  BCMG_CUDA(cudaMemcpyAsync(&h_err, err.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
  BCMG_CUDA(cudaMemcpyAsync(&h_nnz, crow + nc, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  BCMG_CUDA(cudaStreamSynchronize(s));
  if (h_err == 3)
    return set_error(BCMG_ERR_UNSUPPORTED,
                     "a coarse row has more than %d Galerkin terms", kGalCapLong);
  if (h_err)
    return set_error(BCMG_ERR_INTERNAL, "Galerkin run longer than %d terms", kGalMaxRun);
  DevBuf<int32_t> ccol;
  DevBuf<double> cval;
  BCMG_TRY(ccol.alloc(std::max<int32_t>(h_nnz, 1), s));
  BCMG_TRY(cval.alloc(std::max<int32_t>(h_nnz, 1), s));
  launch(k_gal_compact, ceil_div(static_cast<int64_t>(nc) * 32, 256), 256, 0, s, nc, tpos.get(),
         crow, tJ.get(), tV.get(), ccol.get(), cval.get());
  BCMG_LAUNCH_CHECK();
  *cnnz = h_nnz;
  *ccol_out = ccol.release();
  *cval_out = cval.release();
  return BCMG_OK;
}

bcmg_status restrict_exact(int32_t nc, const int32_t *rptr, const int32_t *ridx,
                           const double *p, const double *x, double *y, cudaStream_t s) {
  if (nc <= 0) return BCMG_OK;
  launch(k_restrict_exact, ceil_div(nc, 256), 256, 0, s, nc, rptr, ridx, p, x, y);
  BCMG_LAUNCH_CHECK();
  return BCMG_OK;
}

bcmg_status compose_p(int32_t n, int32_t *agg, double *p, const int32_t *agg2,
                      const double *p2, cudaStream_t s) {
  if (n <= 0) return BCMG_OK;
  launch(k_compose, ceil_div(n, 256), 256, 0, s, n, agg, p, agg2, p2);
  BCMG_LAUNCH_CHECK();
  return BCMG_OK;
}

bcmg_status spgemm(const CsrView &X, const CsrView &Y, int32_t m, int32_t *crow,
                   int32_t **ccol_out, double **cval_out, int32_t *cnnz, cudaStream_t s) {
  *ccol_out = nullptr;
  *cval_out = nullptr;
  *cnnz = 0;
  const int32_t n = X.n;
  if (n <= 0) return BCMG_OK;
  DevBuf<int32_t> list1, list2, counts, tmp;
  DevBuf<unsigned char> tier;
  DevBuf<int> err;
  BCMG_TRY(list1.alloc(n, s));
  BCMG_TRY(list2.alloc(n, s));
  BCMG_TRY(counts.alloc(2, s));  // rows in tier 1, tier 2
  BCMG_TRY(tier.alloc(n, s));
  BCMG_TRY(err.alloc(1, s));
  BCMG_TRY(tmp.alloc(scan_tmp_size(n), s));
  BCMG_CUDA(cudaMemsetAsync(counts.get(), 0, 2 * sizeof(int32_t), s));
  BCMG_CUDA(cudaMemsetAsync(err.get(), 0, sizeof(int), s));
  const size_t smem_warp = kSpWarpsPerBlock * sp_table_bytes(kSpWarpHash);
  const size_t smem_warp_fill =
      kSpWarpsPerBlock * (sp_table_bytes(kSpWarpHash) + kSpStageWarpBytes);
  const size_t smem_block = sp_table_bytes(kSpBlockHash);
  const size_t smem_block_fill = kSpStageBlockBytes + sp_table_bytes(kSpBlockHash);
  BCMG_CUDA(cudaFuncSetAttribute(k_sp_count_warp, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(smem_warp)));
  BCMG_CUDA(cudaFuncSetAttribute(k_sp_fill_warp, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(smem_warp_fill)));
  BCMG_CUDA(cudaFuncSetAttribute(k_sp_count_block, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(smem_block)));
  BCMG_CUDA(cudaFuncSetAttribute(k_sp_fill_block, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(smem_block_fill)));
  const int warp_grid = ceil_div(n, kSpWarpsPerBlock);
  const int block_grid = std::min(n, 2 * kNumSM);  // two blocks per SM
  launch(k_sp_count_warp, warp_grid, kSpWarpsPerBlock * 32, smem_warp, s, n, X.row, X.col,
         Y.row, Y.col, crow, tier.get(), list1.get(), counts.get());
  phase_tick("sp count warp");
  launch(k_sp_count_block, block_grid, kSpThreads, smem_block, s, list1.get(), counts.get(),
         X.row, X.col, Y.row, Y.col, m, crow, tier.get(), list2.get(), counts.get() + 1,
         static_cast<unsigned char *>(nullptr), 0, 1, err.get());
  BCMG_LAUNCH_CHECK();
  int32_t h_counts[2] = {0, 0};
  BCMG_CUDA(cudaMemcpyAsync(h_counts, counts.get(), sizeof(h_counts), cudaMemcpyDeviceToHost, s));
  BCMG_CUDA(cudaStreamSynchronize(s));
  phase_tick("sp count block");
  // Tier 2: a table of ghc slots per block in global memory, ghc a power of
  // two at least twice the row bound min(terms, m), at most 1 GiB in all.
  DevBuf<unsigned char> gtab;
  int ghc = 0, g_grid = 0;
  if (h_counts[1] > 0) {
    DevBuf<unsigned long long> maxt;
    BCMG_TRY(maxt.alloc(1, s));
    BCMG_CUDA(cudaMemsetAsync(maxt.get(), 0, sizeof(unsigned long long), s));
    launch(k_sp_max_terms, ceil_div(n, 256), 256, 0, s, n, X.row, X.col, Y.row, maxt.get());
    unsigned long long h_maxt = 0;
    BCMG_CUDA(cudaMemcpyAsync(&h_maxt, maxt.get(), sizeof(h_maxt), cudaMemcpyDeviceToHost, s));
    BCMG_CUDA(cudaStreamSynchronize(s));
    const int64_t bound = std::min<int64_t>(static_cast<int64_t>(h_maxt), m);
    int64_t c = kSpBlockHash;
    while (c < 2 * bound + 2) c <<= 1;
    constexpr int64_t kTableBudget = int64_t(1) << 30;
    const int64_t per = static_cast<int64_t>(sp_table_bytes(static_cast<int>(
        std::min<int64_t>(c, int64_t(1) << 30))));
    if (c > (int64_t(1) << 26) || per > kTableBudget)
      return set_error(BCMG_ERR_UNSUPPORTED, "sparse product: a row with %lld columns",
                       static_cast<long long>(bound));
    ghc = static_cast<int>(c);
    const int64_t fit = std::min<int64_t>(kTableBudget / per, std::min(h_counts[1], 4 * kNumSM));
    g_grid = static_cast<int>(std::max<int64_t>(1, fit));
    BCMG_TRY(gtab.alloc(per * g_grid, s));
    launch(k_sp_count_block, g_grid, kSpThreads, 0, s, list2.get(), counts.get() + 1, X.row,
           X.col, Y.row, Y.col, m, crow, tier.get(), static_cast<int32_t *>(nullptr),
           static_cast<int32_t *>(nullptr), gtab.get(), ghc, 2, err.get());
    phase_tick("sp count global");
  }
  BCMG_TRY(exclusive_scan(crow, crow, n, crow + n, tmp.get(), s));
  int h_err = 0;
  int32_t h_nnz = 0;
  BCMG_CUDA(cudaMemcpyAsync(&h_err, err.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
  BCMG_CUDA(cudaMemcpyAsync(&h_nnz, crow + n, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  BCMG_CUDA(cudaStreamSynchronize(s));
  if (h_err) return set_error(BCMG_ERR_INTERNAL, "sparse product: row over its table");
  if (h_nnz < 0) return set_error(BCMG_ERR_UNSUPPORTED, "sparse product over 2^31 entries");
  DevBuf<int32_t> ccol;
  DevBuf<double> cval;
  BCMG_TRY(ccol.alloc(std::max<int32_t>(h_nnz, 1), s));
  BCMG_TRY(cval.alloc(std::max<int32_t>(h_nnz, 1), s));
  launch(k_sp_fill_warp, warp_grid, kSpWarpsPerBlock * 32, smem_warp_fill, s, n, X.row, X.col,
         X.val, Y.row, Y.col, Y.val, tier.get(), crow, ccol.get(), cval.get());
  phase_tick("sp fill warp");
  if (h_counts[0] > 0)
    launch(k_sp_fill_block, block_grid, kSpThreads, smem_block_fill, s, list1.get(), counts.get(),
           X.row, X.col, X.val, Y.row, Y.col, Y.val, tier.get(), crow, ccol.get(), cval.get(),
           static_cast<unsigned char *>(nullptr), 0, 1);
  phase_tick("sp fill block");
  if (h_counts[1] > 0)
    launch(k_sp_fill_block, g_grid, kSpThreads, kSpStageBlockBytes, s, list2.get(), counts.get() + 1, X.row,
           X.col, X.val, Y.row, Y.col, Y.val, tier.get(), crow, ccol.get(), cval.get(),
           gtab.get(), ghc, 2);
  BCMG_LAUNCH_CHECK();
  phase_tick("sp fill global");
  *cnnz = h_nnz;
  *ccol_out = ccol.release();
  *cval_out = cval.release();
  return BCMG_OK;
}

bcmg_status csr_transpose(const CsrView &A, int32_t m, int32_t *trow, int32_t *tcol,
                          double *tval, cudaStream_t s) {
  DevBuf<int32_t> cursor, tmp;
  DevBuf<int> err;
  BCMG_TRY(cursor.alloc(std::max(m, 1), s));
  BCMG_TRY(tmp.alloc(scan_tmp_size(m), s));
  BCMG_TRY(err.alloc(1, s));
  BCMG_CUDA(cudaMemsetAsync(trow, 0, sizeof(int32_t) * (m + 1), s));
  BCMG_CUDA(cudaMemsetAsync(cursor.get(), 0, sizeof(int32_t) * std::max(m, 1), s));
  BCMG_CUDA(cudaMemsetAsync(err.get(), 0, sizeof(int), s));
  if (A.nnz > 0)
    launch(k_tr_count, ceil_div(A.nnz, 256), 256, 0, s, A.nnz, A.col, m, trow, err.get());
  BCMG_TRY(exclusive_scan(trow, trow, m, trow + m, tmp.get(), s));
  launch(k_tr_fill, ceil_div(A.n, 256), 256, 0, s, A.n, A.row, A.col, A.val, m, trow,
         cursor.get(), tcol, tval);
  const size_t tr_smem = static_cast<size_t>(kTrSmem) * (sizeof(double) + sizeof(int32_t));
  BCMG_CUDA(cudaFuncSetAttribute(k_tr_sort, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(tr_smem)));
  if (m > 0)
    launch(k_tr_sort, std::min(m, 2 * kNumSM), kTrThreads, tr_smem, s, m, trow, tcol, tval);
  BCMG_LAUNCH_CHECK();
  int h_err = 0;
  BCMG_CUDA(cudaMemcpyAsync(&h_err, err.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
  BCMG_CUDA(cudaStreamSynchronize(s));
  if (h_err) return set_error(BCMG_ERR_INTERNAL, "transpose: column outside [0, %d)", m);
  return BCMG_OK;
}

bcmg_status smoothing_operator(const CsrView &A, const double *D, double *sval,
                               cudaStream_t s) {
  DevBuf<unsigned long long> inf;
  BCMG_TRY(inf.alloc(1, s));
  BCMG_CUDA(cudaMemsetAsync(inf.get(), 0, sizeof(unsigned long long), s));
  launch(k_smooth_scale, ceil_div(A.n, 256), 256, 0, s, A.n, A.row, A.val, D, sval, inf.get());
  unsigned long long bits = 0;
  BCMG_CUDA(cudaMemcpyAsync(&bits, inf.get(), sizeof(bits), cudaMemcpyDeviceToHost, s));
  BCMG_CUDA(cudaStreamSynchronize(s));
  double norm;
  std::memcpy(&norm, &bits, sizeof(norm));
  if (!(norm > 0.0) || !std::isfinite(norm))
    return set_error(BCMG_ERR_INVALID_MATRIX, "smoothed aggregation: bad ||D^-1 A||_inf");
  const double omega = 4.0 / (3.0 * norm);
  launch(k_smooth_omega, ceil_div(A.n, 256), 256, 0, s, A.n, A.row, A.col, omega, sval);
  BCMG_LAUNCH_CHECK();
  return BCMG_OK;
}

bcmg_status iota(int32_t n, int32_t *x, cudaStream_t s) {
  launch(k_iota, ceil_div(static_cast<int64_t>(n) + 1, 256), 256, 0, s, n, x);
  BCMG_LAUNCH_CHECK();
  return BCMG_OK;
}

}  // namespace bcmg
