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
// src/AMG/matching.cu:319-329,401-431).  Non-negative doubles order like
// their bit patterns, so the global min is an integer atomicMin.
template <int G>
__global__ void k_ah_min(int32_t n, const int32_t *__restrict__ row,
                         const int32_t *__restrict__ col,
                         const double *__restrict__ val, const double *__restrict__ w,
                         const double *__restrict__ C, unsigned long long *min_bits) {
  const int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  const int32_t i = static_cast<int32_t>(t / G);
  const int lane = threadIdx.x % G;
  double m = DBL_MAX;
  if (i < n) {
    const double ci = C[i], wi = w[i];
    for (int32_t j = row[i] + lane; j < row[i + 1]; j += G) {
      const int32_t c = col[j];
      if (c == i) continue;
      const double ah = fabs(ah_value(val[j], ci, C[c], wi, w[c]));
      if (ah < m) m = ah;
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmin(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0 && m < DBL_MAX)
    atomicMin(min_bits, static_cast<unsigned long long>(__double_as_longlong(m)));
}

// W_ij = log(|AH_ij| / (0.999 mu)) (_make_w with MAXIMUM_PRODUCT_MATRIX_OP 1,
// src/AMG/matching.cu:387-395), stored over A's pattern with 0 on the
// diagonal (the matcher ignores weights <= 0).
template <int G>
__global__ void k_make_W(int32_t n, const int32_t *__restrict__ row,
                         const int32_t *__restrict__ col,
                         const double *__restrict__ val, const double *__restrict__ w,
                         const double *__restrict__ C,
                         const unsigned long long *__restrict__ min_bits,
                         double *__restrict__ W) {
  const int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  const int32_t i = static_cast<int32_t>(t / G);
  const int lane = threadIdx.x % G;
  if (i >= n) return;
  const double den = 0.999 * __longlong_as_double(static_cast<long long>(*min_bits));
  const double ci = C[i], wi = w[i];
  for (int32_t j = row[i] + lane; j < row[i + 1]; j += G) {
    const int32_t c = col[j];
    W[j] = (c == i) ? 0.0 : log(fabs(ah_value(val[j], ci, C[c], wi, w[c])) / den);
  }
}

// Suitor matching (kernel_for_matching, src/AMG/suitor.cu:242-392).  A group
// of G lanes works one proposer at a time: it finds the neighbour y of
// largest (W_xy, y) whose current offer it beats (find_Candidate,
// suitor.cu:118-214), then installs its offer with a 64-bit CAS.  An offer is
// (edge index << 32 | proposer): the edge index recovers the immutable weight,
// so no lock is needed (the reference spins on per-vertex locks,
// suitor.cu:19-38,69-110).  A displaced proposer is taken over by the
// displacing group (set_suitor, suitor.cu:89-93).  Offers only increase under
// the strict order (weight, proposer id), so the final state is the unique
// proposer-optimal one whatever the interleaving.  Each group is bounded by
// `limit` iterations; on overrun it raises *err and returns.
template <int G>
__global__ void k_suitor(int32_t n, const int32_t *__restrict__ row,
                         const int32_t *__restrict__ col, const double *__restrict__ W,
                         unsigned long long *offer, int64_t limit, int *err) {
  const int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  const int32_t gid = static_cast<int32_t>(t / G);
  const int lane = threadIdx.x % G;
  if (gid >= n) return;
  const unsigned mask = group_mask<G>();
  volatile unsigned long long *voffer = offer;
  int32_t cur = gid;
  for (int64_t it = 0;; ++it) {
    if (it >= limit) {
      if (lane == 0) atomicExch(err, 1);
      return;
    }
    double bw = 0.0;
    int32_t by = -1, be = -1;
    unsigned long long bo = kNoOffer;
    const int32_t jb = row[cur], je = row[cur + 1];
    for (int32_t k = jb + lane; k < je; k += G) {
      const int32_t y = col[k];
      const double we = W[k];
      if (y == cur || !(we > 0.0)) continue;
      const unsigned long long o = voffer[y];
      double cw = 0.0;
      int32_t cid = -1;
      if (o != kNoOffer) {
        cw = W[static_cast<int32_t>(o >> 32)];
        cid = static_cast<int32_t>(o & 0xffffffffull);
      }
      if (!(we > cw || (we == cw && cur > cid))) continue;
      if (by < 0 || we > bw || (we == bw && y > by)) {
        bw = we;
        by = y;
        be = k;
        bo = o;
      }
    }
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) {
      const double w2 = __shfl_xor_sync(mask, bw, o, G);
      const int32_t y2 = __shfl_xor_sync(mask, by, o, G);
      const int32_t e2 = __shfl_xor_sync(mask, be, o, G);
      const unsigned long long o2 = __shfl_xor_sync(mask, bo, o, G);
      const bool better = y2 >= 0 && (by < 0 || w2 > bw || (w2 == bw && y2 > by));
      if (better) {
        bw = w2;
        by = y2;
        be = e2;
        bo = o2;
      }
    }
    if (by < 0) return;
    unsigned long long old = 0;
    if (lane == 0)
      old = atomicCAS(offer + by, bo,
                      (static_cast<unsigned long long>(static_cast<uint32_t>(be)) << 32) |
                          static_cast<uint32_t>(cur));
    old = __shfl_sync(mask, old, 0, G);
    if (old == bo) {
      if (bo == kNoOffer) return;
      cur = static_cast<int32_t>(bo & 0xffffffffull);
    }
  }
}

__global__ void k_offer_to_suitor(int32_t n, const unsigned long long *__restrict__ offer,
                                  int32_t *s) {
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const unsigned long long o = offer[i];
  s[i] = o == kNoOffer ? -1 : static_cast<int32_t>(o & 0xffffffffull);
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
};

__device__ __forceinline__ GalSmem gal_smem(unsigned char *base, int cap) {
  GalSmem s;
  s.key = reinterpret_cast<unsigned long long *>(base);
  s.tv = reinterpret_cast<double *>(base + sizeof(unsigned long long) * cap);
  s.ti = reinterpret_cast<int32_t *>(base + 16 * cap);
  s.tj = reinterpret_cast<int32_t *>(base + 20 * cap);
  return s;
}
constexpr int kGalBytesPerTerm = 24;

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
        const int i0 = 2 * j * (t / j) + (t % j);
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

// Sums the run starting at head position k; returns false if the run is
// longer than kGalMaxRun.
__device__ bool gal_run_sum(const GalSmem &sm, int k, int T, int32_t *J, double *sum) {
  const unsigned long long jj = sm.key[k] >> 32;
  int idx[kGalMaxRun];
  int r = 0;
  for (int q = k; q < T && (sm.key[q] >> 32) == jj; ++q) {
    if (r == kGalMaxRun) return false;
    idx[r++] = static_cast<int>(sm.key[q] & 0xffffffffull);
  }
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

// Warp-team Galerkin: FILL=false counts distinct coarse columns into cnt[I];
// FILL=true writes row I.  Rows over kGalCap terms are queued for the block
// kernel (count pass) or skipped (fill pass).
template <bool FILL>
__global__ void __launch_bounds__(kGalWarpsPerBlock * 32)
    k_gal_warp(int32_t nc, const int32_t *__restrict__ row,
               const int32_t *__restrict__ col, const double *__restrict__ val,
               const int32_t *__restrict__ agg, const double *__restrict__ p,
               const int32_t *__restrict__ rptr, const int32_t *__restrict__ ridx,
               int32_t *cnt_or_crow, int32_t *ccol, double *cval, int32_t *long_rows,
               int32_t *n_long, int *err) {
  extern __shared__ __align__(16) unsigned char gal_dyn[];
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int32_t I = blockIdx.x * kGalWarpsPerBlock + wid;
  if (I >= nc) return;
  GalSmem sm = gal_smem(gal_dyn + static_cast<size_t>(wid) * kGalCap * kGalBytesPerTerm,
                        kGalCap);
  const int T = gal_gather<32>(I, row, col, val, agg, p, rptr, ridx, sm, kGalCap, lane);
  if (T < 0) {
    if (!FILL && lane == 0) {
      long_rows[atomicAdd(n_long, 1)] = I;
      cnt_or_crow[I] = 0;
    }
    return;
  }
  int carry = 0;
  const int32_t out0 = FILL ? cnt_or_crow[I] : 0;
  for (int base = 0; base < T; base += 32) {
    const int k = base + lane;
    const bool h = k < T && gal_head(sm, k);
    const unsigned hm = __ballot_sync(0xffffffffu, h);
    if (FILL && h) {
      int32_t J;
      double s;
      if (gal_run_sum(sm, k, T, &J, &s)) {
        const int32_t pos = out0 + carry + __popc(hm & ((1u << lane) - 1u));
        ccol[pos] = J;
        cval[pos] = s;
      } else {
        atomicExch(err, 2);
      }
    }
    carry += __popc(hm);
  }
  if (!FILL && lane == 0) cnt_or_crow[I] = carry;
}

// Block-team Galerkin for the queued long rows (one block per row).
template <bool FILL>
__global__ void __launch_bounds__(kGalLongThreads)
    k_gal_long(const int32_t *__restrict__ long_rows, const int32_t *__restrict__ row,
               const int32_t *__restrict__ col, const double *__restrict__ val,
               const int32_t *__restrict__ agg, const double *__restrict__ p,
               const int32_t *__restrict__ rptr, const int32_t *__restrict__ ridx,
               int32_t *cnt_or_crow, int32_t *ccol, double *cval, int *err) {
  extern __shared__ __align__(16) unsigned char gal_dyn[];
  const int32_t I = long_rows[blockIdx.x];
  GalSmem sm = gal_smem(gal_dyn, kGalCapLong);
  const int T = gal_gather<kGalLongThreads>(I, row, col, val, agg, p, rptr, ridx, sm,
                                            kGalCapLong, threadIdx.x);
  if (T < 0) {
    if (threadIdx.x == 0) atomicExch(err, 3);
    return;
  }
  if (threadIdx.x >= 32) return;
  const int lane = threadIdx.x;
  int carry = 0;
  const int32_t out0 = FILL ? cnt_or_crow[I] : 0;
  for (int base = 0; base < T; base += 32) {
    const int k = base + lane;
    const bool h = k < T && gal_head(sm, k);
    const unsigned hm = __ballot_sync(0xffffffffu, h);
    if (FILL && h) {
      int32_t J;
      double s;
      if (gal_run_sum(sm, k, T, &J, &s)) {
        const int32_t pos = out0 + carry + __popc(hm & ((1u << lane) - 1u));
        ccol[pos] = J;
        cval[pos] = s;
      } else {
        atomicExch(err, 2);
      }
    }
    carry += __popc(hm);
  }
  if (!FILL && lane == 0) cnt_or_crow[I] = carry;
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
bcmg_status launch_weights(const CsrView &A, const double *w, const double *C,
                           unsigned long long *min_bits, double *W, cudaStream_t s) {
  const int threads = 256;
  const int blocks = ceil_div(static_cast<int64_t>(A.n) * G, threads);
  launch(k_ah_min<G>, blocks, threads, 0, s, A.n, A.row, A.col, A.val, w, C, min_bits);
  launch(k_make_W<G>, blocks, threads, 0, s, A.n, A.row, A.col, A.val, w, C, min_bits, W);
  BCMG_LAUNCH_CHECK();
  return BCMG_OK;
}

template <int G>
void launch_suitor(const CsrView &A, const double *W, unsigned long long *offer,
                   int64_t limit, int *err, cudaStream_t s) {
  const int threads = 256;
  const int blocks = ceil_div(static_cast<int64_t>(A.n) * G, threads);
  launch(k_suitor<G>, blocks, threads, 0, s, A.n, A.row, A.col, W, offer, limit, err);
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
                           int32_t *m_out, cudaStream_t s) {
  const int32_t n = A.n;
  if (n <= 0) {
    *nc_out = 0;
    return BCMG_OK;
  }
  const int T = 256;
  const int nb = ceil_div(n, T);
  DevBuf<double> C, Wb;
  DevBuf<unsigned long long> offer, minb;
  DevBuf<int32_t> sv, mv, m2, tgt, master, rank, tmp, total;
  DevBuf<int> err;
  BCMG_TRY(C.alloc(n, s));
  double *W = W_out;
  if (!W) {
    BCMG_TRY(Wb.alloc(A.nnz, s));
    W = Wb.get();
  }
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
    case 4: BCMG_TRY(launch_weights<4>(A, w, C.get(), minb.get(), W, s)); break;
    case 8: BCMG_TRY(launch_weights<8>(A, w, C.get(), minb.get(), W, s)); break;
    case 16: BCMG_TRY(launch_weights<16>(A, w, C.get(), minb.get(), W, s)); break;
    default: BCMG_TRY(launch_weights<32>(A, w, C.get(), minb.get(), W, s)); break;
  }

  // Suitor matching; every group is bounded by the total number of
  // successful offers (<= nnz) plus failed CASes (each caused by a success).
  BCMG_CUDA(cudaMemsetAsync(offer.get(), 0xff, sizeof(unsigned long long) * n, s));
  BCMG_CUDA(cudaMemsetAsync(err.get(), 0, sizeof(int), s));
  const int64_t limit = 2 * static_cast<int64_t>(A.nnz) + 64;
  switch (G) {
    case 4: launch_suitor<4>(A, W, offer.get(), limit, err.get(), s); break;
    case 8: launch_suitor<8>(A, W, offer.get(), limit, err.get(), s); break;
    case 16: launch_suitor<16>(A, W, offer.get(), limit, err.get(), s); break;
    default: launch_suitor<32>(A, W, offer.get(), limit, err.get(), s); break;
  }
  BCMG_LAUNCH_CHECK();
  launch(k_offer_to_suitor, nb, T, 0, s, n, offer.get(), sv.get());

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

namespace {

bcmg_status galerkin_pass(bool fill, const CsrView &A, const int32_t *agg,
                          const double *p, int32_t nc, const int32_t *rptr,
                          const int32_t *ridx, int32_t *crow, int32_t *cnnz,
                          int32_t *ccol, double *cval, cudaStream_t s) {
  if (nc <= 0) {
    if (cnnz) *cnnz = 0;
    return BCMG_OK;
  }
  DevBuf<int32_t> long_rows, n_long, tmp;
  DevBuf<int> err;
  BCMG_TRY(long_rows.alloc(nc, s));
  BCMG_TRY(n_long.alloc(1, s));
  BCMG_TRY(err.alloc(1, s));
  BCMG_CUDA(cudaMemsetAsync(n_long.get(), 0, sizeof(int32_t), s));
  BCMG_CUDA(cudaMemsetAsync(err.get(), 0, sizeof(int), s));
  const size_t smem_warp = static_cast<size_t>(kGalWarpsPerBlock) * kGalCap * kGalBytesPerTerm;
  const size_t smem_long = static_cast<size_t>(kGalCapLong) * kGalBytesPerTerm;
  BCMG_CUDA(cudaFuncSetAttribute(k_gal_long<false>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(smem_long)));
  BCMG_CUDA(cudaFuncSetAttribute(k_gal_long<true>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(smem_long)));
  const int blocks = ceil_div(nc, kGalWarpsPerBlock);
  // The count pass queues the long rows; the fill pass recomputes the queue
  // the same way by running the count kernel's gather check again.
  if (!fill) {
    launch(k_gal_warp<false>, blocks, kGalWarpsPerBlock * 32, smem_warp, s, 
        nc, A.row, A.col, A.val, agg, p, rptr, ridx, crow, nullptr, nullptr,
        long_rows.get(), n_long.get(), err.get());
  } else {
    // Re-detect long rows without touching crow: count into a scratch array.
    DevBuf<int32_t> scratch;
    BCMG_TRY(scratch.alloc(nc, s));
    launch(k_gal_warp<false>, blocks, kGalWarpsPerBlock * 32, smem_warp, s, 
        nc, A.row, A.col, A.val, agg, p, rptr, ridx, scratch.get(), nullptr, nullptr,
        long_rows.get(), n_long.get(), err.get());
    launch(k_gal_warp<true>, blocks, kGalWarpsPerBlock * 32, smem_warp, s, 
        nc, A.row, A.col, A.val, agg, p, rptr, ridx, crow, ccol, cval, long_rows.get(),
        n_long.get(), err.get());
  }
  BCMG_LAUNCH_CHECK();
  int32_t h_long = 0;
  BCMG_CUDA(cudaMemcpyAsync(&h_long, n_long.get(), sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  BCMG_CUDA(cudaStreamSynchronize(s));
  if (h_long > 0) {
    if (!fill)
      launch(k_gal_long<false>, h_long, kGalLongThreads, smem_long, s, 
          long_rows.get(), A.row, A.col, A.val, agg, p, rptr, ridx, crow, nullptr,
          nullptr, err.get());
    else
      launch(k_gal_long<true>, h_long, kGalLongThreads, smem_long, s, 
          long_rows.get(), A.row, A.col, A.val, agg, p, rptr, ridx, crow, ccol, cval,
          err.get());
    BCMG_LAUNCH_CHECK();
  }
  if (!fill) {
    BCMG_TRY(tmp.alloc(scan_tmp_size(nc), s));
    BCMG_TRY(exclusive_scan(crow, crow, nc, crow + nc, tmp.get(), s));
    BCMG_CUDA(cudaMemcpyAsync(cnnz, crow + nc, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  }
  int h_err = 0;
  BCMG_CUDA(cudaMemcpyAsync(&h_err, err.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
  BCMG_CUDA(cudaStreamSynchronize(s));
  if (h_err == 3)
    return set_error(BCMG_ERR_UNSUPPORTED,
                     "a coarse row has more than %d Galerkin terms", kGalCapLong);
  if (h_err)
    return set_error(BCMG_ERR_INTERNAL, "Galerkin run longer than %d terms", kGalMaxRun);
  return BCMG_OK;
}

}  // namespace

bcmg_status galerkin_count(const CsrView &A, const int32_t *agg, const double *p,
                           int32_t nc, const int32_t *rptr, const int32_t *ridx,
                           int32_t *crow, int32_t *cnnz, cudaStream_t s) {
  return galerkin_pass(false, A, agg, p, nc, rptr, ridx, crow, cnnz, nullptr, nullptr, s);
}

bcmg_status galerkin_fill(const CsrView &A, const int32_t *agg, const double *p,
                          int32_t nc, const int32_t *rptr, const int32_t *ridx,
                          const int32_t *crow, int32_t *ccol, double *cval,
                          cudaStream_t s) {
  return galerkin_pass(true, A, agg, p, nc, rptr, ridx, const_cast<int32_t *>(crow),
                       nullptr, ccol, cval, s);
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

}  // namespace bcmg
