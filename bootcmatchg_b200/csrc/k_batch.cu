// Multi-right-hand-side cycle and FCG kernels on interleaved n x W blocks
// (element (i, c) at x[i * W + c]).  The cycle operations follow the
// single-vector ones -- _jacobi_it (src/AMG/relaxation.cu:176-209), the
// residual / restriction / prolongation of GAMG_cycle
// (src/SOLVER/GAMG_cycle.cu:57-119) -- applied to every column, and the FCG
// kernels are the FCG v3 recurrences (src/SOLVER/FCG.cu:433-585) with one set
// of scalars per column.  The reference solves one right-hand side per call;
// sharing a hierarchy across columns is this library's extension.
//
// Row kernels: a group of L = W / V lanes handles one matrix row, lane g owns
// columns [g V, g V + V).  The group loads L entries (column, value) of the
// row at a time, coalesced, and passes them around with shuffles; each lane
// then gathers its V columns of x at every entry.  The matrix is therefore
// read once per W right-hand sides, and each column's row sum is a
// sequential FMA chain in CSR order, independent of V and of the block size.
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <cfloat>
#include <type_traits>

#include "batch.h"
#include "common.cuh"

namespace bcmg {
namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kUnroll = 8;       // entries whose gathers are in flight together
constexpr int kRedT = 256;       // threads of the reduction kernels
constexpr int kRedWarps = kRedT / 32;

__device__ __forceinline__ double widen(double v) { return v; }
__device__ __forceinline__ float widen(float v) { return v; }
__device__ __forceinline__ float widen(__nv_bfloat16 v) { return __bfloat162float(v); }
__device__ __forceinline__ float widen(__half v) { return __half2float(v); }

// V consecutive columns of one row, loaded and stored as one vector access.
template <typename XT, int V>
struct alignas(sizeof(XT) * V) Cols {
  XT v[V];
};

template <typename XT, int V>
__device__ __forceinline__ Cols<XT, V> ldc(const XT *__restrict__ p) {
  return *reinterpret_cast<const Cols<XT, V> *>(p);
}
template <typename XT, int V>
__device__ __forceinline__ void stc(XT *__restrict__ p, const Cols<XT, V> &c) {
  *reinterpret_cast<Cols<XT, V> *>(p) = c;
}

__host__ __device__ inline int ilog2(int v) {
  int l = 0;
  while ((1 << l) < v) ++l;
  return l;
}

// acc[v] = sum_j a_ij x[col_j, g V + v] for the group's row i (len entries
// from j0; len = 0 for rows past the end).  All 32 lanes of the warp must
// call it together: the loop bounds are warp-uniform.
template <int V, typename VT, typename XT>
__device__ __forceinline__ void bt_row_sum(const int32_t *__restrict__ col,
                                           const VT *__restrict__ val,
                                           const XT *__restrict__ x, int W, int L, int g,
                                           int32_t j0, int len, XT (&acc)[V]) {
  const int maxlen = static_cast<int>(__reduce_max_sync(kFull, static_cast<unsigned>(len)));
  const int64_t cofs = static_cast<int64_t>(g) * V;
#pragma unroll
  for (int v = 0; v < V; ++v) acc[v] = XT(0);
  for (int base = 0; base < maxlen; base += L) {
    int32_t cj = 0;
    XT vj = XT(0);
    if (base + g < len) {
      cj = col[j0 + base + g];
      vj = static_cast<XT>(widen(val[j0 + base + g]));
    }
    const int kn = min(L, maxlen - base);
    for (int k0 = 0; k0 < kn; k0 += kUnroll) {
      int32_t ck[kUnroll];
      XT vk[kUnroll];
#pragma unroll
      for (int u = 0; u < kUnroll; ++u) {
        ck[u] = __shfl_sync(kFull, cj, k0 + u, L);
        vk[u] = __shfl_sync(kFull, vj, k0 + u, L);
      }
      Cols<XT, V> xv[kUnroll];
      // All kUnroll gathers are issued unconditionally, so they are in flight
      // together: an absent entry carries column 0 (a valid row) and its
      // product is dropped below.  Entry k0 + u exists for this row when it
      // lies inside both the chunk (kn entries) and the row.
#pragma unroll
      for (int u = 0; u < kUnroll; ++u)
        xv[u] = ldc<XT, V>(x + static_cast<int64_t>(ck[u]) * W + cofs);
#pragma unroll
      for (int u = 0; u < kUnroll; ++u)
        if (k0 + u < kn && base + k0 + u < len) {
#pragma unroll
          for (int v = 0; v < V; ++v) acc[v] = fma(vk[u], xv[u].v[v], acc[v]);
        }
    }
  }
}

enum { kModeRelax = 0, kModeResid = 1, kModeSpmv = 2 };

// kModeRelax: out = ((-(A u) + f) ./ d) + u;  kModeResid: out = f - A u;
// kModeSpmv: out = A u (A may be rectangular: n rows, columns indexing u).
template <int V, int MODE, typename VT, typename XT>
__global__ void __launch_bounds__(256)
    k_bt_rowop(int32_t n, int W, int lgL, const int32_t *__restrict__ row,
               const int32_t *__restrict__ col, const VT *__restrict__ val,
               const XT *__restrict__ d, const XT *__restrict__ f, const XT *__restrict__ u,
               XT *__restrict__ out) {
  const int L = 1 << lgL;
  const int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  const int64_t gi = t >> lgL;
  const int g = threadIdx.x & (L - 1);
  const bool valid = gi < n;
  const int32_t i = valid ? static_cast<int32_t>(gi) : 0;
  int32_t j0 = 0;
  int len = 0;
  if (valid) {
    j0 = row[i];
    len = row[i + 1] - j0;
  }
  // The row's own f, u and d do not depend on the row sum: load them first.
  const int64_t o = static_cast<int64_t>(i) * W + static_cast<int64_t>(g) * V;
  Cols<XT, V> fv;
  if (MODE != kModeSpmv) fv = ldc<XT, V>(f + o);
  Cols<XT, V> uv;
  XT di = XT(1);
  if (MODE == kModeRelax) {
    uv = ldc<XT, V>(u + o);
    di = d[i];
  }
  XT acc[V];
  bt_row_sum<V, VT, XT>(col, val, u, W, L, g, j0, len, acc);
  if (!valid) return;
  Cols<XT, V> res;
  if (MODE == kModeRelax) {
    if (std::is_same<XT, float>::value) {
      // The FP32 cycle multiplies by one reciprocal per row (within an ulp
      // of dividing; the cycle is an inexact preconditioner either way).
      const XT rdi = XT(1) / di;
#pragma unroll
      for (int v = 0; v < V; ++v) res.v[v] = ((-acc[v] + fv.v[v]) * rdi) + uv.v[v];
    } else {
#pragma unroll
      for (int v = 0; v < V; ++v) res.v[v] = ((-acc[v] + fv.v[v]) / di) + uv.v[v];
    }
  } else if (MODE == kModeResid) {
#pragma unroll
    for (int v = 0; v < V; ++v) res.v[v] = fv.v[v] - acc[v];
  } else {
#pragma unroll
    for (int v = 0; v < V; ++v) res.v[v] = acc[v];
  }
  stc<XT, V>(out + o, res);
}

// First sweep from u = 0: f ./ d.
template <typename XT>
__global__ void k_bt_relax_zero(int64_t total, int lgW, const XT *__restrict__ d,
                                const XT *__restrict__ f, XT *__restrict__ out) {
  for (int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; e < total;
       e += static_cast<int64_t>(gridDim.x) * blockDim.x)
    out[e] = f[e] / d[e >> lgW];
}

template <int V, typename XT>
__global__ void k_bt_restrict(int32_t nc, int W, int lgL, const int32_t *__restrict__ rptr,
                              const int32_t *__restrict__ ridx, const XT *__restrict__ p,
                              const XT *__restrict__ x, XT *__restrict__ y) {
  const int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  const int64_t I = t >> lgL;
  if (I >= nc) return;
  const int64_t cofs = static_cast<int64_t>(threadIdx.x & ((1 << lgL) - 1)) * V;
  XT acc[V];
#pragma unroll
  for (int v = 0; v < V; ++v) acc[v] = XT(0);
  for (int32_t k = rptr[I]; k < rptr[I + 1]; ++k) {
    const int32_t i = ridx[k];
    const XT pi = p[i];
    const Cols<XT, V> xv = ldc<XT, V>(x + static_cast<int64_t>(i) * W + cofs);
#pragma unroll
    for (int v = 0; v < V; ++v) acc[v] = fma(pi, xv.v[v], acc[v]);
  }
  Cols<XT, V> out;
#pragma unroll
  for (int v = 0; v < V; ++v) out.v[v] = acc[v];
  stc<XT, V>(y + I * W + cofs, out);
}

template <int V, typename XT>
__global__ void k_bt_prolong(int32_t n, int W, int lgL, const int32_t *__restrict__ agg,
                             const XT *__restrict__ p, const XT *__restrict__ xc,
                             XT *__restrict__ xf) {
  const int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  const int64_t i = t >> lgL;
  if (i >= n) return;
  const int64_t cofs = static_cast<int64_t>(threadIdx.x & ((1 << lgL) - 1)) * V;
  const XT pi = p[i];
  const Cols<XT, V> c = ldc<XT, V>(xc + static_cast<int64_t>(agg[i]) * W + cofs);
  Cols<XT, V> fv = ldc<XT, V>(xf + i * W + cofs);
#pragma unroll
  for (int v = 0; v < V; ++v) fv.v[v] = fma(pi, c.v[v], fv.v[v]);
  stc<XT, V>(xf + i * W + cofs, fv);
}

// Tiled transposes between column-major and interleaved storage: a block
// moves 32 rows x W columns through shared memory so that both the column
// reads and the interleaved writes are contiguous.
__global__ void k_bt_pack(int32_t n, int m, const double *__restrict__ src, int64_t ld,
                          double *__restrict__ dst, int W, int lgW) {
  __shared__ double tile[32][kBatchMax + 1];
  const int64_t i0 = static_cast<int64_t>(blockIdx.x) * 32;
  const int r = threadIdx.x & 31;
  for (int c = threadIdx.x >> 5; c < W; c += blockDim.x >> 5) {
    const int64_t i = i0 + r;
    tile[r][c] = (c < m && i < n) ? src[c * ld + i] : 0.0;
  }
  __syncthreads();
  for (int e = threadIdx.x; e < 32 * W; e += blockDim.x) {
    const int rr = e >> lgW, c = e & (W - 1);
    const int64_t i = i0 + rr;
    if (i < n) dst[i * W + c] = tile[rr][c];
  }
}

__global__ void k_bt_unpack(int32_t n, int m, const double *__restrict__ src, int W, int lgW,
                            double *__restrict__ dst, int64_t ld) {
  __shared__ double tile[32][kBatchMax + 1];
  const int64_t i0 = static_cast<int64_t>(blockIdx.x) * 32;
  for (int e = threadIdx.x; e < 32 * W; e += blockDim.x) {
    const int rr = e >> lgW, c = e & (W - 1);
    const int64_t i = i0 + rr;
    tile[rr][c] = i < n ? src[i * W + c] : 0.0;
  }
  __syncthreads();
  const int r = threadIdx.x & 31;
  for (int c = threadIdx.x >> 5; c < m; c += blockDim.x >> 5) {
    const int64_t i = i0 + r;
    if (i < n) dst[c * ld + i] = tile[r][c];
  }
}

// ---- per-column deterministic reductions -----------------------------------

// Block sums per column of NV quantities held as acc[k][v] for columns
// g V + v, where lanes g, g + L, g + 2L, ... of a warp own the same
// columns.  Written to partials[(block * 4 + k) * W + c] in a fixed order.
template <int NV, int V>
__device__ __forceinline__ void bt_block_partials(double (&acc)[NV][V], int W, int L,
                                                  double *partials) {
  __shared__ double sh[kRedWarps][NV][kBatchMax];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int o = 16; o >= L; o >>= 1) {
#pragma unroll
    for (int k = 0; k < NV; ++k)
#pragma unroll
      for (int v = 0; v < V; ++v) acc[k][v] += __shfl_down_sync(kFull, acc[k][v], o);
  }
  if (lane < L) {
#pragma unroll
    for (int k = 0; k < NV; ++k)
#pragma unroll
      for (int v = 0; v < V; ++v) sh[wid][k][lane * V + v] = acc[k][v];
  }
  __syncthreads();
  for (int e = threadIdx.x; e < NV * W; e += blockDim.x) {
    const int k = e / W, c = e % W;
    double s = 0.0;
    for (int w = 0; w < kRedWarps; ++w) s += sh[w][k][c];
    partials[(static_cast<int64_t>(blockIdx.x) * 4 + k) * W + c] = s;
  }
}

// Fixed-order sum over the kRedBlocks block partials of quantity k, column c
// (one block of kRedT threads).
__device__ __forceinline__ double bt_reduce_col(const double *partials, int k, int W, int c) {
  __shared__ double sh[kRedT];
  double s = 0.0;
  for (int b = threadIdx.x; b < kRedBlocks; b += blockDim.x)
    s += partials[(static_cast<int64_t>(b) * 4 + k) * W + c];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  const double r = sh[0];
  __syncthreads();
  return r;
}

// Per-column a.b and c.d over an interleaved block (c, d may be null).
__global__ void __launch_bounds__(kRedT)
    k_bt_dots(int64_t total, int W, const double *__restrict__ a, const double *__restrict__ b,
              const double *__restrict__ c, const double *__restrict__ d, double *partials) {
  double acc[2][1] = {{0.0}, {0.0}};
  for (int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; e < total;
       e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    acc[0][0] = fma(a[e], b[e], acc[0][0]);
    if (c) acc[1][0] = fma(c[e], d[e], acc[1][0]);
  }
  bt_block_partials<2, 1>(acc, W, W, partials);
}

__global__ void k_bt_col_norms(const double *partials, int W, double *out) {
  const double s = bt_reduce_col(partials, 0, W, blockIdx.x);
  if (threadIdx.x == 0) out[blockIdx.x] = sqrt(s);
}

__global__ void k_bt_init(const double *partials, int W, double rtol, int itnlim,
                          double *scal) {
  const int c = blockIdx.x;
  const double rr = bt_reduce_col(partials, 0, W, c);
  const double bb = bt_reduce_col(partials, 1, W, c);
  if (threadIdx.x != 0) return;
  double *S = scal + c * kBtStride;
  for (int k = 0; k < kBtStride; ++k) S[k] = 0.0;
  const double delta0 = sqrt(rr), bnorm = sqrt(bb);
  S[kDelta0] = delta0;
  S[kBnorm] = bnorm;
  S[kNorm] = delta0;
  S[kTarget] = rtol * delta0;
  S[kItnlim] = itnlim;
  // Already converged (the reference exits here, FCG.cu:459-462): never
  // iterates.
  S[kBtAct] = delta0 <= DBL_EPSILON * bnorm ? 0.0 : 1.0;
}

__global__ void k_bt_any_active(const double *scal, int W, int *flags) {
  const int c = threadIdx.x;
  const bool a = c < W && scal[c * kBtStride + kBtAct] != 0.0;
  const bool any = __any_sync(kFull, a);
  if (c == 0) flags[0] = any ? 1 : 0;
}

// w = A v fused with the per-column alpha = r.v, beta = w.v, gamma = q.v.
template <int V>
__global__ void __launch_bounds__(kRedT)
    k_bt_fcg_spmv_dots(int32_t n, int W, int lgL, const int32_t *__restrict__ row,
                       const int32_t *__restrict__ col, const double *__restrict__ val,
                       const double *__restrict__ v, double *__restrict__ w,
                       const double *__restrict__ r, const double *__restrict__ q,
                       double *partials) {
  const int L = 1 << lgL;
  const int g = threadIdx.x & (L - 1);
  const int64_t groups = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> lgL;
  const int64_t g0 = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> lgL;
  const int64_t rounds = (n + groups - 1) / groups;
  double acc[3][V];
#pragma unroll
  for (int k = 0; k < 3; ++k)
#pragma unroll
    for (int u = 0; u < V; ++u) acc[k][u] = 0.0;
  for (int64_t rd = 0; rd < rounds; ++rd) {
    const int64_t gi = g0 + rd * groups;
    const bool valid = gi < n;
    const int32_t i = valid ? static_cast<int32_t>(gi) : 0;
    int32_t j0 = 0;
    int len = 0;
    if (valid) {
      j0 = row[i];
      len = row[i + 1] - j0;
    }
    double T[V];
    bt_row_sum<V, double, double>(col, val, v, W, L, g, j0, len, T);
    if (valid) {
      const int64_t o = static_cast<int64_t>(i) * W + static_cast<int64_t>(g) * V;
      Cols<double, V> tw;
#pragma unroll
      for (int u = 0; u < V; ++u) tw.v[u] = T[u];
      stc<double, V>(w + o, tw);
      const Cols<double, V> vv = ldc<double, V>(v + o);
      const Cols<double, V> rv = ldc<double, V>(r + o);
#pragma unroll
      for (int u = 0; u < V; ++u) {
        acc[0][u] = fma(rv.v[u], vv.v[u], acc[0][u]);
        acc[1][u] = fma(T[u], vv.v[u], acc[1][u]);
      }
      if (q) {
        const Cols<double, V> qv = ldc<double, V>(q + o);
#pragma unroll
        for (int u = 0; u < V; ++u) acc[2][u] = fma(qv.v[u], vv.v[u], acc[2][u]);
      }
    }
  }
  bt_block_partials<3, V>(acc, W, L, partials);
}

// Per-column FCG scalar recurrences (FCG.cu:475-478, 531-534), the same
// arithmetic as the single-vector k_fcg_scalars; columns that stopped
// iterating are left untouched.
__global__ void k_bt_fcg_scalars(const double *partials, double *scal, int W, int first) {
  const int c = blockIdx.x;
  const double alpha = bt_reduce_col(partials, 0, W, c);
  const double beta = bt_reduce_col(partials, 1, W, c);
  const double gamma = bt_reduce_col(partials, 2, W, c);
  if (threadIdx.x != 0) return;
  double *S = scal + c * kBtStride;
  if (S[kBtAct] == 0.0) return;
  S[kAlpha] = alpha;
  S[kBeta] = beta;
  S[kGamma] = gamma;
  if (first) {
    S[kDelta] = beta;
    S[kTheta] = alpha / beta;
    if (!(beta > 0.0)) S[kIndef] = 1.0;
  } else {
    const double delta = S[kDelta];
    const double theta = gamma / delta;
    const double nd = beta - (gamma * gamma) / delta;
    if (nd > 0.0) {
      S[kTheta] = theta;
      S[kDelta] = nd;
      S[kTheta2] = alpha / nd;
    } else if (alpha == 0.0 && gamma == 0.0) {
      S[kTheta] = 0.0;  // exact previous step: no-op update
      S[kTheta2] = 0.0;
    } else {
      S[kTheta] = theta;
      S[kDelta] = nd;
      S[kTheta2] = alpha / nd;
      S[kIndef] = 1.0;
    }
  }
}

// The fused FCG update of k_fcg_update per column; stopped columns keep x and
// r.  The grid stride is a multiple of W, so a thread always serves the same
// column.
__global__ void __launch_bounds__(kRedT)
    k_bt_fcg_update(int64_t total, int W, int first, const double *__restrict__ z,
                    double *__restrict__ zp, const double *__restrict__ az,
                    double *__restrict__ azp, double *__restrict__ x, double *__restrict__ r,
                    const double *__restrict__ scal, double *partials) {
  double acc[1][1] = {{0.0}};
  const int64_t t0 = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  const double *S = scal + (t0 & (W - 1)) * kBtStride;
  if (S[kBtAct] != 0.0) {
    const double theta = S[kTheta];
    const double theta2 = first ? theta : S[kTheta2];
    for (int64_t e = t0; e < total; e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
      double zi = z[e], ai = az[e];
      if (!first) {
        zi = fma(-theta, zp[e], zi);
        ai = fma(-theta, azp[e], ai);
      }
      zp[e] = zi;
      azp[e] = ai;
      x[e] = fma(theta2, zi, x[e]);
      const double ri = fma(-theta2, ai, r[e]);
      r[e] = ri;
      acc[0][0] = fma(ri, ri, acc[0][0]);
    }
  }
  bt_block_partials<1, 1>(acc, W, W, partials);
}

// kNorm = sqrt(sum) for active columns (key = kBtAct) or for columns that
// replaced their residual (key = kReplace).
__global__ void k_bt_norm_final(const double *partials, double *scal, int W, int key) {
  const int c = blockIdx.x;
  const double s = bt_reduce_col(partials, 0, W, c);
  if (threadIdx.x == 0 && scal[c * kBtStride + key] != 0.0) scal[c * kBtStride + kNorm] = sqrt(s);
}

// Residual replacement decision per column (k_replace_flag); flags[1] says
// whether any column replaces.
__global__ void k_bt_replace_flag(double *scal, int W, int every, int *flags) {
  const int c = threadIdx.x;
  bool due = false;
  if (c < W) {
    double *S = scal + c * kBtStride;
    const int i = static_cast<int>(S[kIter]) + 1;
    due = S[kBtAct] != 0.0 &&
          ((every > 0 && i % every == 0) || S[kNorm] <= S[kTarget]);
    S[kReplace] = due ? 1.0 : 0.0;
  }
  const bool any = __any_sync(kFull, due);
  if (c == 0) flags[1] = any ? 1 : 0;
}

// r = b - A x in FP64 for the columns that replace their residual, with the
// partial sums of r.r.
template <int V>
__global__ void __launch_bounds__(kRedT)
    k_bt_true_residual(int32_t n, int W, int lgL, const int32_t *__restrict__ row,
                       const int32_t *__restrict__ col, const double *__restrict__ val,
                       const double *__restrict__ b, const double *__restrict__ x,
                       double *__restrict__ r, const double *__restrict__ scal,
                       const int *flags, double *partials) {
  if (flags[1] == 0) return;  // uniform over the grid
  const int L = 1 << lgL;
  const int g = threadIdx.x & (L - 1);
  const int64_t groups = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> lgL;
  const int64_t g0 = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> lgL;
  const int64_t rounds = (n + groups - 1) / groups;
  bool rep[V];
#pragma unroll
  for (int u = 0; u < V; ++u) rep[u] = scal[(g * V + u) * kBtStride + kReplace] != 0.0;
  double acc[1][V];
#pragma unroll
  for (int u = 0; u < V; ++u) acc[0][u] = 0.0;
  for (int64_t rd = 0; rd < rounds; ++rd) {
    const int64_t gi = g0 + rd * groups;
    const bool valid = gi < n;
    const int32_t i = valid ? static_cast<int32_t>(gi) : 0;
    int32_t j0 = 0;
    int len = 0;
    if (valid) {
      j0 = row[i];
      len = row[i + 1] - j0;
    }
    double T[V];
    bt_row_sum<V, double, double>(col, val, x, W, L, g, j0, len, T);
    if (valid) {
      const int64_t o = static_cast<int64_t>(i) * W + static_cast<int64_t>(g) * V;
#pragma unroll
      for (int u = 0; u < V; ++u)
        if (rep[u]) {
          const double ri = b[o + u] - T[u];
          r[o + u] = ri;
          acc[0][u] = fma(ri, ri, acc[0][u]);
        }
    }
  }
  bt_block_partials<1, V>(acc, W, L, partials);
}

// End of an iteration per column (k_fcg_continue): count it, stop the column
// when it converged, hit itnlim or broke down; the WHILE condition is "some
// column still iterating".
__global__ void k_bt_continue(double *scal, int W, int *flags, cudaGraphConditionalHandle cond,
                              int use_cond) {
  const int c = threadIdx.x;
  bool go = false;
  if (c < W) {
    double *S = scal + c * kBtStride;
    if (S[kBtAct] != 0.0) {
      const double iter = S[kIter] + 1.0;
      S[kIter] = iter;
      go = S[kNorm] > S[kTarget] && iter < S[kItnlim] && S[kIndef] == 0.0;
      if (!go) S[kBtAct] = 0.0;
    }
  }
  const bool any = __any_sync(kFull, go);
  if (c == 0) {
    flags[0] = any ? 1 : 0;
    if (use_cond) cudaGraphSetConditional(cond, any ? 1u : 0u);
  }
}

// ---- launch helpers -----------------------------------------------------------

inline int grid_of(int64_t threads, int block) {
  const int64_t b = (threads + block - 1) / block;
  return static_cast<int>(b < 1 ? 1 : b);
}

inline int stream_grid(int64_t total) {
  return static_cast<int>(std::min<int64_t>(grid_of(total, 256), 8 * kNumSM));
}

bcmg_status check_cfg(int W, BtCfg cfg, size_t xbytes) {
  if (W < 1 || W > kBatchMax || (W & (W - 1)))
    return set_error(BCMG_ERR_INTERNAL, "batch width %d is not a power of two <= %d", W,
                     kBatchMax);
  if (cfg.V < 1 || cfg.V > W || (cfg.V & (cfg.V - 1)) || cfg.V * xbytes > 16)
    return set_error(BCMG_ERR_INTERNAL, "bad columns per lane %d (W %d)", cfg.V, W);
  if (cfg.threads < 32 || cfg.threads > 256 || cfg.threads % 32)
    return set_error(BCMG_ERR_INTERNAL, "bad block size %d", cfg.threads);
  return BCMG_OK;
}

template <int MODE, typename VT, typename XT>
void launch_rowop_v(const MatView &A, int W, BtCfg cfg, const XT *d, const XT *f,
                    const XT *u, XT *out, cudaStream_t s) {
  const VT *val = static_cast<const VT *>(A.val);
  const int L = W / cfg.V, lgL = ilog2(L);
  const int blocks = grid_of(static_cast<int64_t>(A.n) * L, cfg.threads);
  switch (cfg.V) {
    case 1:
      launch(k_bt_rowop<1, MODE, VT, XT>, blocks, cfg.threads, 0, s, A.n, W, lgL, A.row,
             A.col, val, d, f, u, out);
      break;
    case 2:
      launch(k_bt_rowop<2, MODE, VT, XT>, blocks, cfg.threads, 0, s, A.n, W, lgL, A.row,
             A.col, val, d, f, u, out);
      break;
    default:
      if constexpr (sizeof(XT) <= 4)
        launch(k_bt_rowop<4, MODE, VT, XT>, blocks, cfg.threads, 0, s, A.n, W, lgL, A.row,
               A.col, val, d, f, u, out);
      break;
  }
}

template <int MODE, typename XT>
bcmg_status launch_rowop(const MatView &A, int W, BtCfg cfg, const XT *d, const XT *f,
                         const XT *u, XT *out, cudaStream_t s) {
  BCMG_TRY(check_cfg(W, cfg, sizeof(XT)));
  if constexpr (sizeof(XT) == 8) {
    if (A.vtype != kValF64) return set_error(BCMG_ERR_INTERNAL, "FP64 batch needs FP64 values");
    launch_rowop_v<MODE, double, double>(A, W, cfg, d, f, u, out, s);
  } else {
    switch (A.vtype) {
      case kValF32: launch_rowop_v<MODE, float, float>(A, W, cfg, d, f, u, out, s); break;
      case kValBF16: launch_rowop_v<MODE, __nv_bfloat16, float>(A, W, cfg, d, f, u, out, s); break;
      case kValF16: launch_rowop_v<MODE, __half, float>(A, W, cfg, d, f, u, out, s); break;
      default: return set_error(BCMG_ERR_INTERNAL, "FP32 batch needs low-precision values");
    }
  }
  BCMG_LAUNCH_CHECK();
  return BCMG_OK;
}

// Widest vector access for elementwise batch kernels.
template <typename XT>
int elem_v(int W) {
  const int v = 16 / static_cast<int>(sizeof(XT));
  return W < v ? W : v;
}

}  // namespace

template <typename XT>
bcmg_status bt_relax(const MatView &A, int W, BtCfg cfg, const XT *d, const XT *f, XT *u,
                     XT *u_tmp, int k, bool zero_start, cudaStream_t s) {
  const int32_t n = A.n;
  if (n <= 0) return BCMG_OK;
  const int64_t total = static_cast<int64_t>(n) * W;
  if (k <= 0) {
    if (zero_start) BCMG_TRY(fill_t<XT>(u, total, XT(0), s));
    return BCMG_OK;
  }
  XT *cur;
  int left = k;
  if (zero_start) {
    cur = (k % 2 == 1) ? u : u_tmp;
    launch(k_bt_relax_zero<XT>, stream_grid(total), 256, 0, s, total, ilog2(W), d, f, cur);
    --left;
  } else if (k % 2 == 1) {
    BCMG_CUDA(cudaMemcpyAsync(u_tmp, u, sizeof(XT) * total, cudaMemcpyDeviceToDevice, s));
    cur = u_tmp;
  } else {
    cur = u;
  }
  for (; left > 0; --left) {
    XT *dst = (cur == u) ? u_tmp : u;
    BCMG_TRY((launch_rowop<kModeRelax, XT>(A, W, cfg, d, f, cur, dst, s)));
    cur = dst;
  }
  BCMG_LAUNCH_CHECK();
  return BCMG_OK;
}

template <typename XT>
bcmg_status bt_residual(const MatView &A, int W, BtCfg cfg, const XT *f, const XT *u, XT *res,
                        cudaStream_t s) {
  if (A.n <= 0) return BCMG_OK;
  return launch_rowop<kModeResid, XT>(A, W, cfg, nullptr, f, u, res, s);
}

template <typename XT>
bcmg_status bt_spmm(const MatView &A, int W, BtCfg cfg, const XT *x, XT *y, cudaStream_t s) {
  if (A.n <= 0) return BCMG_OK;
  return launch_rowop<kModeSpmv, XT>(A, W, cfg, nullptr, nullptr, x, y, s);
}

template <typename XT>
bcmg_status bt_restrict(int32_t nc, const int32_t *rptr, const int32_t *ridx, const XT *p,
                        const XT *x, XT *y, int W, cudaStream_t s) {
  if (nc <= 0) return BCMG_OK;
  const int V = elem_v<XT>(W), L = W / V, lgL = ilog2(L);
  const int blocks = grid_of(static_cast<int64_t>(nc) * L, 256);
  switch (V) {
    case 1: launch(k_bt_restrict<1, XT>, blocks, 256, 0, s, nc, W, lgL, rptr, ridx, p, x, y); break;
    case 2: launch(k_bt_restrict<2, XT>, blocks, 256, 0, s, nc, W, lgL, rptr, ridx, p, x, y); break;
    default:
      if constexpr (sizeof(XT) <= 4)
        launch(k_bt_restrict<4, XT>, blocks, 256, 0, s, nc, W, lgL, rptr, ridx, p, x, y);
      break;
  }
  BCMG_LAUNCH_CHECK();
  return BCMG_OK;
}

template <typename XT>
bcmg_status bt_prolong(int32_t n, const int32_t *agg, const XT *p, const XT *xc, XT *xf, int W,
                       cudaStream_t s) {
  if (n <= 0) return BCMG_OK;
  const int V = elem_v<XT>(W), L = W / V, lgL = ilog2(L);
  const int blocks = grid_of(static_cast<int64_t>(n) * L, 256);
  switch (V) {
    case 1: launch(k_bt_prolong<1, XT>, blocks, 256, 0, s, n, W, lgL, agg, p, xc, xf); break;
    case 2: launch(k_bt_prolong<2, XT>, blocks, 256, 0, s, n, W, lgL, agg, p, xc, xf); break;
    default:
      if constexpr (sizeof(XT) <= 4)
        launch(k_bt_prolong<4, XT>, blocks, 256, 0, s, n, W, lgL, agg, p, xc, xf);
      break;
  }
  BCMG_LAUNCH_CHECK();
  return BCMG_OK;
}

bcmg_status bt_pack(int32_t n, int m, const double *src, int64_t ld, double *dst, int W,
                    cudaStream_t s) {
  if (n <= 0) return BCMG_OK;
  if (m < 0 || m > W || ld < n) return set_error(BCMG_ERR_INTERNAL, "bad pack shape");
  launch(k_bt_pack, ceil_div(n, 32), 256, 0, s, n, m, src, ld, dst, W, ilog2(W));
  BCMG_LAUNCH_CHECK();
  return BCMG_OK;
}

bcmg_status bt_unpack(int32_t n, int m, const double *src, int W, double *dst, int64_t ld,
                      cudaStream_t s) {
  if (n <= 0 || m <= 0) return BCMG_OK;
  if (m > W || ld < n) return set_error(BCMG_ERR_INTERNAL, "bad unpack shape");
  launch(k_bt_unpack, ceil_div(n, 32), 256, 0, s, n, m, src, W, ilog2(W), dst, ld);
  BCMG_LAUNCH_CHECK();
  return BCMG_OK;
}

bcmg_status bt_fcg_init(int32_t n, int W, const double *r, const double *b, double rtol,
                        int itnlim, double *partials, double *scal, int *flags,
                        cudaStream_t s) {
  const int64_t total = static_cast<int64_t>(n) * W;
  launch(k_bt_dots, kRedBlocks, kRedT, 0, s, total, W, r, r, b, b, partials);
  launch(k_bt_init, W, kRedT, 0, s, partials, W, rtol, itnlim, scal);
  launch(k_bt_any_active, 1, 32, 0, s, scal, W, flags);
  BCMG_LAUNCH_CHECK();
  return BCMG_OK;
}

bcmg_status bt_fcg_spmv_dots(const CsrView &A, int W, BtCfg cfg, const double *v, double *w,
                             const double *r, const double *q, double *partials,
                             cudaStream_t s) {
  BCMG_TRY(check_cfg(W, cfg, sizeof(double)));
  const int lgL = ilog2(W / cfg.V);
  if (cfg.V == 1)
    launch(k_bt_fcg_spmv_dots<1>, kRedBlocks, kRedT, 0, s, A.n, W, lgL, A.row, A.col, A.val,
           v, w, r, q, partials);
  else
    launch(k_bt_fcg_spmv_dots<2>, kRedBlocks, kRedT, 0, s, A.n, W, lgL, A.row, A.col, A.val,
           v, w, r, q, partials);
  BCMG_LAUNCH_CHECK();
  return BCMG_OK;
}

bcmg_status bt_fcg_scalars(const double *partials, double *scal, int W, bool first,
                           cudaStream_t s) {
  launch(k_bt_fcg_scalars, W, kRedT, 0, s, partials, scal, W, first ? 1 : 0);
  BCMG_LAUNCH_CHECK();
  return BCMG_OK;
}

bcmg_status bt_fcg_update(int32_t n, int W, bool first, const double *z, double *zp,
                          const double *az, double *azp, double *x, double *r,
                          double *partials, double *scal, cudaStream_t s) {
  const int64_t total = static_cast<int64_t>(n) * W;
  launch(k_bt_fcg_update, kRedBlocks, kRedT, 0, s, total, W, first ? 1 : 0, z, zp, az, azp, x,
         r, scal, partials);
  launch(k_bt_norm_final, W, kRedT, 0, s, partials, scal, W, static_cast<int>(kBtAct));
  BCMG_LAUNCH_CHECK();
  return BCMG_OK;
}

bcmg_status bt_fcg_replace(const CsrView &A, int W, BtCfg cfg, const double *b,
                           const double *x, double *r, double *partials, double *scal,
                           int *flags, int every, cudaStream_t s) {
  BCMG_TRY(check_cfg(W, cfg, sizeof(double)));
  launch(k_bt_replace_flag, 1, 32, 0, s, scal, W, every, flags);
  const int lgL = ilog2(W / cfg.V);
  if (cfg.V == 1)
    launch(k_bt_true_residual<1>, kRedBlocks, kRedT, 0, s, A.n, W, lgL, A.row, A.col, A.val,
           b, x, r, scal, flags, partials);
  else
    launch(k_bt_true_residual<2>, kRedBlocks, kRedT, 0, s, A.n, W, lgL, A.row, A.col, A.val,
           b, x, r, scal, flags, partials);
  launch(k_bt_norm_final, W, kRedT, 0, s, partials, scal, W, static_cast<int>(kReplace));
  BCMG_LAUNCH_CHECK();
  return BCMG_OK;
}

bcmg_status bt_fcg_continue(double *scal, int W, int *flags, cudaGraphConditionalHandle cond,
                            bool use_cond, cudaStream_t s) {
  launch(k_bt_continue, 1, 32, 0, s, scal, W, flags, cond, use_cond ? 1 : 0);
  BCMG_LAUNCH_CHECK();
  return BCMG_OK;
}

bcmg_status bt_col_norms(int32_t n, int W, const double *a, double *partials, double *out,
                         cudaStream_t s) {
  const int64_t total = static_cast<int64_t>(n) * W;
  launch(k_bt_dots, kRedBlocks, kRedT, 0, s, total, W, a, a, nullptr, nullptr, partials);
  launch(k_bt_col_norms, W, kRedT, 0, s, partials, W, out);
  BCMG_LAUNCH_CHECK();
  return BCMG_OK;
}

#define BCMG_BT_INSTANTIATE(XT)                                                               \
  template bcmg_status bt_relax<XT>(const MatView &, int, BtCfg, const XT *, const XT *, XT *, \
                                    XT *, int, bool, cudaStream_t);                            \
  template bcmg_status bt_residual<XT>(const MatView &, int, BtCfg, const XT *, const XT *,    \
                                       XT *, cudaStream_t);                                    \
  template bcmg_status bt_spmm<XT>(const MatView &, int, BtCfg, const XT *, XT *, cudaStream_t); \
  template bcmg_status bt_restrict<XT>(int32_t, const int32_t *, const int32_t *, const XT *,  \
                                       const XT *, XT *, int, cudaStream_t);                   \
  template bcmg_status bt_prolong<XT>(int32_t, const int32_t *, const XT *, const XT *, XT *,  \
                                      int, cudaStream_t);

BCMG_BT_INSTANTIATE(double)
BCMG_BT_INSTANTIATE(float)

}  // namespace bcmg
