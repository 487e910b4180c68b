// Sliced matrix format for the solve phase and its kernels.
//
// Rows are cut into slices of 32 (one warp, one thread per row).  A slice
// stores W slots of 32 values in slot-major order, so every slot of a slice
// is one contiguous 32-element segment and a slice is one contiguous block.
// Two slot kinds:
//   offset slice: the slice's rows share a set of W column offsets
//                 (col - row), e.g. a stencil; column indices are implicit
//                 (row + offset) and W offsets are stored per slice.  Runs of
//                 consecutive slices with identical offset lists read one
//                 copy (the run head's), which stays cache-resident;
//   column slice: W = longest row; explicit int32 columns per slot (SELL-32).
// Missing entries are stored as 0 (with an in-range column), which adds exact
// zeros to the row sums.  Values, columns and offsets are padded by kSlotPad
// slots so a batch of loads may run past a slice's last slot without a bounds
// test (those products are discarded).  Built on the device from the level's
// CSR after setup; CSR stays the setup / introspection format.
//
// Row passes (smoother sweep, residual, SpMV, FCG SpMV + dots) run as one
// warp-specialised pipeline per CTA: a producer warp streams each chunk of
// kPipeWarps consecutive slices (values, explicit columns, slice metadata and
// the row vectors the epilogue reads) into shared memory with bulk async
// copies (cp.async.bulk, the TMA engine) under full/empty mbarriers, while the
// kPipeWarps consumer warps compute the previous chunks.  A consumer warp
// issues all gathers of a batch of slots before its first FMA, so each warp
// keeps a full row's gathers in flight.  Every wait is bounded; a wait that
// runs out sets a device error word (sliced_wait_status) and the kernel
// returns without touching the stage.
#include <cooperative_groups.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <algorithm>
#include <climits>
#include <map>
#include <mutex>
#include <utility>
#include <vector>

#include "common.cuh"
#include "kernels.h"
#include "reduce.cuh"
#include "scan.cuh"

namespace bcmg {
namespace {

constexpr int kWarpsPerBlock = 8;    // build kernels: one warp per slice
constexpr int kMaxOffsetSlots = 64;  // wider unions fall back to column slices
constexpr int kPipeWarps = 8;        // consumer warps per CTA = slices per chunk
constexpr int kPipeStages = 2;  // more stages took L1 from the gathers and ran slower
constexpr int kPipeThreads = (kPipeWarps + 1) * 32;
constexpr int kSlotPad = 32;                       // >= the largest slot batch
constexpr size_t kMaxStageBytes = 108 * 1024;      // two stages fit in 227 KB
// A CTA leaves only after the copies it issued have landed: the producer's
// final drain waits at least this long, whatever bound the handle sets on the
// pipeline's other waits (S.wait_ns).
constexpr unsigned long long kDrainLimitNs = 2000000000ull;

// Set by a pipeline wait that ran out (a bulk copy that never landed).
__device__ int g_sliced_wait_error;

__device__ __forceinline__ double widen(double v) { return v; }
__device__ __forceinline__ float widen(float v) { return v; }
__device__ __forceinline__ float widen(__nv_bfloat16 v) { return __bfloat162float(v); }
__device__ __forceinline__ float widen(__half v) { return __half2float(v); }

template <typename VT>
__device__ __forceinline__ VT narrow(double v);
template <>
__device__ __forceinline__ double narrow<double>(double v) { return v; }
template <>
__device__ __forceinline__ float narrow<float>(double v) { return static_cast<float>(v); }
template <>
__device__ __forceinline__ __nv_bfloat16 narrow<__nv_bfloat16>(double v) {
  return __double2bfloat16(v);
}
template <>
__device__ __forceinline__ __half narrow<__half>(double v) { return __double2half(v); }

// ---- format build -----------------------------------------------------------

// Pass 1: per slice, the longest row and the size of the union of column
// offsets (merging the 32 sorted rows); chooses the slice kind and width.
// Also widens offrange[0..1] (min, max) to every offset of an offset slice.
__global__ void k_slice_shape(int32_t n, int32_t nslices, const int32_t *__restrict__ row,
                              const int32_t *__restrict__ col, int32_t *width,
                              int32_t *kind, int32_t *offrange) {
  const int lane = threadIdx.x & 31;
  const int32_t s = blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5);
  if (s >= nslices) return;
  const int32_t r = s * 32 + lane;
  int32_t b = 0, e = 0;
  if (r < n) {
    b = row[r];
    e = row[r + 1];
  }
  int len = e - b;
  int maxlen = len;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) maxlen = max(maxlen, __shfl_xor_sync(0xffffffffu, maxlen, o));
  // Merge the sorted offset lists; count distinct offsets up to the cap.
  int32_t pos = b;
  int distinct = 0;
  int32_t lo = 0, hi = 0;  // smallest and largest offset
  while (distinct <= kMaxOffsetSlots) {
    const int32_t cur = pos < e ? col[pos] - r : INT_MAX;
    int32_t m = cur;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = min(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (m == INT_MAX) break;
    if (distinct == 0) lo = m;
    hi = m;
    ++distinct;
    if (cur == m) ++pos;
  }
  if (lane == 0) {
    const bool offsets = distinct <= kMaxOffsetSlots && distinct <= maxlen + maxlen / 4 + 2;
    kind[s] = offsets ? 1 : 0;
    width[s] = offsets ? distinct : maxlen;
    if (offsets && distinct > 0) {
      atomicMin(offrange, lo);
      atomicMax(offrange + 1, hi);
    }
  }
}

// Format statistics from the scanned slot pointers: stats[0] = the most slots
// in one chunk of kPipeWarps slices, stats[1] = 1 if any slice is a column
// slice.
__global__ void k_slice_stats(int32_t nslices, const int32_t *__restrict__ sptr,
                              const int32_t *__restrict__ kind, int32_t *stats) {
  const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  const int32_t s0 = c * kPipeWarps;
  if (s0 >= nslices) return;
  const int32_t s1 = min(s0 + kPipeWarps, nslices);
  atomicMax(stats, sptr[s1] - sptr[s0]);
  for (int32_t s = s0; s < s1; ++s)
    if (!kind[s]) {
      atomicOr(stats + 1, 1);
      break;
    }
}

// Which narrower types hold every value exactly (bitwise round trip):
// bit 0 FP32, bit 1 BF16, bit 2 FP16; stats[2] starts at 7 and is and-ed.
__global__ void k_value_exact(int64_t nnz, const double *__restrict__ val, int32_t *stats) {
  int ok = 7;
  for (int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; e < nnz;
       e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const double v = val[e];
    if (static_cast<double>(static_cast<float>(v)) != v) ok &= ~1;
    if (static_cast<double>(__bfloat162float(__double2bfloat16(v))) != v) ok &= ~2;
    if (static_cast<double>(__half2float(__double2half(v))) != v) ok &= ~4;
  }
  ok = __reduce_and_sync(0xffffffffu, ok);
  if ((threadIdx.x & 31) == 0 && ok != 7) atomicAnd(stats + 2, ok);
}

// Pass 2: fill values (and columns or offsets).
template <typename VT>
__global__ void k_slice_fill(int32_t n, int32_t nslices, const int32_t *__restrict__ row,
                             const int32_t *__restrict__ col,
                             const double *__restrict__ val,
                             const int32_t *__restrict__ sptr,
                             const int32_t *__restrict__ width,
                             const int32_t *__restrict__ kind, VT *sval, int32_t *scol,
                             int32_t *soff) {
  const int lane = threadIdx.x & 31;
  const int32_t s = blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5);
  if (s >= nslices) return;
  const int32_t r = s * 32 + lane;
  const int32_t rr = r < n ? r : n - 1;
  int32_t b = 0, e = 0;
  if (r < n) {
    b = row[r];
    e = row[r + 1];
  }
  const int64_t base = static_cast<int64_t>(sptr[s]) * 32;
  const int W = width[s];
  if (kind[s]) {
    int32_t pos = b;
    for (int k = 0; k < W; ++k) {
      const int32_t cur = pos < e ? col[pos] - r : INT_MAX;
      int32_t m = cur;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) m = min(m, __shfl_xor_sync(0xffffffffu, m, o));
      double v = 0.0;
      if (cur == m) {
        v = val[pos];
        ++pos;
      }
      sval[base + static_cast<int64_t>(k) * 32 + lane] = narrow<VT>(v);
      if (lane == 0) soff[sptr[s] + k] = m;
    }
  } else {
    for (int k = 0; k < W; ++k) {
      const int32_t j = b + k;
      const bool have = j < e;
      sval[base + static_cast<int64_t>(k) * 32 + lane] = narrow<VT>(have ? val[j] : 0.0);
      if (scol) scol[base + static_cast<int64_t>(k) * 32 + lane] = have ? col[j] : rr;
    }
  }
}

// flag[s] = 1 when slice s starts a new run: it is a column slice, or its
// offset list differs from slice s-1's.
__global__ void k_slice_runs(int32_t nslices, const int32_t *__restrict__ sptr,
                             const int32_t *__restrict__ width,
                             const int32_t *__restrict__ kind,
                             const int32_t *__restrict__ soff, int32_t *flag) {
  const int lane = threadIdx.x & 31;
  const int32_t s = blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5);
  if (s >= nslices) return;
  bool same = s > 0 && kind[s] && kind[s - 1] && width[s] == width[s - 1];
  if (same) {
    const int32_t *a = soff + sptr[s], *b = soff + sptr[s - 1];
    bool eq = true;
    for (int k = lane; k < width[s]; k += 32) eq = eq && a[k] == b[k];
    same = __all_sync(0xffffffffu, eq);
  }
  if (lane == 0) flag[s] = same ? 0 : 1;
}

__global__ void k_slice_heads(int32_t nslices, const int32_t *__restrict__ flag,
                              const int32_t *__restrict__ rid, int32_t *head) {
  const int32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s < nslices && flag[s]) head[rid[s]] = s;
}

// meta.z: 0 column slice, 1 offset slice, 2 interior offset slice — every
// row r of the slice is below n and r + o stays in [0, n) for every offset o
// in offrange, which bounds every entry of soff (offsets of offset slices,
// zeros elsewhere), so its gathers need no clamping; 3 (k_slice_stencil) an
// interior slice whose offsets are the copy's stencil.
__global__ void k_slice_meta(int32_t n, int32_t nslices, const int32_t *__restrict__ sptr,
                             const int32_t *__restrict__ width,
                             const int32_t *__restrict__ kind,
                             const int32_t *__restrict__ flag,
                             const int32_t *__restrict__ rid,
                             const int32_t *__restrict__ head,
                             const int32_t *__restrict__ offrange, int4 *meta) {
  const int32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nslices) return;
  const int32_t h = head[rid[s] + flag[s] - 1];
  const int64_t r0 = static_cast<int64_t>(s) * 32, r1 = r0 + 31;
  const bool interior =
      kind[s] == 1 && r1 < n && r0 + offrange[0] >= 0 && r1 + offrange[1] < n;
  meta[s] = make_int4(sptr[s], width[s], interior ? 2 : kind[s], sptr[h]);
}

// The first interior slice exactly w slots wide (none: *first stays nslices).
__global__ void k_stencil_pick(int32_t nslices, const int4 *__restrict__ meta, int32_t w,
                               int32_t *first) {
  const int32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  bool hit = false;
  if (s < nslices) {
    const int4 m = meta[s];
    hit = m.z == 2 && m.y == w;
  }
  const unsigned lo = __reduce_min_sync(0xffffffffu, hit ? static_cast<unsigned>(s) : ~0u);
  if ((threadIdx.x & 31) == 0 && lo != ~0u) atomicMin(first, static_cast<int32_t>(lo));
}

// Marks interior slices whose offset list is the stencil soff[base .. base +
// w) (the list of one interior slice of width w) as kind 3.
__global__ void k_slice_stencil(int32_t nslices, const int32_t *__restrict__ soff,
                                int32_t base, int32_t w, int4 *meta) {
  const int32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nslices) return;
  int4 m = meta[s];
  if (m.z != 2 || m.y != w) return;
  for (int32_t i = 0; i < w; ++i)
    if (soff[m.w + i] != soff[base + i]) return;
  m.z = 3;
  meta[s] = m;
}

// ---- pipeline primitives (mbarrier + bulk async copy) ---------------------

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t *b, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(b)), "r"(count)
               : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t *b) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(b)) : "memory");
}
__device__ __forceinline__ void mbar_arrive_tx(uint64_t *b, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(b)),
               "r"(bytes)
               : "memory");
}
// One try_wait: the thread may sleep until the phase completes or about
// kSuspendHintNs pass (a waiting warp issues no instructions meanwhile).
constexpr uint32_t kSuspendHintNs = 1000000;
__device__ __forceinline__ bool mbar_test(uint64_t *b, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3; "
      "selp.u32 %0, 1, 0, p; }"
      : "=r"(ok)
      : "r"(smem_addr(b)), "r"(parity), "r"(kSuspendHintNs)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
// Waits (one thread) for the phase with the given parity; false after
// limit_ns.
__device__ __forceinline__ bool mbar_wait(uint64_t *b, uint32_t parity,
                                          unsigned long long limit_ns) {
  if (mbar_test(b, parity)) return true;
  const unsigned long long t0 = global_ns();
  while (!mbar_test(b, parity))
    if (global_ns() - t0 > limit_ns) return false;
  return true;
}
// The same for a whole converged warp, with one outcome for all its lanes:
// true once every lane has seen the phase complete, false when lane 0's
// clock passes limit_ns first.  (Lanes that decided differently would leave
// the full-warp shuffles of the row sums unmatched.)
__device__ __forceinline__ bool mbar_wait_warp(uint64_t *b, uint32_t parity,
                                               unsigned long long limit_ns) {
  bool seen = mbar_test(b, parity);
  if (__all_sync(0xffffffffu, seen)) return true;
  const unsigned long long t0 = global_ns();
  while (true) {
    seen = seen || mbar_test(b, parity);
    if (__all_sync(0xffffffffu, seen)) return true;
    const int late = (global_ns() - t0 > limit_ns) ? 1 : 0;
    if (__shfl_sync(0xffffffffu, late, 0)) return false;
  }
}
// Global -> shared bulk copy (16-byte aligned, size a multiple of 16).
__device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes,
                                          uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}

// Gathers issued as volatile loads so a batch is in flight before its first
// use (the index is computed outside, the address inside).
__device__ __forceinline__ float gather(const float *x, int32_t i) {
  float v;
  asm volatile(
      "{ .reg .s64 a; mul.wide.s32 a, %2, 4; add.s64 a, %1, a; ld.global.nc.f32 %0, [a]; }"
      : "=f"(v)
      : "l"(x), "r"(i));
  return v;
}
__device__ __forceinline__ double gather(const double *x, int32_t i) {
  double v;
  asm volatile(
      "{ .reg .s64 a; mul.wide.s32 a, %2, 8; add.s64 a, %1, a; ld.global.nc.f64 %0, [a]; }"
      : "=d"(v)
      : "l"(x), "r"(i));
  return v;
}

// Gathers of a row sum from the iterate in global memory: x[i], or x[r + o]
// relative to the row set by row() (one 64-bit multiply-add per gather).
template <typename XT>
struct GlobalGather {
  const XT *x;
  const XT *xr;
  __device__ void row(int32_t r) { xr = x + r; }
  __device__ XT operator()(int32_t i) const { return gather(x, i); }
  __device__ XT rel(int32_t o) const { return gather(xr, o); }
  // x[r + o] for an offset held in a kernel parameter: plain C, so the
  // offset stays a constant-bank operand of the address arithmetic.
  __device__ XT rel_param(int32_t o) const { return __ldg(xr + o); }
};

// One batch of KB slots of a slice row sum (see row_sum); Full: every slot
// of the batch is below the slice width, so no slot is tested.
template <typename VT, typename XT, int KB, bool Full, typename G>
__device__ __forceinline__ void row_batch(XT (&t)[4], const VT *v, const int32_t *cidx,
                                          const int32_t *off, int k, int W, int32_t r,
                                          int32_t hi, bool interior, const G &g) {
  const int lane = threadIdx.x & 31;
  XT xv[KB];
  if (cidx) {
#pragma unroll
    for (int q = 0; q < KB; ++q) xv[q] = g(min(max(cidx[(k + q) * 32], 0), hi));
  } else if (interior) {
    const int32_t offl = __ldg(off + k + lane);
#pragma unroll
    for (int q = 0; q < KB; ++q) xv[q] = g.rel(__shfl_sync(0xffffffffu, offl, q));
  } else {
    const int32_t offl = __ldg(off + k + lane);
#pragma unroll
    for (int q = 0; q < KB; ++q)
      xv[q] = g(min(max(r + __shfl_sync(0xffffffffu, offl, q), 0), hi));
  }
#pragma unroll
  for (int q = 0; q < KB; ++q)
    if (Full || k + q < W)
      t[q & 3] = fma(static_cast<XT>(widen(v[(k + q) * 32])), xv[q], t[q & 3]);
}

// Row sum t = sum_k val[k] * x[col_k] of one slice row, slots in batches of
// KB.  v: the slice's values at this lane (shared or global memory); cidx: the
// slice's explicit columns at this lane (column slices), else off: the
// slice's offsets (offset slices; interior: every r + o lies in [0, n), as
// every entry of the offset array does for an interior slice, so no clamp).
// Gathers past slot W-1 read inside the padding and their products are
// dropped.  The four partial sums by slot index within the batch mod 4 fix
// the summation order, which therefore depends on KB; the gather functor g
// (g(i), g.rel(o) = x[r + o]) decides where x lives.
template <typename VT, typename XT, int KB, typename G>
__device__ __forceinline__ XT row_sum(const VT *v, const int32_t *cidx, const int32_t *off,
                                      int W, int32_t r, int32_t hi, bool interior,
                                      const G &g) {
  XT t[4] = {XT(0), XT(0), XT(0), XT(0)};
  int k = 0;
  for (; k + KB <= W; k += KB)
    row_batch<VT, XT, KB, true>(t, v, cidx, off, k, W, r, hi, interior, g);
  if (k < W) row_batch<VT, XT, KB, false>(t, v, cidx, off, k, W, r, hi, interior, g);
  return (t[0] + t[1]) + (t[2] + t[3]);
}

// row_sum of a stencil slice (meta.z == 3, width W = S.sten_w <= 2 KB): the
// offsets are kernel parameters, so no offset is loaded or shuffled; the
// batches and the summation order are row_sum's.  Offsets past W are zero,
// so the padding gathers stay in the row.
template <typename VT, typename XT, int KB, typename G>
__device__ __forceinline__ XT stencil_row_sum(const VT *v, const SlicedView &S, const G &g) {
  const int W = S.sten_w;
  XT t[4] = {XT(0), XT(0), XT(0), XT(0)};
  {
    XT xv[KB];
#pragma unroll
    for (int q = 0; q < KB; ++q) xv[q] = g.rel_param(S.sten_off[q]);
    if (W >= KB) {
#pragma unroll
      for (int q = 0; q < KB; ++q)
        t[q & 3] = fma(static_cast<XT>(widen(v[q * 32])), xv[q], t[q & 3]);
    } else {
#pragma unroll
      for (int q = 0; q < KB; ++q)
        if (q < W) t[q & 3] = fma(static_cast<XT>(widen(v[q * 32])), xv[q], t[q & 3]);
    }
  }
  if constexpr (KB < kStencilMax) {
    constexpr int K2 = kStencilMax - KB < KB ? kStencilMax - KB : KB;
    if (W > KB) {
      XT xv[K2];
#pragma unroll
      for (int q = 0; q < K2; ++q) xv[q] = g.rel_param(S.sten_off[KB + q]);
#pragma unroll
      for (int q = 0; q < K2; ++q)
        if (KB + q < W) t[q & 3] = fma(static_cast<XT>(widen(v[(KB + q) * 32])), xv[q], t[q & 3]);
    }
  }
  return (t[0] + t[1]) + (t[2] + t[3]);
}

// ---- epilogues ---------------------------------------------------------------
// NV row vectors are staged per chunk (rows()[i] in global memory); apply()
// consumes the row sum T of row r with those NV values.

template <typename XT>
struct EpiRelax {  // out = ((-T + f) / d) + u
  static constexpr int NV = 3;
  __device__ bool active() const { return true; }
  const XT *f, *d, *u;
  XT *out;
  __device__ const XT *row_vec(int i) const { return i == 0 ? f : (i == 1 ? d : u); }
  __device__ void apply(int32_t r, XT T, const XT *rv) { out[r] = ((-T + rv[0]) / rv[1]) + rv[2]; }
  __device__ void finish(int, int) {}
};

// EpiRelax on FP32 vectors whose result is written widened to FP64 (the last
// sweep of the mixed cycle, which hands its result to FP64 vectors).
struct EpiRelaxWiden {  // out = double(((-T + f) / d) + u)
  static constexpr int NV = 3;
  __device__ bool active() const { return true; }
  const float *f, *d, *u;
  double *out;
  __device__ const float *row_vec(int i) const { return i == 0 ? f : (i == 1 ? d : u); }
  __device__ void apply(int32_t r, float T, const float *rv) {
    out[r] = static_cast<double>(((-T + rv[0]) / rv[1]) + rv[2]);
  }
  __device__ void finish(int, int) {}
};

template <typename XT>
struct EpiResidual {  // out = f - T
  static constexpr int NV = 1;
  __device__ bool active() const { return true; }
  const XT *f;
  XT *out;
  __device__ const XT *row_vec(int) const { return f; }
  __device__ void apply(int32_t r, XT T, const XT *rv) { out[r] = rv[0] - T; }
  __device__ void finish(int, int) {}
};

template <typename XT>
struct EpiSpmvT {  // out = T
  static constexpr int NV = 0;
  __device__ bool active() const { return true; }
  XT *out;
  __device__ const XT *row_vec(int) const { return nullptr; }
  __device__ void apply(int32_t r, XT T, const XT *) { out[r] = T; }
  __device__ void finish(int, int) {}
};
using EpiSpmv = EpiSpmvT<double>;

// FCG: w = T with alpha = r.v, beta = w.v, gamma = q.v (v is the gathered
// vector); per-CTA partial sums in warp order, written to partials[4 b + k].
struct EpiFcgDots {
  static constexpr int NV = 3;
  __device__ bool active() const { return true; }
  const double *v, *r, *q;  // q == nullptr: no gamma
  double *w, *partials;
  double acc[3];
  __device__ const double *row_vec(int i) const { return i == 0 ? v : (i == 1 ? r : (q ? q : v)); }
  __device__ void apply(int32_t row, double T, const double *rv) {
    w[row] = T;
    acc[0] = fma(rv[1], rv[0], acc[0]);
    acc[1] = fma(T, rv[0], acc[1]);
    if (q) acc[2] = fma(rv[2], rv[0], acc[2]);
  }
  __device__ void finish(int wid, int lane) {
    __shared__ double red[kPipeWarps][3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      double a = acc[k];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) a += __shfl_down_sync(0xffffffffu, a, o);
      if (lane == 0) red[wid][k] = a;
    }
    // consumer warps only (the producer warp has left)
    asm volatile("bar.sync 1, %0;" ::"n"(kPipeWarps * 32) : "memory");
    if (wid == 0 && lane < 3) {
      double s = 0.0;
      for (int w2 = 0; w2 < kPipeWarps; ++w2) s += red[w2][lane];
      partials[blockIdx.x * 4 + lane] = s;
      for (int b = blockIdx.x + gridDim.x; b < kRedBlocks; b += gridDim.x)
        partials[b * 4 + lane] = 0.0;
    }
  }
};

// Residual replacement (mixed precision): r = b - A x with per-CTA partial
// sums of ||r||^2 (as EpiFcgDots, partial 0), only when the device flag
// scal[kReplace] is set; otherwise every CTA returns at once.
struct EpiReplace {
  static constexpr int NV = 1;
  const double *b;
  double *r, *partials;
  const double *scal;
  double acc[1];
  __device__ bool active() const { return scal[kReplace] != 0.0; }
  __device__ const double *row_vec(int) const { return b; }
  __device__ void apply(int32_t row, double T, const double *rv) {
    const double ri = rv[0] - T;
    r[row] = ri;
    acc[0] = fma(ri, ri, acc[0]);
  }
  __device__ void finish(int wid, int lane) {
    __shared__ double red[kPipeWarps];
    double a = acc[0];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) a += __shfl_down_sync(0xffffffffu, a, o);
    if (lane == 0) red[wid] = a;
    asm volatile("bar.sync 1, %0;" ::"n"(kPipeWarps * 32) : "memory");
    if (wid == 0 && lane == 0) {
      double t = 0.0;
      for (int w2 = 0; w2 < kPipeWarps; ++w2) t += red[w2];
      partials[blockIdx.x * 4] = t;
      for (int b2 = blockIdx.x + gridDim.x; b2 < kRedBlocks; b2 += gridDim.x)
        partials[b2 * 4] = 0.0;
    }
  }
};

// Shared-memory layout of one stage, identical on host and device.
struct StageLayout {
  uint32_t vals, cols, meta, rows, bytes;
  __host__ __device__ StageLayout(int cap_slots, int vbytes, int xbytes, bool cols_staged,
                                  int nv) {
    const uint32_t slots = static_cast<uint32_t>(cap_slots + kSlotPad);
    vals = 0;
    cols = vals + slots * 32u * vbytes;
    meta = cols + (cols_staged ? slots * 32u * 4u : 0u);
    rows = meta + kPipeWarps * 16u;
    bytes = rows + static_cast<uint32_t>(nv) * kPipeWarps * 32u * xbytes;
    bytes = (bytes + 127u) & ~127u;
  }
};

struct __align__(16) StageCtl {
  int32_t slot0, staged, rows_staged, pad;
};

// Resident CTAs per SM the register budget is sized for: FP64 vectors three
// (24 consumer warps, with at most 14 gathers per batch), FP32 vectors four
// (more would spill), FP32 batches of 27 or more three (four spilled and ran
// 7% slower on a 27-point level).
constexpr int kWideMinBlocks = 3;
template <typename XT, int KB>
constexpr int pipe_min_blocks() {
  return sizeof(XT) == 8 ? 3 : (KB >= 27 ? kWideMinBlocks : 4);
}

template <typename VT, typename XT, typename Epi, int KB>
__global__ void __launch_bounds__(kPipeThreads, pipe_min_blocks<XT, KB>())
    k_sl_pipe(SlicedView S, const VT *__restrict__ val, const XT *__restrict__ x, Epi epi,
              int cap_slots, int cols_staged) {
  pdl_wait();
  pdl_trigger();
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ __align__(8) uint64_t full[kPipeStages], empty[kPipeStages];
  __shared__ StageCtl ctl[kPipeStages];
  constexpr int NVS = Epi::NV > 0 ? Epi::NV : 1;
  if (!epi.active()) return;  // uniform: a device flag read by every thread
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int32_t nchunks = (S.nslices + kPipeWarps - 1) / kPipeWarps;
  const StageLayout L(cap_slots, sizeof(VT), sizeof(XT), cols_staged != 0, Epi::NV);
  if (threadIdx.x == 0) {
    for (int i = 0; i < kPipeStages; ++i) {
      mbar_init(&full[i], 1);
      mbar_init(&empty[i], kPipeWarps);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();

  if (wid == kPipeWarps) {  // producer
    if (lane != 0) return;
    uint32_t armed = 0;  // stages whose last phase carries a copy
    // Row vectors are staged only from 16-byte aligned bases.
    bool rows_aligned = Epi::NV > 0;
    for (int i = 0; i < Epi::NV; ++i)
      rows_aligned = rows_aligned && (reinterpret_cast<uintptr_t>(epi.row_vec(i)) & 15u) == 0;
    int32_t c = blockIdx.x;
    int32_t p0 = c < nchunks ? __ldg(S.sptr + c * kPipeWarps) : 0;
    int32_t p1 = c < nchunks ? __ldg(S.sptr + min((c + 1) * kPipeWarps, S.nslices)) : 0;
    int j = 0;
    for (; c < nchunks; ++j, c += gridDim.x) {
      const int32_t cn = c + gridDim.x;  // next chunk's bounds, loaded ahead
      const int32_t q0 = cn < nchunks ? __ldg(S.sptr + cn * kPipeWarps) : 0;
      const int32_t q1 = cn < nchunks ? __ldg(S.sptr + min((cn + 1) * kPipeWarps, S.nslices)) : 0;
      const int st = j % kPipeStages;
      if (j >= kPipeStages &&
          !mbar_wait(&empty[st], static_cast<uint32_t>(((j / kPipeStages) - 1) & 1),
                     S.wait_ns)) {
        atomicExch(&g_sliced_wait_error, 1);
        break;
      }
      const int32_t s0 = c * kPipeWarps, s1 = min(s0 + kPipeWarps, S.nslices);
      const int32_t r0 = s0 * 32, r1 = min(s1 * 32, S.n);
      const uint32_t rbytes = static_cast<uint32_t>(r1 - r0) * sizeof(XT);
      const bool rows_ok = rows_aligned && (rbytes % 16u) == 0;
      const bool fits = p1 - p0 <= cap_slots;
      ctl[st].slot0 = p0;
      ctl[st].staged = fits;
      ctl[st].rows_staged = rows_ok;
      unsigned char *base = smem + static_cast<size_t>(st) * L.bytes;
      if (fits) {
        const uint32_t nsl = static_cast<uint32_t>(p1 - p0) * 32u;
        const uint32_t vb = nsl * sizeof(VT);
        const uint32_t cb = cols_staged ? nsl * 4u : 0u;
        const uint32_t mb = static_cast<uint32_t>(s1 - s0) * 16u;
        mbar_arrive_tx(&full[st], vb + cb + mb + (rows_ok ? Epi::NV * rbytes : 0u));
        if (vb) bulk_load(base + L.vals, val + static_cast<int64_t>(p0) * 32, vb, &full[st]);
        if (cb) bulk_load(base + L.cols, S.scol + static_cast<int64_t>(p0) * 32, cb, &full[st]);
        bulk_load(base + L.meta, S.meta + s0, mb, &full[st]);
        if (rows_ok)
          for (int i = 0; i < Epi::NV; ++i)
            bulk_load(base + L.rows + i * kPipeWarps * 32 * sizeof(XT), epi.row_vec(i) + r0,
                      rbytes, &full[st]);
        armed |= 1u << st;
      } else {
        armed &= ~(1u << st);
        mbar_arrive(&full[st]);
      }
      p0 = q0;
      p1 = q1;
    }
    // Copies still in flight complete before the producer leaves.
    for (int k = 0; k < kPipeStages && k < j; ++k) {
      const int jj = j - 1 - k;
      const int st = jj % kPipeStages;
      if ((armed >> st) & 1u) {
        if (!mbar_wait(&full[st], static_cast<uint32_t>((jj / kPipeStages) & 1),
                       S.wait_ns > kDrainLimitNs ? S.wait_ns : kDrainLimitNs))
          atomicExch(&g_sliced_wait_error, 1);
      }
    }
    return;
  }

  // consumers
  const int32_t hi = S.n - 1;
  int32_t c = blockIdx.x;
  for (int j = 0; c < nchunks; ++j, c += gridDim.x) {
    const int st = j % kPipeStages;
    if (!mbar_wait_warp(&full[st], static_cast<uint32_t>((j / kPipeStages) & 1),
                        S.wait_ns)) {
      if (lane == 0) atomicExch(&g_sliced_wait_error, 1);
      break;
    }
    const StageCtl cl = ctl[st];
    const unsigned char *base = smem + static_cast<size_t>(st) * L.bytes;
    const int32_t s = c * kPipeWarps + wid;
    if (s < S.nslices) {
      const int32_t r = s * 32 + lane;
      GlobalGather<XT> g{x, x};
      g.row(r);
      const int4 m = cl.staged ? reinterpret_cast<const int4 *>(base + L.meta)[wid]
                               : __ldg(S.meta + s);
      XT rv[NVS];
#pragma unroll
      for (int i = 0; i < NVS; ++i) rv[i] = XT(0);
      if (r < S.n) {
        if (cl.staged && cl.rows_staged) {
          const XT *rs = reinterpret_cast<const XT *>(base + L.rows) + wid * 32 + lane;
#pragma unroll
          for (int i = 0; i < Epi::NV; ++i) rv[i] = rs[i * kPipeWarps * 32];
        } else {
#pragma unroll
          for (int i = 0; i < Epi::NV; ++i) rv[i] = epi.row_vec(i)[r];
        }
      }
      XT T;
      if (cl.staged) {
        const int64_t rel = static_cast<int64_t>(m.x - cl.slot0) * 32 + lane;
        const VT *v = reinterpret_cast<const VT *>(base + L.vals) + rel;
        const int32_t *ci =
            m.z ? nullptr
                : (cols_staged ? reinterpret_cast<const int32_t *>(base + L.cols) + rel
                               : S.scol + static_cast<int64_t>(m.x) * 32 + lane);
        T = m.z == 3 ? stencil_row_sum<VT, XT, KB>(v, S, g)
                     : row_sum<VT, XT, KB>(v, ci, S.soff + m.w, m.y, r, hi, m.z == 2, g);
      } else {
        const int64_t at = static_cast<int64_t>(m.x) * 32 + lane;
        T = m.z == 3 ? stencil_row_sum<VT, XT, KB>(val + at, S, g)
                     : row_sum<VT, XT, KB>(val + at, m.z ? nullptr : S.scol + at, S.soff + m.w,
                                           m.y, r, hi, m.z == 2, g);
      }
      if (r < S.n) epi.apply(r, T, rv);
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(&empty[st]);
  }
  epi.finish(wid, lane);
}

// Self-test of the bounded pipeline waits with the pipeline's own wait
// functions: one CTA; lane 0 of warp 0 (the producer) stages one real bulk
// copy on barrier 0 and drains it; warp 1 (a consumer) waits on barrier 1,
// which nothing ever arms, until limit_ns runs out, and reports that as a
// pipelined pass does.  flags bit 0: the consumer gave up; bit 1: the copy
// landed before the producer left.
__global__ void k_wait_selftest(const int4 *__restrict__ src, unsigned long long limit_ns,
                                int *flags) {
  __shared__ __align__(128) int4 buf[16];
  __shared__ __align__(8) uint64_t bar[2];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (threadIdx.x == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (wid == 0) {
    if (lane != 0) return;
    mbar_arrive_tx(&bar[0], sizeof(buf));
    bulk_load(buf, src, sizeof(buf), &bar[0]);
    if (mbar_wait(&bar[0], 0, kDrainLimitNs)) atomicOr(flags, 2);
    return;
  }
  if (!mbar_wait_warp(&bar[1], 0, limit_ns) && lane == 0) {
    atomicOr(flags, 1);
    atomicExch(&g_sliced_wait_error, 1);
  }
}

// ---- small levels on one thread-block cluster ---------------------------------
// A level whose sliced copy fits in the shared memory of a cluster of at most
// kClusterMax CTAs runs all its sweeps (and the residual after them) in one
// launch: CTA q loads slices [q spc, (q + 1) spc) -- values, explicit
// columns, metadata, f, d and its rows of the iterate -- once, and every pass
// reads the iterate of the other CTAs through distributed shared memory, with
// a cluster barrier between passes.  The row sums repeat slice_row_sum
// operation for operation (same gather indices, same partial sums, same
// batch size), so the results are those of the separate launches bit for
// bit, while the level costs one launch instead of one per pass.
namespace cg = cooperative_groups;

constexpr int kClusterWarps = 16;
constexpr int kClusterThreads = kClusterWarps * 32;
constexpr int kClusterMax = 8;  // the portable cluster size
constexpr size_t kClusterSmem = 220 * 1024;
// A pass costs about one dependent shared-memory gather chain per slot of
// the busiest warp; beyond this many slots a separate launch per sweep over
// the whole GPU is faster (27-point stencils: one 32-row slice per warp).
constexpr int32_t kClusterWarpSlots = 32;

// One CTA's shared memory: the same offsets in every CTA of the cluster, so
// a remote CTA's iterate sits where the local one does.
struct ClusterLayout {
  uint32_t vals, cols, meta, x0, x1, f, d, bytes;
  __host__ __device__ ClusterLayout(int slots, int vbytes, bool cols_on, int spc, int xbytes) {
    vals = 0;
    cols = vals + ((static_cast<uint32_t>(slots) * 32u * vbytes + 15u) & ~15u);
    meta = cols + (cols_on ? static_cast<uint32_t>(slots) * 32u * 4u : 0u);
    const uint32_t rows = static_cast<uint32_t>(spc) * 32u * xbytes;
    x0 = meta + static_cast<uint32_t>(spc) * 16u;
    x1 = x0 + rows;
    f = x1 + rows;
    d = f + rows;
    bytes = d + rows;
  }
};

template <typename XT>
struct ClusterArgs {
  const XT *f, *d;
  XT *u;      // the iterate: read unless zero_start, written at the end
  XT *res;    // f - A u after the sweeps (nullptr: none)
  int k;      // sweeps
  int zero_start;
};

// Gathers from the iterate held across the cluster's shared memory: row j
// lives in CTA j >> shift at position j & mask.
template <typename XT>
struct ClusterGather {
  XT *xc;
  int shift;
  int32_t mask, r;
  __device__ void row(int32_t rr) { r = rr; }
  __device__ XT operator()(int32_t j) const {
    cg::cluster_group cl = cg::this_cluster();
    const XT *base = cl.map_shared_rank(xc, static_cast<int>(j >> shift));
    return base[j & mask];
  }
  __device__ XT rel(int32_t o) const { return (*this)(r + o); }
  __device__ XT rel_param(int32_t o) const { return (*this)(r + o); }
};

template <typename VT, typename XT, int KB>
__global__ void __launch_bounds__(kClusterThreads)
    k_sl_cluster(SlicedView S, ClusterArgs<XT> a) {
  pdl_wait();
  pdl_trigger();
  cg::cluster_group cl = cg::this_cluster();
  extern __shared__ __align__(128) unsigned char smem[];
  const ClusterLayout L(S.cl_slots, sizeof(VT), S.cols_staged != 0, S.cl_spc, sizeof(XT));
  __shared__ __align__(8) uint64_t loaded;
  const int q = static_cast<int>(cl.block_rank());
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  // slices per CTA are a power of two: a row's owner is a shift away
  const int32_t spc = S.cl_spc, rows_cta = spc * 32;
  const int rshift = __ffs(rows_cta) - 1;
  const int32_t s0 = min(q * spc, S.nslices), s1 = min(s0 + spc, S.nslices);
  const int32_t r0 = s0 * 32, nrow = max(0, min(s1 * 32, S.n) - r0);
  const int32_t p0 = S.sptr[s0], p1 = S.sptr[s1];
  VT *sv = reinterpret_cast<VT *>(smem + L.vals);
  int32_t *sc = reinterpret_cast<int32_t *>(smem + L.cols);
  int4 *sm = reinterpret_cast<int4 *>(smem + L.meta);
  XT *xb0 = reinterpret_cast<XT *>(smem + L.x0), *xb1 = reinterpret_cast<XT *>(smem + L.x1);
  XT *sf = reinterpret_cast<XT *>(smem + L.f), *sd = reinterpret_cast<XT *>(smem + L.d);
  const VT *val = static_cast<const VT *>(S.val);
  // The CTA's slots plus the padding a batch may read past its last slice
  // (the global copy is padded the same way; those values are never used),
  // its columns and metadata: bulk async copies under one mbarrier (all
  // 16-byte multiples at 16-byte aligned addresses).
  const uint32_t nsl = static_cast<uint32_t>(p1 - p0 + kSlotPad) * 32u;
  if (tid == 0) {
    mbar_init(&loaded, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    const uint32_t vbytes = nsl * sizeof(VT), cbytes = S.cols_staged ? nsl * 4u : 0u;
    const uint32_t mbytes = static_cast<uint32_t>(s1 - s0) * 16u;
    mbar_arrive_tx(&loaded, vbytes + cbytes + mbytes);
    bulk_load(sv, val + static_cast<int64_t>(p0) * 32, vbytes, &loaded);
    if (cbytes) bulk_load(sc, S.scol + static_cast<int64_t>(p0) * 32, cbytes, &loaded);
    bulk_load(sm, S.meta + s0, mbytes, &loaded);
  }
  for (int32_t i = tid; i < nrow; i += kClusterThreads) {
    const XT fi = a.f[r0 + i], di = a.d[r0 + i];
    sf[i] = fi;
    sd[i] = di;
    xb0[i] = a.zero_start ? fi / di : a.u[r0 + i];
  }
  __syncthreads();  // (the barrier's initialisation before anyone waits on it)
  if (!mbar_wait(&loaded, 0, kDrainLimitNs)) atomicExch(&g_sliced_wait_error, 1);
  cl.sync();
  const int32_t hi = S.n - 1;
  const int sweeps = a.k - (a.zero_start ? 1 : 0);
  const int passes = sweeps + (a.res ? 1 : 0);
  int cur = 0;
  for (int p = 0; p < passes; ++p) {
    const bool resid = p == sweeps;
    XT *xc = cur ? xb1 : xb0;
    XT *xn = cur ? xb0 : xb1;
    ClusterGather<XT> gath{xc, rshift, rows_cta - 1, 0};
    for (int32_t ls = wid; ls < s1 - s0; ls += kClusterWarps) {
      const int4 m = sm[ls];
      const int32_t r = (s0 + ls) * 32 + lane;
      const int64_t rel = static_cast<int64_t>(m.x - p0) * 32 + lane;
      gath.row(r);
      const XT T = m.z == 3 ? stencil_row_sum<VT, XT, KB>(sv + rel, S, gath)
                            : row_sum<VT, XT, KB>(sv + rel, m.z ? nullptr : sc + rel,
                                                  S.soff + m.w, m.y, r, hi, m.z == 2, gath);
      if (r < S.n) {
        const int32_t rl = r - r0;
        if (resid)
          a.res[r] = sf[rl] - T;
        else
          xn[rl] = ((-T + sf[rl]) / sd[rl]) + xc[rl];
      }
    }
    cl.sync();  // every read of this pass's iterate is done before the next
    if (!resid) cur ^= 1;
  }
  const XT *xf = cur ? xb1 : xb0;
  for (int32_t i = tid; i < nrow; i += kClusterThreads) a.u[r0 + i] = xf[i];
}

// ---- launch configuration ----------------------------------------------------

struct PipeCfg {
  int grid = 0;
  size_t smem = 0;
};

// Occupancy-derived persistent grid for one kernel and stage size, cached
// (the occupancy query and the shared-memory attribute are host calls made
// once per kernel and size, outside any stream capture: sliced_build warms
// the cache for the kernels a matrix will use).
template <typename K>
bcmg_status pipe_cfg(K kernel, size_t stage_bytes, int32_t nchunks, PipeCfg *out) {
  static std::mutex mu;
  static std::map<std::pair<const void *, size_t>, int> cache;
  const size_t smem = kPipeStages * stage_bytes;
  int per_sm = 0;
  {
    std::lock_guard<std::mutex> lk(mu);
    auto key = std::make_pair(reinterpret_cast<const void *>(kernel), smem);
    auto it = cache.find(key);
    if (it != cache.end()) {
      per_sm = it->second;
    } else {
      // Always the largest size any matrix may ask for, so a later matrix
      // never lowers the limit another one relies on.
      BCMG_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     static_cast<int>(kPipeStages * kMaxStageBytes)));
      BCMG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kPipeThreads,
                                                              smem));
      if (per_sm < 1) return set_error(BCMG_ERR_INTERNAL, "sliced pipeline does not fit an SM");
      cache[key] = per_sm;
    }
  }
  int dev = 0, sms = kNumSM;
  if (cudaGetDevice(&dev) == cudaSuccess)
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  // At most kRedBlocks CTAs: the FCG epilogue writes one partial per CTA.
  out->grid = static_cast<int>(std::min<int64_t>(
      std::min<int64_t>(nchunks, static_cast<int64_t>(per_sm) * sms), kRedBlocks));
  out->smem = smem;
  return BCMG_OK;
}

// Gathers per batch (KB) of a copy with mean slice width `batch`, matched to
// it so that 5-point (2-D), 7- and 27-point (3-D) stencils issue no padding
// gathers and test no slot (27: FP32 vectors).  FP64 vectors take at most 14
// gathers per batch (two batches cover a 27-point row), which keeps three
// CTAs per SM in the register file.  The summation order depends on KB, so
// every kernel reading a copy uses this rule.
inline int slot_batch(int32_t batch, bool f64) {
  if (batch <= 5) return 5;
  if (batch <= 7) return 7;
  if (batch <= 8) return 8;
  if (f64) return 14;
  if (batch <= 16) return 16;
  return batch <= 27 ? 27 : 28;
}

inline int value_bytes(int vtype) {
  return vtype == kValF64 ? 8 : (vtype == kValF32 ? 4 : 2);
}

template <typename VT, typename XT, typename Epi>
bcmg_status pipe_launch(const SlicedView &S, const XT *x, const Epi &epi, cudaStream_t st,
                        bool warm_only = false) {
  if (S.nslices <= 0) return BCMG_OK;
  const int32_t nchunks = ceil_div(S.nslices, kPipeWarps);
  const StageLayout L(S.cap_slots, sizeof(VT), sizeof(XT), S.cols_staged != 0, Epi::NV);
  PipeCfg cfg;
#define BCMG_PIPE_KB(KB_)                                                                   \
  do {                                                                                      \
    auto kern = k_sl_pipe<VT, XT, Epi, KB_>;                                                \
    BCMG_TRY(pipe_cfg(kern, L.bytes, nchunks, &cfg));                                       \
    if (!warm_only)                                                                         \
      launch_pdl(kern, cfg.grid, kPipeThreads, cfg.smem, st, S, static_cast<const VT *>(S.val), \
             x, epi, S.cap_slots, S.cols_staged);                                           \
  } while (0)
  switch (slot_batch(S.batch, sizeof(XT) == 8)) {
    case 5: BCMG_PIPE_KB(5); break;
    case 7: BCMG_PIPE_KB(7); break;
    case 8: BCMG_PIPE_KB(8); break;
    case 14: if constexpr (sizeof(XT) == 8) BCMG_PIPE_KB(14); break;
    case 16: if constexpr (sizeof(XT) == 4) BCMG_PIPE_KB(16); break;
    case 27: if constexpr (sizeof(XT) == 4) BCMG_PIPE_KB(27); break;
    default: if constexpr (sizeof(XT) == 4) BCMG_PIPE_KB(28); break;
  }
#undef BCMG_PIPE_KB
  if (!warm_only) BCMG_LAUNCH_CHECK();
  return BCMG_OK;
}

// One cluster launch (k_sl_cluster): a grid of exactly one cluster, the
// gather batch chosen as pipe_launch chooses it (the partial sums depend on
// it).  The shared-memory attribute is set on first use, which sliced_build
// makes happen outside any stream capture.
template <typename VT, typename XT, int KB>
bcmg_status cluster_launch_kb(const SlicedView &S, const ClusterArgs<XT> &a, cudaStream_t st,
                              bool warm_only) {
  auto kern = k_sl_cluster<VT, XT, KB>;
  {
    static std::mutex mu;
    static bool attr_set = false;
    std::lock_guard<std::mutex> lk(mu);
    if (!attr_set) {
      BCMG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     static_cast<int>(kClusterSmem)));
      attr_set = true;
    }
  }
  if (warm_only) return BCMG_OK;
  const ClusterLayout L(S.cl_slots, sizeof(VT), S.cols_staged != 0, S.cl_spc, sizeof(XT));
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(S.cl_size);
  cfg.blockDim = dim3(kClusterThreads);
  cfg.dynamicSmemBytes = L.bytes;
  cfg.stream = st;
  cudaLaunchAttribute attr[2];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = S.cl_size;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  attr[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[1].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 2;
  g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
  BCMG_CUDA(cudaLaunchKernelEx(&cfg, kern, S, a));
  return BCMG_OK;
}

template <typename VT, typename XT>
bcmg_status cluster_launch(const SlicedView &S, const ClusterArgs<XT> &a, cudaStream_t st,
                           bool warm_only = false) {
  switch (slot_batch(S.batch, sizeof(XT) == 8)) {
    case 5: return cluster_launch_kb<VT, XT, 5>(S, a, st, warm_only);
    case 7: return cluster_launch_kb<VT, XT, 7>(S, a, st, warm_only);
    case 8: return cluster_launch_kb<VT, XT, 8>(S, a, st, warm_only);
    default: break;
  }
  if constexpr (sizeof(XT) == 8) {
    return cluster_launch_kb<VT, XT, 14>(S, a, st, warm_only);
  } else {
    switch (slot_batch(S.batch, false)) {
      case 16: return cluster_launch_kb<VT, XT, 16>(S, a, st, warm_only);
      case 27: return cluster_launch_kb<VT, XT, 27>(S, a, st, warm_only);
      default: return cluster_launch_kb<VT, XT, 28>(S, a, st, warm_only);
    }
  }
}

template <typename XT>
bcmg_status cluster_dispatch(const SlicedView &S, const ClusterArgs<XT> &a, cudaStream_t st,
                             bool warm_only) {
  if constexpr (sizeof(XT) == 8) {
    switch (S.vtype) {
      case kValF64: return cluster_launch<double, double>(S, a, st, warm_only);
      case kValF32: return cluster_launch<float, double>(S, a, st, warm_only);
      case kValBF16: return cluster_launch<__nv_bfloat16, double>(S, a, st, warm_only);
      default: return cluster_launch<__half, double>(S, a, st, warm_only);
    }
  } else {
    switch (S.vtype) {
      case kValF32: return cluster_launch<float, float>(S, a, st, warm_only);
      case kValBF16: return cluster_launch<__nv_bfloat16, float>(S, a, st, warm_only);
      case kValF16: return cluster_launch<__half, float>(S, a, st, warm_only);
      default: return set_error(BCMG_ERR_INTERNAL, "FP32-vector cluster passes on FP64 values");
    }
  }
}

template <typename VT, typename XT>
bcmg_status relax_as(const SlicedView &S, const XT *d, const XT *f, const XT *u, XT *u_out,
                     cudaStream_t st, bool warm_only = false) {
  EpiRelax<XT> e{f, d, u, u_out};
  return pipe_launch<VT, XT>(S, u, e, st, warm_only);
}

template <typename VT>
bcmg_status relax_widen_as(const SlicedView &S, const float *d, const float *f, const float *u,
                           double *out, cudaStream_t st, bool warm_only = false) {
  EpiRelaxWiden e{f, d, u, out};
  return pipe_launch<VT, float>(S, u, e, st, warm_only);
}

template <typename VT, typename XT>
bcmg_status residual_as(const SlicedView &S, const XT *f, const XT *u, XT *res,
                        cudaStream_t st, bool warm_only = false) {
  EpiResidual<XT> e{f, res};
  return pipe_launch<VT, XT>(S, u, e, st, warm_only);
}

// Fills the occupancy cache for the kernels this matrix will run, so no
// attribute or occupancy call happens inside a captured solve.
template <typename VT>
bcmg_status warm_f64_vectors(const SlicedView &S) {
  BCMG_TRY((relax_as<VT, double>(S, nullptr, nullptr, nullptr, nullptr, 0, true)));
  BCMG_TRY((residual_as<VT, double>(S, nullptr, nullptr, nullptr, 0, true)));
  EpiSpmv e1{nullptr};
  BCMG_TRY((pipe_launch<VT, double>(S, static_cast<const double *>(nullptr), e1, 0, true)));
  EpiFcgDots e2{};
  BCMG_TRY((pipe_launch<VT, double>(S, static_cast<const double *>(nullptr), e2, 0, true)));
  EpiReplace e3{};
  BCMG_TRY((pipe_launch<VT, double>(S, static_cast<const double *>(nullptr), e3, 0, true)));
  return BCMG_OK;
}

template <typename VT>
bcmg_status warm_f32_vectors(const SlicedView &S) {
  BCMG_TRY((relax_as<VT, float>(S, nullptr, nullptr, nullptr, nullptr, 0, true)));
  BCMG_TRY((relax_widen_as<VT>(S, nullptr, nullptr, nullptr, nullptr, 0, true)));
  BCMG_TRY((residual_as<VT, float>(S, nullptr, nullptr, nullptr, 0, true)));
  EpiSpmvT<float> e{nullptr};
  BCMG_TRY((pipe_launch<VT, float>(S, static_cast<const float *>(nullptr), e, 0, true)));
  return BCMG_OK;
}

bcmg_status warm_cluster(const SlicedView &S) {
  if (S.cl_size <= 0) return BCMG_OK;
  if (S.xtype == kValF64) return cluster_dispatch<double>(S, ClusterArgs<double>{}, 0, true);
  return cluster_dispatch<float>(S, ClusterArgs<float>{}, 0, true);
}

bcmg_status warm_kernels(const SlicedView &S) {
  BCMG_TRY(warm_cluster(S));
  if (S.xtype == kValF64) {
    switch (S.vtype) {
      case kValF64: return warm_f64_vectors<double>(S);
      case kValF32: return warm_f64_vectors<float>(S);
      case kValBF16: return warm_f64_vectors<__nv_bfloat16>(S);
      default: return warm_f64_vectors<__half>(S);
    }
  }
  switch (S.vtype) {
    case kValF32: return warm_f32_vectors<float>(S);
    case kValBF16: return warm_f32_vectors<__nv_bfloat16>(S);
    case kValF16: return warm_f32_vectors<__half>(S);
    default: return set_error(BCMG_ERR_INTERNAL, "FP32-vector copy with FP64 values");
  }
}

// Small levels: the thread-block cluster that holds the whole copy, if one
// does (cl_size 0 otherwise).
bcmg_status plan_cluster(SlicedMat *out, cudaStream_t s) {
  const int32_t ns = out->nslices;
  out->cl_size = out->cl_spc = out->cl_slots = 0;
  if (ns <= kClusterMax * 64) {
    std::vector<int32_t> h_sptr(static_cast<size_t>(ns) + 1);
    BCMG_CUDA(cudaMemcpyAsync(h_sptr.data(), out->sptr, sizeof(int32_t) * (ns + 1),
                              cudaMemcpyDeviceToHost, s));
    BCMG_CUDA(cudaStreamSynchronize(s));
    int32_t spc = 1;  // a power of two with at most kClusterMax CTAs
    while (static_cast<int64_t>(spc) * kClusterMax < ns) spc <<= 1;
    const int32_t csize = ceil_div(ns, spc);
    int32_t cap = 0, warp_slots = 0;
    for (int32_t q = 0; q < csize; ++q) {
      const int32_t s0 = q * spc, s1 = std::min(s0 + spc, ns);
      cap = std::max(cap, h_sptr[s1] - h_sptr[s0]);
      for (int32_t w = 0; w < kClusterWarps; ++w) {
        int32_t t = 0;
        for (int32_t i = s0 + w; i < s1; i += kClusterWarps) t += h_sptr[i + 1] - h_sptr[i];
        warp_slots = std::max(warp_slots, t);
      }
    }
    cap += kSlotPad;
    const ClusterLayout CL(cap, static_cast<int>(value_bytes(out->vtype)), out->has_columns, spc,
                           out->xtype == kValF64 ? 8 : 4);
    if (CL.bytes <= kClusterSmem && warp_slots <= kClusterWarpSlots) {
      out->cl_size = csize;
      out->cl_spc = spc;
      out->cl_slots = cap;
    }
  }
  return BCMG_OK;
}

}  // namespace

size_t SlicedMat::bytes() const {
  if (!nslices || borrowed) return 0;
  const size_t vb = value_bytes(vtype);
  const size_t sl = (static_cast<size_t>(slots) + kSlotPad) * 32;
  return vb * sl + (has_columns ? 4 * sl : 0) + 4 * (static_cast<size_t>(slots) + kSlotPad) +
         4 * (static_cast<size_t>(nslices) + 1) + 16 * static_cast<size_t>(nslices);
}

void SlicedMat::release(cudaStream_t s) {
  if (borrowed) {  // another copy owns the arrays
    sptr = scol = soff = nullptr;
    meta = nullptr;
    val = nullptr;
    borrowed = false;
  }
  dev_free(sptr, s);
  dev_free(meta, s);
  dev_free(scol, s);
  dev_free(soff, s);
  char *vp = static_cast<char *>(val);
  dev_free(vp, s);
  val = nullptr;
  cl_size = cl_spc = cl_slots = 0;
  sten_w = 0;
  nslices = 0;
  has_columns = false;
}

SlicedView SlicedMat::view() const {
  SlicedView v;
  v.n = n;
  v.nslices = nslices;
  v.sptr = sptr;
  v.meta = meta;
  v.scol = scol;
  v.soff = soff;
  v.val = val;
  v.vtype = vtype;
  v.cap_slots = cap_slots;
  v.cols_staged = has_columns ? 1 : 0;
  v.batch = batch;
  v.xtype = xtype;
  v.wait_ns = wait_ns;
  v.cl_size = cl_size;
  v.cl_spc = cl_spc;
  v.cl_slots = cl_slots;
  v.sten_w = sten_w;
  for (int i = 0; i < kStencilMax; ++i) v.sten_off[i] = sten_off[i];
  return v;
}

bcmg_status sliced_build(const CsrView &A, int vtype, SlicedMat *out, cudaStream_t s,
                         bool narrow) {
  out->release(s);
  const int32_t n = A.n;
  if (n <= 0) return BCMG_OK;
  const int32_t ns = ceil_div(n, 32);
  out->n = n;
  out->nslices = ns;
  out->xtype = vtype == kValF64 ? kValF64 : kValF32;
  out->vtype = vtype;
  DevBuf<int32_t> width, kind, stats, tmp, offrange;
  BCMG_TRY(offrange.alloc(2, s));
  BCMG_CUDA(cudaMemsetAsync(offrange.get(), 0, 2 * sizeof(int32_t), s));  // 0 in the range
  BCMG_TRY(dev_alloc(&out->sptr, ns + 1, s));
  BCMG_TRY(dev_alloc(&out->meta, ns, s));
  BCMG_TRY(width.alloc(ns, s));
  BCMG_TRY(kind.alloc(ns, s));
  BCMG_TRY(stats.alloc(3, s));  // chunk max, any column slice, exact types
  BCMG_TRY(tmp.alloc(scan_tmp_size(ns), s));
  const int blocks = ceil_div(ns, kWarpsPerBlock);
  launch(k_slice_shape, blocks, kWarpsPerBlock * 32, 0, s, n, ns, A.row, A.col, width.get(),
         kind.get(), offrange.get());
  BCMG_TRY(exclusive_scan(width.get(), out->sptr, ns, out->sptr + ns, tmp.get(), s));
  BCMG_CUDA(cudaMemsetAsync(stats.get(), 0, 2 * sizeof(int32_t), s));
  // FP64 -> BF16 cuts the value stream 4x, FP32 -> BF16 2x; a copy serving
  // FP32 vectors narrows to BF16 or FP16 only, and copies already stored in
  // 16 bits (rounded on purpose) stay as they are.
  const bool try_narrow = narrow && (vtype == kValF64 || vtype == kValF32) && A.nnz > 0;
  {
    const int32_t all = 7;
    BCMG_CUDA(cudaMemcpyAsync(stats.get() + 2, &all, sizeof(int32_t), cudaMemcpyHostToDevice, s));
  }
  if (try_narrow)
    launch(k_value_exact, std::min<int64_t>(ceil_div(A.nnz, 256), 8 * kNumSM), 256, 0, s,
           static_cast<int64_t>(A.nnz), A.val, stats.get());
  const int32_t nchunks = ceil_div(ns, kPipeWarps);
  launch(k_slice_stats, ceil_div(nchunks, 256), 256, 0, s, ns, out->sptr, kind.get(),
         stats.get());
  BCMG_LAUNCH_CHECK();
  int32_t h_stats[4] = {0, 0, 0, 0};
  BCMG_CUDA(cudaMemcpyAsync(h_stats, stats.get(), 3 * sizeof(int32_t), cudaMemcpyDeviceToHost,
                            s));
  BCMG_CUDA(cudaMemcpyAsync(h_stats + 3, out->sptr + ns, sizeof(int32_t),
                            cudaMemcpyDeviceToHost, s));
  BCMG_CUDA(cudaStreamSynchronize(s));
  const int32_t slots = h_stats[3];
  // Exact narrowing: the narrowest storage that holds every value bit for bit
  // (BF16, then FP16, then FP32); the kernels widen and accumulate in the
  // vector type, so the arithmetic is unchanged.
  if (try_narrow) {
    const int exact = h_stats[2];
    if (exact & 2) vtype = kValBF16;
    else if (exact & 4) vtype = kValF16;
    else if ((exact & 1) && vtype == kValF64) vtype = kValF32;
  }
  out->vtype = vtype;
  out->narrowed = out->vtype != (out->xtype == kValF64 ? kValF64 : kValF32);
  out->slots = slots;
  out->has_columns = h_stats[1] != 0;
  out->batch = static_cast<int32_t>((static_cast<int64_t>(slots) + ns - 1) / ns);
  const size_t vb = value_bytes(vtype);
  const int64_t padded = static_cast<int64_t>(slots) + kSlotPad;
  {
    char *vp = nullptr;
    BCMG_TRY(dev_alloc(&vp, static_cast<int64_t>(vb) * padded * 32, s));
    out->val = vp;
  }
  BCMG_CUDA(cudaMemsetAsync(static_cast<char *>(out->val) + vb * static_cast<size_t>(slots) * 32,
                            0, vb * kSlotPad * 32, s));
  // Explicit columns are only read in column slices; a matrix made of offset
  // slices alone (a stencil) stores none.
  if (out->has_columns) {
    BCMG_TRY(dev_alloc(&out->scol, padded * 32, s));
    BCMG_CUDA(cudaMemsetAsync(out->scol, 0, sizeof(int32_t) * padded * 32, s));
  }
  BCMG_TRY(dev_alloc(&out->soff, padded, s));
  BCMG_CUDA(cudaMemsetAsync(out->soff, 0, sizeof(int32_t) * padded, s));
  switch (vtype) {
    case kValF64:
      launch(k_slice_fill<double>, blocks, kWarpsPerBlock * 32, 0, s, n, ns, A.row, A.col,
             A.val, out->sptr, width.get(), kind.get(), static_cast<double *>(out->val),
             out->scol, out->soff);
      break;
    case kValF32:
      launch(k_slice_fill<float>, blocks, kWarpsPerBlock * 32, 0, s, n, ns, A.row, A.col,
             A.val, out->sptr, width.get(), kind.get(), static_cast<float *>(out->val),
             out->scol, out->soff);
      break;
    case kValBF16:
      launch(k_slice_fill<__nv_bfloat16>, blocks, kWarpsPerBlock * 32, 0, s, n, ns, A.row,
             A.col, A.val, out->sptr, width.get(), kind.get(),
             static_cast<__nv_bfloat16 *>(out->val), out->scol, out->soff);
      break;
    default:
      launch(k_slice_fill<__half>, blocks, kWarpsPerBlock * 32, 0, s, n, ns, A.row, A.col,
             A.val, out->sptr, width.get(), kind.get(), static_cast<__half *>(out->val),
             out->scol, out->soff);
      break;
  }
  BCMG_LAUNCH_CHECK();
  // Runs of identical offset lists share the run head's copy.
  {
    DevBuf<int32_t> flag, rid, head;
    BCMG_TRY(flag.alloc(ns, s));
    BCMG_TRY(rid.alloc(ns + 1, s));
    BCMG_TRY(head.alloc(ns, s));
    launch(k_slice_runs, blocks, kWarpsPerBlock * 32, 0, s, ns, out->sptr, width.get(),
           kind.get(), out->soff, flag.get());
    BCMG_TRY(exclusive_scan(flag.get(), rid.get(), ns, rid.get() + ns, tmp.get(), s));
    launch(k_slice_heads, ceil_div(ns, 256), 256, 0, s, ns, flag.get(), rid.get(), head.get());
    launch(k_slice_meta, ceil_div(ns, 256), 256, 0, s, n, ns, out->sptr, width.get(),
           kind.get(), flag.get(), rid.get(), head.get(), offrange.get(), out->meta);
    BCMG_LAUNCH_CHECK();
  }
  // Stencil: the offsets of the first interior slice as wide as the mean
  // slice width (at most two slot batches and kStencilMax) become kernel
  // parameters for every slice that has the same list (kind 3).
  out->sten_w = 0;
  std::fill(out->sten_off, out->sten_off + kStencilMax, 0);
  if (const int kb = out->batch;
      kb <= kStencilMax && kb <= 2 * slot_batch(out->batch, out->xtype == kValF64)) {
    BCMG_CUDA(cudaMemcpyAsync(stats.get(), &ns, sizeof(int32_t), cudaMemcpyHostToDevice, s));
    launch(k_stencil_pick, ceil_div(ns, 256), 256, 0, s, ns, out->meta, kb, stats.get());
    BCMG_LAUNCH_CHECK();
    int32_t first = ns;
    BCMG_CUDA(cudaMemcpyAsync(&first, stats.get(), sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    BCMG_CUDA(cudaStreamSynchronize(s));
    int4 hm = make_int4(0, 0, 0, 0);
    if (first < ns) {
      BCMG_CUDA(cudaMemcpyAsync(&hm, out->meta + first, sizeof(int4), cudaMemcpyDeviceToHost,
                                s));
      BCMG_CUDA(cudaStreamSynchronize(s));
    }
    if (first < ns && hm.z == 2 && hm.y == kb) {
      BCMG_CUDA(cudaMemcpyAsync(out->sten_off, out->soff + hm.w, sizeof(int32_t) * kb,
                                cudaMemcpyDeviceToHost, s));
      launch(k_slice_stencil, ceil_div(ns, 256), 256, 0, s, ns, out->soff, hm.w, kb, out->meta);
      BCMG_LAUNCH_CHECK();
      BCMG_CUDA(cudaStreamSynchronize(s));
      out->sten_w = kb;
    }
  }
  // Stage capacity: the largest chunk, capped so two stages fit in shared
  // memory (larger chunks are read from global memory by the consumers).
  const size_t per_slot = 32 * (vb + (out->has_columns ? 4 : 0));
  const size_t fixed = kPipeWarps * 16 + 3 * kPipeWarps * 32 * 8 + 128;
  const int32_t cap_max =
      static_cast<int32_t>((kMaxStageBytes - fixed) / per_slot) - kSlotPad;
  out->cap_slots = std::max<int32_t>(1, std::min<int32_t>(h_stats[0], cap_max));
  BCMG_TRY(plan_cluster(out, s));
  BCMG_TRY(warm_kernels(out->view()));
  return BCMG_OK;
}

bcmg_status sliced_alias(const SlicedMat &src, int xtype, SlicedMat *out, cudaStream_t s) {
  out->release(s);
  if (src.borrowed || !src.narrowed || value_bytes(src.vtype) != 2)
    return set_error(BCMG_ERR_INTERNAL, "sliced copy cannot be shared");
  *out = src;  // same arrays: sptr, meta (stencil marks included), offsets, values
  out->borrowed = true;
  out->xtype = xtype;
  BCMG_TRY(plan_cluster(out, s));  // the iterate's width enters the layout
  BCMG_TRY(warm_kernels(out->view()));
  return BCMG_OK;
}

template <typename XT>
bcmg_status sliced_relax_sweep(const SlicedView &S, const XT *d, const XT *f, const XT *u,
                               XT *u_out, cudaStream_t s) {
  if (std::is_same<XT, double>::value) {
    const double *dd = reinterpret_cast<const double *>(d);
    const double *fd = reinterpret_cast<const double *>(f);
    const double *ud = reinterpret_cast<const double *>(u);
    double *od = reinterpret_cast<double *>(u_out);
    switch (S.vtype) {
      case kValF64: return relax_as<double, double>(S, dd, fd, ud, od, s);
      case kValF32: return relax_as<float, double>(S, dd, fd, ud, od, s);
      case kValBF16: return relax_as<__nv_bfloat16, double>(S, dd, fd, ud, od, s);
      default: return relax_as<__half, double>(S, dd, fd, ud, od, s);
    }
  }
  const float *df = reinterpret_cast<const float *>(d);
  const float *ff = reinterpret_cast<const float *>(f);
  const float *uf = reinterpret_cast<const float *>(u);
  float *of = reinterpret_cast<float *>(u_out);
  if (S.vtype == kValF32) return relax_as<float, float>(S, df, ff, uf, of, s);
  if (S.vtype == kValBF16) return relax_as<__nv_bfloat16, float>(S, df, ff, uf, of, s);
  if (S.vtype == kValF16) return relax_as<__half, float>(S, df, ff, uf, of, s);
  return set_error(BCMG_ERR_INTERNAL, "sliced type mismatch");
}

bcmg_status sliced_relax_sweep_widen(const SlicedView &S, const float *d, const float *f,
                                     const float *u, double *out, cudaStream_t s) {
  if (S.xtype != kValF32) return set_error(BCMG_ERR_INTERNAL, "sliced type mismatch");
  if (S.vtype == kValF32) return relax_widen_as<float>(S, d, f, u, out, s);
  if (S.vtype == kValBF16) return relax_widen_as<__nv_bfloat16>(S, d, f, u, out, s);
  if (S.vtype == kValF16) return relax_widen_as<__half>(S, d, f, u, out, s);
  return set_error(BCMG_ERR_INTERNAL, "sliced type mismatch");
}

template <typename XT>
bcmg_status sliced_residual(const SlicedView &S, const XT *f, const XT *u, XT *res,
                            cudaStream_t s) {
  if (std::is_same<XT, double>::value) {
    const double *fd = reinterpret_cast<const double *>(f);
    const double *ud = reinterpret_cast<const double *>(u);
    double *rd = reinterpret_cast<double *>(res);
    switch (S.vtype) {
      case kValF64: return residual_as<double, double>(S, fd, ud, rd, s);
      case kValF32: return residual_as<float, double>(S, fd, ud, rd, s);
      case kValBF16: return residual_as<__nv_bfloat16, double>(S, fd, ud, rd, s);
      default: return residual_as<__half, double>(S, fd, ud, rd, s);
    }
  }
  const float *ff = reinterpret_cast<const float *>(f);
  const float *uf = reinterpret_cast<const float *>(u);
  float *rf = reinterpret_cast<float *>(res);
  if (S.vtype == kValF32) return residual_as<float, float>(S, ff, uf, rf, s);
  if (S.vtype == kValBF16) return residual_as<__nv_bfloat16, float>(S, ff, uf, rf, s);
  if (S.vtype == kValF16) return residual_as<__half, float>(S, ff, uf, rf, s);
  return set_error(BCMG_ERR_INTERNAL, "sliced type mismatch");
}

bcmg_status sliced_fcg_spmv_dots(const SlicedView &S, const double *v, double *w,
                                 const double *r, const double *q, double *partials,
                                 cudaStream_t s) {
  if (S.xtype != kValF64) return set_error(BCMG_ERR_INTERNAL, "FCG SpMV needs an FP64 copy");
  EpiFcgDots e{v, r, q, w, partials, {0.0, 0.0, 0.0}};
  switch (S.vtype) {
    case kValF64: return pipe_launch<double, double>(S, v, e, s);
    case kValF32: return pipe_launch<float, double>(S, v, e, s);
    case kValBF16: return pipe_launch<__nv_bfloat16, double>(S, v, e, s);
    default: return pipe_launch<__half, double>(S, v, e, s);
  }
}

bcmg_status sliced_replace(const SlicedView &S, const double *b, const double *x, double *r,
                           double *partials, const double *scal, cudaStream_t s) {
  if (S.xtype != kValF64) return set_error(BCMG_ERR_INTERNAL, "replacement needs an FP64 copy");
  EpiReplace e{b, r, partials, scal, {0.0}};
  switch (S.vtype) {
    case kValF64: return pipe_launch<double, double>(S, x, e, s);
    case kValF32: return pipe_launch<float, double>(S, x, e, s);
    case kValBF16: return pipe_launch<__nv_bfloat16, double>(S, x, e, s);
    default: return pipe_launch<__half, double>(S, x, e, s);
  }
}

bcmg_status sliced_spmv(const SlicedView &S, const double *x, double *y, cudaStream_t s) {
  if (S.xtype != kValF64) return set_error(BCMG_ERR_INTERNAL, "sliced SpMV needs an FP64 copy");
  EpiSpmv e{y};
  switch (S.vtype) {
    case kValF64: return pipe_launch<double, double>(S, x, e, s);
    case kValF32: return pipe_launch<float, double>(S, x, e, s);
    case kValBF16: return pipe_launch<__nv_bfloat16, double>(S, x, e, s);
    default: return pipe_launch<__half, double>(S, x, e, s);
  }
}

template <>
bcmg_status sliced_spmv_t<double>(const SlicedView &S, const double *x, double *y,
                                  cudaStream_t s) {
  return sliced_spmv(S, x, y, s);
}

template <>
bcmg_status sliced_spmv_t<float>(const SlicedView &S, const float *x, float *y,
                                 cudaStream_t s) {
  EpiSpmvT<float> e{y};
  switch (S.vtype) {
    case kValF32: return pipe_launch<float, float>(S, x, e, s);
    case kValBF16: return pipe_launch<__nv_bfloat16, float>(S, x, e, s);
    case kValF16: return pipe_launch<__half, float>(S, x, e, s);
    default: return set_error(BCMG_ERR_INTERNAL, "FP32-vector SpMV on FP64 values");
  }
}

template <typename XT>
bcmg_status sliced_cluster(const SlicedView &S, const XT *d, const XT *f, XT *u, int k,
                           bool zero_start, XT *res, cudaStream_t s) {
  if (S.cl_size <= 0 || k < 1)
    return set_error(BCMG_ERR_INTERNAL, "no cluster plan for this level");
  ClusterArgs<XT> a{};
  a.f = f;
  a.d = d;
  a.u = u;
  a.res = res;
  a.k = k;
  a.zero_start = zero_start ? 1 : 0;
  return cluster_dispatch<XT>(S, a, s, false);
}
template bcmg_status sliced_cluster<double>(const SlicedView &, const double *, const double *,
                                            double *, int, bool, double *, cudaStream_t);
template bcmg_status sliced_cluster<float>(const SlicedView &, const float *, const float *,
                                           float *, int, bool, float *, cudaStream_t);

bcmg_status wait_selftest(unsigned long long limit_ns, cudaStream_t s) {
  DevBuf<int4> src;
  DevBuf<int> flags;
  BCMG_TRY(src.alloc(16, s));
  BCMG_TRY(flags.alloc(1, s));
  BCMG_CUDA(cudaMemsetAsync(src.get(), 0, sizeof(int4) * 16, s));
  BCMG_CUDA(cudaMemsetAsync(flags.get(), 0, sizeof(int), s));
  launch(k_wait_selftest, 1, 64, 0, s, src.get(), limit_ns, flags.get());
  BCMG_LAUNCH_CHECK();
  int h_flags = 0;
  BCMG_CUDA(cudaMemcpyAsync(&h_flags, flags.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
  BCMG_CUDA(cudaStreamSynchronize(s));
  if (!(h_flags & 2)) return set_error(BCMG_ERR_INTERNAL, "self-test copy did not drain");
  if (!(h_flags & 1)) return set_error(BCMG_ERR_INTERNAL, "self-test wait did not give up");
  return sliced_wait_status(s);
}

bcmg_status sliced_wait_status(cudaStream_t s) {
  int flag = 0;
  BCMG_CUDA(cudaMemcpyFromSymbolAsync(&flag, g_sliced_wait_error, sizeof(int), 0,
                                      cudaMemcpyDeviceToHost, s));
  BCMG_CUDA(cudaStreamSynchronize(s));
  if (flag) {
    const int zero = 0;
    BCMG_CUDA(cudaMemcpyToSymbolAsync(g_sliced_wait_error, &zero, sizeof(int), 0,
                                      cudaMemcpyHostToDevice, s));
    BCMG_CUDA(cudaStreamSynchronize(s));
    return set_error(BCMG_ERR_DEVICE_TIMEOUT,
                     "a sliced row pass gave up waiting for its staged copies");
  }
  return BCMG_OK;
}

template bcmg_status sliced_relax_sweep<double>(const SlicedView &, const double *,
                                                const double *, const double *, double *,
                                                cudaStream_t);
template bcmg_status sliced_relax_sweep<float>(const SlicedView &, const float *,
                                               const float *, const float *, float *,
                                               cudaStream_t);
template bcmg_status sliced_residual<double>(const SlicedView &, const double *,
                                             const double *, double *, cudaStream_t);
template bcmg_status sliced_residual<float>(const SlicedView &, const float *, const float *,
                                            float *, cudaStream_t);

}  // namespace bcmg
