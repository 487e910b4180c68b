// CUDA-side helpers shared by the library's .cu files: error checking that
// turns CUDA failures into bcmg_status, stream-ordered device buffers, launch
// geometry and small warp utilities.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <utility>

#include "host_util.h"

#define BCMG_CUDA(expr)                                                        \
  do {                                                                         \
    cudaError_t _e = (expr);                                                   \
    if (_e != cudaSuccess)                                                     \
      return ::bcmg::set_error(BCMG_ERR_CUDA, "%s:%d %s: %s", __FILE__,        \
                               __LINE__, #expr, cudaGetErrorString(_e));       \
  } while (0)

#define BCMG_LAUNCH_CHECK() BCMG_CUDA(cudaGetLastError())

namespace bcmg {

constexpr int kWarp = 32;
// 148 SMs on B200; grids of fixed-size reductions are multiples of this.
constexpr int kNumSM = 148;
constexpr uint64_t kNoOffer = ~0ull;

// Kernel launches issued by this library (bcmg_kernel_launches()).
extern std::atomic<unsigned long long> g_kernel_launches;
// Device allocations made by dev_alloc and not yet freed, all made so far
// (bcmg_debug_alloc_stats), and the countdown of an injected allocation
// failure (bcmg_debug_fail_alloc; -1: none armed).
extern std::atomic<long long> g_live_allocs;
extern std::atomic<long long> g_made_allocs;
extern std::atomic<long long> g_fail_alloc_countdown;

// True for the one allocation an armed bcmg_debug_fail_alloc picks (the
// countdown then disarms itself).
inline bool injected_alloc_failure() {
  long long c = g_fail_alloc_countdown.load(std::memory_order_relaxed);
  while (c >= 0)
    if (g_fail_alloc_countdown.compare_exchange_weak(c, c - 1, std::memory_order_relaxed))
      return c == 0;
  return false;
}

// Every kernel of the library is launched through here so launches are
// counted.
template <typename... KArgs, typename... Args>
inline void launch(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem,
                   cudaStream_t s, Args &&...args) {
  g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
  kernel<<<grid, block, smem, s>>>(std::forward<Args>(args)...);
}

// Programmatic dependent launch (solve-phase kernels): a kernel launched with
// launch_pdl may begin while the previous kernel on its stream is still
// running.  Every such kernel calls pdl_wait() first — it returns once the
// previous grid has completed and its writes are visible (a no-op for a
// normal launch) — and pdl_trigger() to let the next one start launching;
// a grid can only start after every CTA of its predecessor has triggered or
// exited, so those CTAs are all resident already.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// The dependency a launch_pdl kernel relaxes is on the kernel before it: a
// stream copy or memset just before it is not ordered by its pdl_wait().  A
// test that ran five sweeps after a device-to-device copy of the iterate
// read rows the copy had not yet written.  So copies between solve-phase
// kernels are kernels themselves (copy_t), and an upload that a launch_pdl
// kernel follows is closed by pdl_fence: an empty kernel launched normally,
// which starts only after everything before it on the stream has finished.
namespace {
__global__ void k_pdl_fence() {}
}  // namespace
inline void pdl_fence(cudaStream_t s) { k_pdl_fence<<<1, 1, 0, s>>>(); }

template <typename... KArgs, typename... Args>
inline void launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem,
                       cudaStream_t s, Args &&...args) {
  g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

inline int ceil_div(int64_t a, int64_t b) { return static_cast<int>((a + b - 1) / b); }

// Lanes per row for row-group kernels, from the average row length.
inline int group_for(int64_t nnz, int64_t n) {
  const int64_t avg = n > 0 ? nnz / n : 1;
  if (avg <= 4) return 4;
  if (avg <= 8) return 8;
  if (avg <= 16) return 16;
  return 32;
}

// Stream-ordered device allocation from the device's default memory pool.
template <typename T>
bcmg_status dev_alloc(T **p, int64_t count, cudaStream_t s) {
  *p = nullptr;
  if (count <= 0) return BCMG_OK;
  if (injected_alloc_failure())
    return set_error(BCMG_ERR_ALLOC,
                     "device allocation of %lld bytes failed: injected by bcmg_debug_fail_alloc",
                     static_cast<long long>(sizeof(T) * count));
  cudaError_t e = cudaMallocAsync(reinterpret_cast<void **>(p),
                                  sizeof(T) * static_cast<size_t>(count), s);
  if (e != cudaSuccess) {
    *p = nullptr;
    cudaGetLastError();
    return set_error(e == cudaErrorMemoryAllocation ? BCMG_ERR_ALLOC : BCMG_ERR_CUDA,
                     "device allocation of %lld bytes failed: %s",
                     static_cast<long long>(sizeof(T) * count), cudaGetErrorString(e));
  }
  g_live_allocs.fetch_add(1, std::memory_order_relaxed);
  g_made_allocs.fetch_add(1, std::memory_order_relaxed);
  return BCMG_OK;
}

template <typename T>
void dev_free(T *&p, cudaStream_t s) {
  if (p) {
    cudaFreeAsync(p, s);
    g_live_allocs.fetch_sub(1, std::memory_order_relaxed);
  }
  p = nullptr;
}

// Owning device array freed on the stream it was allocated on.
template <typename T>
struct DevBuf {
  T *ptr = nullptr;
  int64_t count = 0;
  cudaStream_t stream = nullptr;
  DevBuf() = default;
  DevBuf(const DevBuf &) = delete;
  DevBuf &operator=(const DevBuf &) = delete;
  DevBuf(DevBuf &&o) noexcept : ptr(o.ptr), count(o.count), stream(o.stream) {
    o.ptr = nullptr;
    o.count = 0;
  }
  DevBuf &operator=(DevBuf &&o) noexcept {
    if (this != &o) {
      reset();
      ptr = o.ptr;
      count = o.count;
      stream = o.stream;
      o.ptr = nullptr;
      o.count = 0;
    }
    return *this;
  }
  ~DevBuf() { reset(); }
  bcmg_status alloc(int64_t n, cudaStream_t s) {
    reset();
    stream = s;
    count = n;
    return dev_alloc(&ptr, n, s);
  }
  void reset() {
    dev_free(ptr, stream);
    count = 0;
  }
  T *get() const { return ptr; }
  T *release() {
    T *p = ptr;
    ptr = nullptr;
    count = 0;
    return p;
  }
};

}  // namespace bcmg
