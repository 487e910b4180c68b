// bcmg_k_relax_noalloc: the smoother sweeps of bcmg_k_relax without any
// device allocation.
//
// Who needs it: code that calls the smoother where it may not allocate
// device memory -- a host framework whose caching allocator owns all of the
// device memory, a plugin that must keep its footprint fixed after
// initialisation, or a latency-critical loop that cannot pay for an
// allocation and the synchronisation it can imply.  bcmg_k_relax takes a
// stream-ordered allocation for its ping-pong vector on every call; this
// variant uses a buffer that exists for the whole life of the process
// instead.
//
// The buffer is a file-scope __device__ array of kNoAllocMaxRows doubles
// (8 MiB).  Every GPU on which the library's module is loaded holds it until
// the process exits.  Host code cannot pass the array's name to a kernel (on
// the host that name is a stand-in, not a device address), so the device
// address is looked up with cudaGetSymbolAddress once per device, with that
// device current, on the first call made on the device; that first call
// should therefore happen before any stream capture.  The address stays
// cached per device ordinal for the rest of the process, so the entry point
// must not be used after the device was reset (cudaDeviceReset) or its
// primary context destroyed; `stream` must belong to the current device.
// Each call synchronises `stream` before it returns.  All calls share the
// one buffer: calls whose work overlaps on the GPU (other streams, other
// host threads) race on it and must be serialised by the caller.  The
// ping-pong buffer is fully written before it is read, so nothing has to be
// cleared between calls.
#include <mutex>

#include "common.cuh"
#include "kernels.h"

namespace bcmg {
namespace {

constexpr int32_t kNoAllocMaxRows = 1 << 20;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double g_relax_scratch[kNoAllocMaxRows];

std::mutex g_scratch_mutex;
double *g_scratch_addr[kMaxDevices] = {};

bcmg_status scratch_for_current_device(double **out) {
  int dev = 0;
  BCMG_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices)
    return set_error(BCMG_ERR_UNSUPPORTED, "device ordinal %d out of range", dev);
  std::lock_guard<std::mutex> lock(g_scratch_mutex);
  if (!g_scratch_addr[dev]) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_relax_scratch);
    if (e != cudaSuccess || !p)
      return set_error(BCMG_ERR_CUDA, "cudaGetSymbolAddress of the smoother buffer: %s",
                       cudaGetErrorString(e));
    g_scratch_addr[dev] = static_cast<double *>(p);
  }
  *out = g_scratch_addr[dev];
  return BCMG_OK;
}

}  // namespace
}  // namespace bcmg

using namespace bcmg;

extern "C" bcmg_status bcmg_k_relax_noalloc(int32_t n, int32_t nnz, const int32_t *d_row,
                                            const int32_t *d_col, const double *d_val,
                                            const double *d_d, const double *d_f,
                                            double *d_u, int k, void *stream) {
  clear_error();
  if (n <= 0 || !d_row || !d_col || !d_val || !d_d || !d_f || !d_u || k < 0)
    return set_error(BCMG_ERR_PARAM, "bad arguments");
  if (n > kNoAllocMaxRows)
    return set_error(BCMG_ERR_PARAM,
                     "bcmg_k_relax_noalloc handles at most %d rows (got %d); use "
                     "bcmg_k_relax for larger systems",
                     kNoAllocMaxRows, n);
  double *scratch = nullptr;
  BCMG_TRY(scratch_for_current_device(&scratch));
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  CsrView A;
  A.n = n;
  A.nnz = nnz;
  A.row = d_row;
  A.col = d_col;
  A.val = d_val;
  BCMG_TRY(relax_t<double>(mat_f64(A), d_d, d_f, d_u, scratch, k, false, s));
  BCMG_CUDA(cudaStreamSynchronize(s));
  return BCMG_OK;
}
