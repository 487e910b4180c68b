"""bcmg_k_relax_noalloc: the smoother entry point for callers that cannot
allocate device memory where they call it (another framework's allocator owns
the device, a plugin with a fixed footprint, a latency-critical loop).  It
must give the same sweeps as bcmg_k_relax, which allocates its ping-pong
vector per call, on consecutive calls that reuse its process-lifetime buffer;
it must not allocate (neither through the library's allocator nor from the
device's stream-ordered memory pool); and it must reject systems larger than
that buffer.  This file is collected last.
"""
import ctypes as C

import numpy as np
import pytest

import bootcmatchg_b200 as bc
import workloads as wl
from bootcmatchg_b200._lib import check, lib

pytestmark = pytest.mark.gpu

MAX_ROWS = 1 << 20
USED_MEM_HIGH = 8  # cudaMemPoolAttrUsedMemHigh


def _cudart():
    import torch  # its CUDA runtime library is the one to bind
    import glob
    import os
    base = os.path.join(os.path.dirname(torch.__file__), "..", "nvidia", "cuda_runtime", "lib")
    found = sorted(glob.glob(os.path.join(base, "libcudart.so*")))
    return C.CDLL(found[0] if found else "libcudart.so")


def pool_used_high(rt, reset=False):
    """High watermark of memory in use from device 0's default pool (the pool
    cudaMallocAsync draws from); reset=True first sets it back to the memory
    in use now."""
    pool = C.c_void_p()
    assert rt.cudaDeviceGetDefaultMemPool(C.byref(pool), 0) == 0
    if reset:
        zero = C.c_uint64(0)
        assert rt.cudaMemPoolSetAttribute(pool, USED_MEM_HIGH, C.byref(zero)) == 0
    v = C.c_uint64()
    assert rt.cudaMemPoolGetAttribute(pool, USED_MEM_HIGH, C.byref(v)) == 0
    return v.value


def made_allocations():
    made = C.c_int64()
    lib.bcmg_debug_alloc_stats(None, C.byref(made))
    return made.value


def test_noalloc_relax_matches_allocating_relax_twice():
    import torch
    A = wl.poisson(27, 24, 22, 20)
    S = A.to_scipy()
    d = np.asarray(abs(S).sum(axis=1)).ravel()
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    P = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731
    row, col, val, dd = dev(A.row), dev(A.col), dev(A.val), dev(d)
    for call, k in enumerate((3, 4)):  # odd and even sweep counts, back to back
        f = wl.vector(1, 10 + call, A.n)
        u0 = wl.vector(2, 20 + call, A.n)
        ff = dev(f)
        ua, ub = dev(u0), dev(u0)
        check(lib.bcmg_k_relax(A.n, A.nnz, P(row), P(col), P(val), P(dd), P(ff), P(ua), k,
                               None), "bcmg_k_relax")
        torch.cuda.synchronize()
        rt = _cudart()
        high0 = pool_used_high(rt, reset=True)
        made0 = made_allocations()
        check(lib.bcmg_k_relax_noalloc(A.n, A.nnz, P(row), P(col), P(val), P(dd), P(ff),
                                       P(ub), k, None), "bcmg_k_relax_noalloc")
        assert made_allocations() == made0, "the no-alloc smoother allocated"
        assert pool_used_high(rt) == high0, "the no-alloc smoother drew from the memory pool"
        np.testing.assert_allclose(ub.cpu().numpy(), ua.cpu().numpy(), rtol=1e-13, atol=1e-13)


def test_noalloc_relax_rejects_oversized_systems():
    n = MAX_ROWS + 1
    dummy = C.c_void_p(8)  # never dereferenced: the size check comes first
    st = lib.bcmg_k_relax_noalloc(n, n, dummy, dummy, dummy, dummy, dummy, dummy, 1, None)
    assert bc.lib.bcmg_status_string(st) == b"BCMG_ERR_PARAM"
    assert b"at most" in lib.bcmg_last_error()
