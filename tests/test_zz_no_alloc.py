"""bcmg_k_relax_noalloc: the smoother entry point for callers that cannot
allocate device memory where they call it (another framework's allocator owns
the device, a plugin with a fixed footprint, a latency-critical loop).  It
must give the same sweeps as bcmg_k_relax, which allocates its ping-pong
vector per call, on consecutive calls that reuse its process-lifetime buffer,
and reject systems larger than that buffer.  This file is collected last.
"""
import ctypes as C

import numpy as np
import pytest

import bootcmatchg_b200 as bc
import workloads as wl
from bootcmatchg_b200._lib import check, lib

pytestmark = pytest.mark.gpu

MAX_ROWS = 1 << 20


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
        check(lib.bcmg_k_relax_noalloc(A.n, A.nnz, P(row), P(col), P(val), P(dd), P(ff),
                                       P(ub), k, None), "bcmg_k_relax_noalloc")
        np.testing.assert_allclose(ub.cpu().numpy(), ua.cpu().numpy(), rtol=1e-13, atol=1e-13)


def test_noalloc_relax_rejects_oversized_systems():
    n = MAX_ROWS + 1
    dummy = C.c_void_p(8)  # never dereferenced: the size check comes first
    st = lib.bcmg_k_relax_noalloc(n, n, dummy, dummy, dummy, dummy, dummy, dummy, 1, None)
    assert bc.lib.bcmg_status_string(st) == b"BCMG_ERR_PARAM"
    assert b"at most" in lib.bcmg_last_error()
