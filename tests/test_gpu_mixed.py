"""GPU tests of the mixed-precision cycle and the graph-captured FCG loop.

Mixed precision: FP32 cycle (level 0 FP32, coarse levels FP32/BF16/FP16),
FP64 FCG with residual replacement.  Tolerance: the true FP64 relative
residual at most 1.05 rtol (rtol 1e-8) and the solution within 1e-6 relative
of the FP64 oracle's.  The hierarchy itself is built in FP64 and must stay
bit-identical to the oracle's in every precision mode.
"""
import numpy as np
import pytest

import bootcmatchg_b200 as bc
import workloads as wl
from helpers import c1_params
from oracle import oracle as orc

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("storage", [bc.STORE_FP32, bc.STORE_BF16, bc.STORE_FP16])
@pytest.mark.parametrize("case", ["poisson27_24", "fv2d_96"])
def test_mixed_solve_meets_fp64_tolerance(case, storage):
    A = wl.poisson(27, 24, 24, 24) if case == "poisson27_24" else wl.fv2d(96, 96, seed=2)
    p = c1_params()
    b = wl.vector(1, 1, A.n)
    ext = bc.Extensions(precision=bc.PREC_MIXED, coarse_storage=storage, replace_every=10)
    with bc.Handle(A, p, ext) as h:
        x, info = h.solve(b)
        lv = h.level(0, 1)
    o = orc.OracleHandle(A, p)
    olv = o.level(0, 1)
    assert np.array_equal(lv.A.val, olv["val"])  # setup stays FP64 and exact
    xo, oi, _ = o.solve(b)
    assert info.converged
    r = b - A.to_scipy() @ x
    assert np.linalg.norm(r) / np.linalg.norm(b) <= 1.05 * p.rtol
    assert info.true_rel_residual <= 1.05 * p.rtol
    assert np.linalg.norm(x - xo) / np.linalg.norm(xo) < 1e-6
    assert info.iters <= oi["iters"] + 6


def test_mixed_bootstrap_composite():
    A = wl.fv2d(80, 80, seed=2)
    p = c1_params()
    p.max_hrc, p.conv_ratio, p.solver_type = 3, 0.1, 1
    b = wl.vector(2, 2, A.n)
    ext = bc.Extensions(precision=bc.PREC_MIXED, replace_every=5)
    with bc.Handle(A, p, ext) as h, bc.Handle(A, p) as h64:
        assert h.num_hierarchies() == h64.num_hierarchies()
        x, info = h.solve(b)
        x64, info64 = h64.solve(b)
    assert info.converged and info.true_rel_residual <= 1.05 * p.rtol
    assert np.linalg.norm(x - x64) / np.linalg.norm(x64) < 1e-6


@pytest.mark.parametrize("prec", [bc.PREC_FP64, bc.PREC_MIXED])
def test_graph_loop_equals_host_loop(prec):
    A = wl.poisson(7, 20, 20, 20)
    p = c1_params()
    b = wl.vector(1, 4, A.n)
    e1 = bc.Extensions(precision=prec, use_graphs=1, replace_every=7 if prec else 0)
    e0 = bc.Extensions(precision=prec, use_graphs=0, replace_every=7 if prec else 0)
    with bc.Handle(A, p, e1) as h1, bc.Handle(A, p, e0) as h0:
        x1, i1 = h1.solve(b)
        x0, i0 = h0.solve(b)
        x1b, i1b = h1.solve(b)  # second solve reuses the captured graph
    assert i1.iters == i0.iters == i1b.iters
    assert np.array_equal(x1, x0) and np.array_equal(x1, x1b)


def test_itnlim_respected():
    A = wl.poisson(7, 16, 16, 16)
    p = c1_params()
    p.itnlim, p.rtol = 3, 1e-14
    with bc.Handle(A, p) as h:
        x, info = h.solve(np.ones(A.n))
    assert info.iters == 4 and not info.converged  # num_iter = iter + 1


@pytest.mark.parametrize("case", ["poisson27_20", "rgg_20000"])
def test_sliced_level_relax_matches_oracle(case):
    """Sweeps on the sliced copies (offset slices on the stencil level 0,
    explicit-column slices on coarse / irregular levels) against the oracle's
    CSR sweep, FP64."""
    import ctypes as C
    import torch
    from bootcmatchg_b200._lib import check, lib
    A = wl.poisson(27, 20, 20, 20) if case == "poisson27_20" else wl.rgg(20000, seed=3)
    p = c1_params()
    with bc.Handle(A, p) as h:
        L = h.hierarchy_info()["num_levels"]
        for level in range(min(3, L)):
            lv = h.level(0, level)
            f, u0 = wl.vector(1, level + 1, lv.n), wl.vector(2, level + 2, lv.n)
            ft = torch.from_numpy(f).cuda()
            ut = torch.from_numpy(u0).cuda()
            check(lib.bcmg_level_relax(h.ptr, 0, level, C.c_void_p(ft.data_ptr()),
                                       C.c_void_p(ut.data_ptr()), 3), "level_relax")
            d = lv.M if (level < L - 1 or p.coarse_solver == 4) else lv.D
            ref = orc.relax(lv.A, d, f, u0, 3)
            np.testing.assert_allclose(ut.cpu().numpy(), ref, rtol=1e-12,
                                       atol=1e-12 * np.abs(ref).max())


def test_sliced_and_csr_solves_agree():
    A = wl.rgg(30000, seed=2)
    p = c1_params()
    b = wl.vector(1, 8, A.n)
    with bc.Handle(A, p, bc.Extensions(sliced=1)) as h1, \
            bc.Handle(A, p, bc.Extensions(sliced=0)) as h0:
        x1, i1 = h1.solve(b)
        x0, i0 = h0.solve(b)
    assert abs(i1.iters - i0.iters) <= 1
    assert np.linalg.norm(x1 - x0) / np.linalg.norm(x0) < 1e-7


@pytest.mark.parametrize("prec", [bc.PREC_FP64, bc.PREC_MIXED])
def test_exact_value_narrowing_is_bit_identical(prec):
    """Solve-phase copies (the FP64 or FP32 cycle, and the FCG SpMV in both
    modes) store a level's values in BF16 when every value converts exactly
    (the 27-point stencil's 26 and -1); the kernels widen them, so the
    solution matches the unnarrowed run bit for bit."""
    import ctypes as C
    from bootcmatchg_b200._lib import check, lib
    A = wl.poisson(27, 32, 32, 32)
    p = c1_params()
    b = wl.vector(1, 5, A.n)
    out = []
    for narrow in (1, 0):
        ext = bc.Extensions(precision=prec, replace_every=10 if prec else 0,
                            narrow_values=narrow)
        with bc.Handle(A, p, ext) as h:
            x, info = h.solve(b)
            slots, cslots = C.c_int64(), C.c_int64()
            nsl, vb = C.c_int32(), C.c_int32()
            check(lib.bcmg_level_format(h.ptr, 0, 0, C.byref(slots), C.byref(cslots),
                                        C.byref(nsl), C.byref(vb)), "level_format")
        assert info.converged
        out.append((x, info.iters, vb.value))
    assert out[0][2] == 2
    assert out[1][2] == (4 if prec == bc.PREC_MIXED else 8)
    assert out[0][1] == out[1][1]
    assert np.array_equal(out[0][0], out[1][0])


@pytest.mark.parametrize("prec", [bc.PREC_FP64, bc.PREC_MIXED])
@pytest.mark.parametrize("case", ["poisson27_48", "rgg_20000", "fv2d_128"])
def test_fused_sweeps_equal_single_sweeps(case, prec):
    """k sweeps in one call (one launch on levels small enough for a
    thread-block cluster, whose iterate stays in distributed shared memory)
    give the bits of k calls of one sweep each, on every level."""
    import ctypes as C
    import torch
    from bootcmatchg_b200._lib import check, lib
    A = {"poisson27_48": lambda: wl.poisson(27, 48, 48, 48),
         "rgg_20000": lambda: wl.rgg(20000, seed=3),
         "fv2d_128": lambda: wl.fv2d(128, 128, seed=2)}[case]()
    dt = torch.float32 if prec == bc.PREC_MIXED else torch.float64
    ext = bc.Extensions(precision=prec, replace_every=10 if prec else 0)
    with bc.Handle(A, c1_params(), ext) as h:
        for level in range(h.hierarchy_info()["num_levels"]):
            n = h.level(0, level).n
            g = torch.Generator(device="cuda").manual_seed(level)
            f = torch.randn(n, dtype=dt, device="cuda", generator=g)
            u0 = torch.randn(n, dtype=dt, device="cuda", generator=g)
            for k in (2, 5, 16):
                ua, ub = u0.clone(), u0.clone()
                check(lib.bcmg_level_relax(h.ptr, 0, level, C.c_void_p(f.data_ptr()),
                                           C.c_void_p(ua.data_ptr()), k), "k sweeps")
                for _ in range(k):
                    check(lib.bcmg_level_relax(h.ptr, 0, level, C.c_void_p(f.data_ptr()),
                                               C.c_void_p(ub.data_ptr()), 1), "one sweep")
                assert torch.equal(ua, ub), (level, k)
