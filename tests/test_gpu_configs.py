"""Parity at the benchmark workloads' own sizes, and mixed precision at the
FP64 tolerance.

27-point Poisson 128^3 (2,097,152 rows, 55,742,968 nonzeros) and 7-point
Poisson 32^3 (b = 1) and 96^3: every level of the GPU hierarchy -- row
pointers, columns, values, D, M, the smooth vector w, aggregates and
prolongator values -- equal bit for bit to the CPU oracle's.  Solves to rtol
1e-8 from x0 = 0: the true FP64 relative residual at most 1.05 rtol, the
solution within 1e-6 relative of the oracle's FP64 solution of the same
PCG + AMG, iteration counts within one of the oracle's (FP64 path) or six
(mixed-precision cycle, an inexact preconditioner that flexible CG absorbs).

Residual replacement at rtol 1e-10: the mixed-precision path (FP32 cycle,
FP32 or BF16 coarse storage, FP64 FCG) on a 27-point and an anisotropic FV
matrix reaches a true FP64 relative residual of at most 1.05e-10, and its
solution is within 1e-8 relative of the oracle's solution at the same
tolerance.
"""
import numpy as np
import pytest

import bootcmatchg_b200 as bc
import workloads as wl
from helpers import c1_params
from oracle import oracle as orc
from test_gpu_parity import compare_hierarchies

pytestmark = pytest.mark.gpu


def check_solution(A, b, x, info, xo, oi, rtol, err_tol, iter_slack):
    assert info.converged and oi["converged"]
    r = b - A.to_scipy() @ x
    assert np.linalg.norm(r) / np.linalg.norm(b) <= 1.05 * rtol
    assert info.true_rel_residual <= 1.05 * rtol
    err = np.linalg.norm(x - xo) / np.linalg.norm(xo)
    assert err < err_tol, err
    assert abs(info.iters - oi["iters"]) <= iter_slack, (info.iters, oi["iters"])
    return err


def test_poisson27_128_hierarchy_and_solves():
    """27-point Poisson 128^3, b ~ N(0,1) seed 1 (the headline workload)."""
    A = wl.poisson(27, 128, 128, 128)
    b = wl.vector(1, 1, A.n)
    p = c1_params()
    o = orc.OracleHandle(A, p)
    with bc.Handle(A, p) as h:
        compare_hierarchies(h, o)
        x, info = h.solve(b)
    xo, oi, st = o.solve(b)
    assert st == 0
    check_solution(A, b, x, info, xo, oi, p.rtol, 1e-6, 1)
    ext = bc.Extensions(precision=bc.PREC_MIXED, replace_every=10)
    with bc.Handle(A, p, ext) as h:
        lv = h.level(0, 1)
        assert np.array_equal(lv.A.val, o.level(0, 1)["val"])  # setup stays FP64
        x, info = h.solve(b)
    check_solution(A, b, x, info, xo, oi, p.rtol, 1e-6, 6)
    o.close()


@pytest.mark.parametrize("case", ["poisson7_32_ones", "poisson7_96"])
def test_poisson7_hierarchy_and_solve(case):
    """7-point Poisson 32^3 with b = 1 and 96^3 with b ~ N(0,1) seed 3."""
    if case == "poisson7_32_ones":
        A = wl.poisson(7, 32, 32, 32)
        b = np.ones(A.n)
    else:
        A = wl.poisson(7, 96, 96, 96)
        b = wl.vector(1, 3, A.n)
    p = c1_params()
    o = orc.OracleHandle(A, p)
    with bc.Handle(A, p) as h:
        compare_hierarchies(h, o)
        x, info = h.solve(b)
    xo, oi, st = o.solve(b)
    assert st == 0
    check_solution(A, b, x, info, xo, oi, p.rtol, 1e-6, 1)
    with bc.Handle(A, p, bc.Extensions(precision=bc.PREC_MIXED, replace_every=10)) as h:
        x, info = h.solve(b)
    check_solution(A, b, x, info, xo, oi, p.rtol, 1e-6, 6)


@pytest.mark.parametrize("case", ["poisson27_64", "fv2d_512"])
def test_mixed_residual_replacement_reaches_1e10(case):
    if case == "poisson27_64":
        A = wl.poisson(27, 64, 64, 64)
        b = wl.vector(1, 1, A.n)
        storage = bc.STORE_FP32
    else:
        A = wl.fv2d(512, 512, seed=2)
        b = wl.vector(2, 2, A.n)
        storage = bc.STORE_BF16
    p = c1_params()
    p.rtol = 1e-10
    o = orc.OracleHandle(A, p)
    xo, oi, st = o.solve(b)
    assert st == 0
    ext = bc.Extensions(precision=bc.PREC_MIXED, coarse_storage=storage, replace_every=10)
    with bc.Handle(A, p, ext) as h:
        x, info = h.solve(b)
    check_solution(A, b, x, info, xo, oi, p.rtol, 1e-8, 8)
