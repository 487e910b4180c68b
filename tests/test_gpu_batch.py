"""GPU tests of the multi-right-hand-side solve (bcmg_solve_batch).

Every column must solve exactly the problem bcmg_solve solves for it alone:
converged to rtol 1e-8 with the true FP64 relative residual at most
1.05 rtol, the solution within 1e-5 relative of the FP64 oracle's and of the
single-vector solve's (the batched kernels sum rows and dot products in a
different order, so last bits and at most a couple of iterations may differ).
The shape chosen by the autotuner must not change a single bit, and a batch
must be reproducible bit for bit.
"""
import numpy as np
import pytest

import bootcmatchg_b200 as bc
import workloads as wl
from helpers import c1_params
from oracle import oracle as orc

pytestmark = pytest.mark.gpu

TOL_X = 1e-5
ERR_PARAM = 1  # BCMG_ERR_PARAM


def rhs_block(n, seeds, zero_cols=()):
    B = np.zeros((n, len(seeds)), order="F")
    for j, s in enumerate(seeds):
        if j not in zero_cols:
            B[:, j] = wl.vector(1, s, n)
    return B


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def check_column(A, b, x, info, rtol, x0=None):
    """Converged to rtol relative to the initial residual ||b - A x0||."""
    if not b.any() and x0 is None:
        assert info.iters == 0 and info.converged and not x.any()
        return
    assert info.converged, info
    r0 = b if x0 is None else b - A.to_scipy() @ x0
    r = b - A.to_scipy() @ x
    assert np.linalg.norm(r) / np.linalg.norm(r0) <= 1.05 * rtol
    assert info.true_rel_residual <= 1.05 * rtol


@pytest.mark.parametrize("prec", [bc.PREC_FP64, bc.PREC_MIXED])
def test_batch_matches_oracle_and_single(prec):
    A = wl.poisson(7, 16, 16, 16)
    p = c1_params()
    B = rhs_block(A.n, [11, 12, 13, 14, 15], zero_cols=(3,))
    ext = bc.Extensions(precision=prec, replace_every=10 if prec == bc.PREC_MIXED else 0)
    with bc.Handle(A, p, ext) as h:
        X, infos = h.solve_batch(B)
        singles = [h.solve(B[:, j]) for j in range(B.shape[1])]
    o = orc.OracleHandle(A, p)
    for j in range(B.shape[1]):
        check_column(A, B[:, j], X[:, j], infos[j], p.rtol)
        xs, si = singles[j]
        if not B[:, j].any():
            assert si.iters == 0
            continue
        xo, oi, _ = o.solve(B[:, j])
        assert rel(X[:, j], xo) < TOL_X
        assert rel(X[:, j], xs) < TOL_X
        assert abs(infos[j].iters - si.iters) <= 2, (infos[j].iters, si.iters)
        assert abs(infos[j].iters - oi["iters"]) <= (2 if prec == bc.PREC_FP64 else 6)


@pytest.mark.parametrize("prec", [bc.PREC_FP64, bc.PREC_MIXED])
def test_autotune_does_not_change_bits(prec):
    A = wl.poisson(27, 14, 14, 14)
    p = c1_params()
    B = rhs_block(A.n, list(range(20, 28)))
    out = []
    for tune in (0, 1):
        ext = bc.Extensions(precision=prec, autotune=tune,
                            replace_every=8 if prec == bc.PREC_MIXED else 0)
        with bc.Handle(A, p, ext) as h:
            X, infos = h.solve_batch(B)
            cfg = [h.batch_config(B.shape[1], 0, l)
                   for l in range(h.hierarchy_info(0)["num_levels"])]
        out.append((X, [i.iters for i in infos], cfg))
    assert np.array_equal(out[0][0], out[1][0])
    assert out[0][1] == out[1][1]
    for c in out[0][2] + out[1][2]:
        assert c["width"] == 8
        assert c["cols_per_lane"] in (1, 2, 4) and c["threads"] in (128, 256)


def test_batch_is_reproducible_and_device_path_agrees():
    import torch
    A = wl.poisson(7, 18, 18, 18)
    p = c1_params()
    nrhs, ld = 6, A.n + 5
    B = rhs_block(A.n, list(range(40, 40 + nrhs)))
    with bc.Handle(A, p) as h:
        X1, i1 = h.solve_batch(B)
        X2, i2 = h.solve_batch(B)
        dev = torch.device("cuda:0")
        Bd = torch.zeros((nrhs, ld), dtype=torch.float64, device=dev)
        Bd[:, :A.n] = torch.from_numpy(np.ascontiguousarray(B.T)).to(dev)
        Xd = torch.zeros((nrhs, ld), dtype=torch.float64, device=dev)
        torch.cuda.synchronize()
        i3 = h.solve_batch_device(nrhs, Bd.data_ptr(), ld, Xd.data_ptr(), ld)
        X3 = Xd[:, :A.n].cpu().numpy().T
    assert np.array_equal(X1, X2)
    assert np.array_equal(X1, X3)
    assert [a.iters for a in i1] == [a.iters for a in i2] == [a.iters for a in i3]


def test_more_columns_than_one_group():
    A = wl.poisson(7, 12, 12, 12)
    p = c1_params()
    B = rhs_block(A.n, list(range(100, 140)))  # 32 + 8 (padded) columns
    with bc.Handle(A, p) as h:
        X, infos = h.solve_batch(B)
        for j in (0, 17, 31, 32, 39):
            xs, si = h.solve(B[:, j])
            assert rel(X[:, j], xs) < TOL_X
            assert abs(infos[j].iters - si.iters) <= 2
    for j in range(B.shape[1]):
        check_column(A, B[:, j], X[:, j], infos[j], p.rtol)


@pytest.mark.parametrize("solver_type", [0, 1, 2])
def test_batch_bootstrap_composites(solver_type):
    A = wl.fv2d(48, 48, seed=3)
    p = c1_params()
    p.max_hrc, p.conv_ratio, p.solver_type = 3, 0.1, solver_type
    B = rhs_block(A.n, [7, 8, 9])
    with bc.Handle(A, p) as h:
        assert h.num_hierarchies()[0] >= 2
        X, infos = h.solve_batch(B)
        for j in range(B.shape[1]):
            xs, si = h.solve(B[:, j])
            check_column(A, B[:, j], X[:, j], infos[j], p.rtol)
            assert rel(X[:, j], xs) < TOL_X
            assert abs(infos[j].iters - si.iters) <= 2


def test_batch_initial_guess_and_itnlim():
    A = wl.poisson(7, 14, 14, 14)
    p = c1_params()
    B = rhs_block(A.n, [3, 4])
    X0 = np.asfortranarray(np.stack([wl.vector(2, 5, A.n), np.zeros(A.n)], axis=1))
    with bc.Handle(A, p) as h:
        X, infos = h.solve_batch(B, X0)
        for j in range(2):
            xs, si = h.solve(B[:, j], X0[:, j])
            assert rel(X[:, j], xs) < TOL_X
            check_column(A, B[:, j], X[:, j], infos[j], p.rtol, X0[:, j])
    p.itnlim = 3
    with bc.Handle(A, p) as h:
        X, infos = h.solve_batch(B)
        xs, si = h.solve(B[:, 0])
    assert [i.iters for i in infos] == [si.iters, si.iters]
    assert not any(i.converged for i in infos)


def test_precond_apply_batch_matches_single():
    import torch
    A = wl.poisson(27, 12, 12, 12)
    p = c1_params()
    n, nrhs = A.n, 4
    dev = torch.device("cuda:0")
    R = torch.from_numpy(rhs_block(n, [61, 62, 63, 64]).T.copy()).to(dev)  # nrhs x n rows
    Z = torch.zeros_like(R)
    Zs = torch.zeros_like(R)
    with bc.Handle(A, p) as h:
        torch.cuda.synchronize()
        h.precond_apply_batch_device(nrhs, R.data_ptr(), n, Z.data_ptr(), n)
        for j in range(nrhs):
            h.precond_apply_device(R[j].data_ptr(), Zs[j].data_ptr())
        torch.cuda.synchronize()
    z, zs = Z.cpu().numpy(), Zs.cpu().numpy()
    for j in range(nrhs):
        assert rel(z[j], zs[j]) < 1e-12


def test_batch_errors():
    A = wl.poisson(7, 8, 8, 8)
    with bc.Handle(A, c1_params()) as h:
        B = np.zeros((A.n, 2))
        X = np.zeros((A.n, 2))
        st = bc.lib.bcmg_solve_batch(h.ptr, 0, B.ctypes.data, A.n, X.ctypes.data, A.n, 0, None)
        assert st == ERR_PARAM
        st = bc.lib.bcmg_solve_batch(h.ptr, 2, B.ctypes.data, A.n - 1, X.ctypes.data, A.n, 0,
                                     None)
        assert st == ERR_PARAM
