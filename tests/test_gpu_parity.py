"""GPU parity tests: the CUDA path through the C ABI against the CPU oracle.

Bit-exact: matching (suitor array, symmetric matching), aggregates, coarse
index maps, prolongator values, Galerkin matrices, smooth vectors, D and M of
every level.  Matching weights W: equal up to the last-bit differences of the
device and host log (4 ulps).  Solve: x within 1e-6 relative of the oracle's
FP64 solution at rtol 1e-8, iteration counts within one, true FP64 residual
at most 1.05 rtol.
"""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest
import scipy.sparse as sp

import bootcmatchg_b200 as bc
import workloads as wl
from bootcmatchg_b200._lib import check, lib
from helpers import c1_params, random_sym_graph
from oracle import oracle as orc

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def P(t):
    return C.c_void_p(t.data_ptr())


def gpu_pair_aggregate(A, w):
    n = A.n
    row, col, val, wd = dev(A.row), dev(A.col), dev(A.val), dev(np.asarray(w, np.float64))
    agg = torch.empty(n, dtype=torch.int32, device="cuda")
    p = torch.empty(n, dtype=torch.float64, device="cuda")
    W = torch.empty(A.nnz, dtype=torch.float64, device="cuda")
    s = torch.empty(n, dtype=torch.int32, device="cuda")
    m = torch.empty(n, dtype=torch.int32, device="cuda")
    nc = C.c_int32()
    check(lib.bcmg_k_pair_aggregate(n, A.nnz, P(row), P(col), P(val), P(wd), P(agg), P(p),
                                    C.byref(nc), P(W), P(s), P(m), None), "pair_aggregate")
    return {"agg": agg.cpu().numpy(), "p": p.cpu().numpy(), "nc": nc.value,
            "W": W.cpu().numpy(), "suitor": s.cpu().numpy(), "match": m.cpu().numpy()}


def gpu_galerkin(A, agg, p, nc):
    row, col, val = dev(A.row), dev(A.col), dev(A.val)
    ag, pp = dev(np.asarray(agg, np.int32)), dev(np.asarray(p, np.float64))
    crow = torch.empty(nc + 1, dtype=torch.int32, device="cuda")
    cnnz = C.c_int32()
    check(lib.bcmg_k_galerkin(A.n, A.nnz, P(row), P(col), P(val), nc, P(ag), P(pp), P(crow),
                              C.byref(cnnz), None, None, None), "galerkin count")
    ccol = torch.empty(cnnz.value, dtype=torch.int32, device="cuda")
    cval = torch.empty(cnnz.value, dtype=torch.float64, device="cuda")
    check(lib.bcmg_k_galerkin(A.n, A.nnz, P(row), P(col), P(val), nc, P(ag), P(pp), P(crow),
                              C.byref(cnnz), P(ccol), P(cval), None), "galerkin fill")
    return crow.cpu().numpy(), ccol.cpu().numpy(), cval.cpu().numpy()


def asym(A, seed):
    rng = np.random.default_rng(seed)
    S = A.to_scipy().tocoo()
    off = S.row != S.col
    v = S.data.copy()
    v[off] *= rng.uniform(0.7, 1.3, off.sum())
    return bc.CsrMatrix.from_scipy(sp.coo_matrix((v, (S.row, S.col)), shape=S.shape).tocsr())


def star(n_leaves):
    """Hub joined to every leaf plus a ring: rows far longer than a warp team."""
    n = n_leaves + 1
    i = np.concatenate([np.zeros(n_leaves, int), np.arange(1, n)])
    j = np.concatenate([np.arange(1, n), np.r_[np.arange(2, n), 1]])
    off = sp.coo_matrix((-np.ones(i.shape[0]), (i, j)), shape=(n, n)).tocsr()
    off = off + off.T
    d = np.asarray(abs(off).sum(axis=1)).ravel() + 1.0
    return bc.CsrMatrix.from_scipy((off + sp.diags(d)).tocsr())


CASES = {
    "poisson7_16": lambda: (wl.poisson(7, 16, 16, 16), None),
    "poisson27_10": lambda: (wl.poisson(27, 10, 10, 10), None),
    "poisson5_40": lambda: (wl.poisson(5, 40, 40), None),
    "fv2d_64": lambda: (wl.fv2d(64, 64, seed=2), None),
    "rgg_20000": lambda: (wl.rgg(20000, seed=4), None),
    "rand_int_ties": lambda: (random_sym_graph(5000, 8, seed=3, int_weights=True), None),
    "rand_float_w": lambda: (random_sym_graph(5000, 8, seed=4, int_weights=False),
                             wl.vector(1, 9, 5000)),
    "asymmetric": lambda: (asym(random_sym_graph(4000, 8, seed=6, int_weights=False), 1),
                           None),
    "zero_w_entries": lambda: (random_sym_graph(3000, 6, seed=8, int_weights=False),
                               np.where(np.arange(3000) % 13 == 0, 0.0, 1.0)),
    "star_long_rows": lambda: (star(700), None),
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_pair_aggregate_parity(case):
    A, w = CASES[case]()
    if w is None:
        w = np.ones(A.n)
    g = gpu_pair_aggregate(A, w)
    o = orc.pair_aggregate(A, w)
    np.testing.assert_allclose(g["W"], o["W"], rtol=4 * 2.0 ** -52, atol=0)
    assert np.array_equal(g["suitor"], o["suitor"]), "suitor arrays differ"
    assert np.array_equal(g["match"], o["match"]), "matchings differ"
    assert g["nc"] == o["nc"]
    assert np.array_equal(g["agg"], o["agg"]), "coarse index maps differ"
    assert np.array_equal(g["p"], o["p"]), "prolongator values differ"


@pytest.mark.parametrize("case", sorted(CASES))
def test_galerkin_parity(case):
    A, w = CASES[case]()
    if w is None:
        w = np.ones(A.n)
    o = orc.pair_aggregate(A, w)
    go = gpu_galerkin(A, o["agg"], o["p"], o["nc"])
    oo = orc.galerkin(A, o["agg"], o["p"], o["nc"])
    for a, b, name in zip(go, oo, ("row", "col", "val")):
        assert np.array_equal(a, b), f"Galerkin {name} differs"


def test_relax_and_spmv_parity():
    A = wl.poisson(27, 12, 11, 10)
    S = A.to_scipy()
    d = np.asarray(abs(S).sum(axis=1)).ravel()
    f, u0 = wl.vector(1, 1, A.n), wl.vector(2, 2, A.n)
    row, col, val = dev(A.row), dev(A.col), dev(A.val)
    dd, ff, uu = dev(d), dev(f), dev(u0)
    for k in (1, 2, 3):
        uu.copy_(dev(u0))
        check(lib.bcmg_k_relax(A.n, A.nnz, P(row), P(col), P(val), P(dd), P(ff), P(uu), k,
                               None), "relax")
        np.testing.assert_allclose(uu.cpu().numpy(), orc.relax(A, d, f, u0, k), rtol=1e-13,
                                   atol=1e-13)
    x, y0 = wl.vector(1, 3, A.n), wl.vector(1, 4, A.n)
    xx, yy = dev(x), dev(y0)
    check(lib.bcmg_k_spmv(A.n, A.nnz, P(row), P(col), P(val), 2.0, P(xx), -0.5, P(yy), None),
          "spmv")
    np.testing.assert_allclose(yy.cpu().numpy(), 2.0 * (S @ x) - 0.5 * y0, rtol=1e-13,
                               atol=1e-12)


def compare_hierarchies(h, o, hrc=0, ohrc=None):
    ohrc = hrc if ohrc is None else ohrc
    gi, oi = h.hierarchy_info(hrc), o.hierarchy_info(ohrc)
    assert gi["num_levels"] == oi["num_levels"], (gi, oi)
    for l in range(gi["num_levels"]):
        g, r = h.level(hrc, l), o.level(ohrc, l)
        assert (g.n, g.nnz, g.n_coarse) == (r["n"], r["nnz"], r["n_coarse"]), l
        for name, a, b in (("row", g.A.row, r["row"]), ("col", g.A.col, r["col"]),
                           ("val", g.A.val, r["val"]), ("D", g.D, r["D"]), ("M", g.M, r["M"]),
                           ("w", g.w, r["w"])):
            assert np.array_equal(a, b), f"level {l}: {name} differs"
        if g.n_coarse:
            assert np.array_equal(g.agg, r["agg"]), f"level {l}: agg differs"
            assert np.array_equal(g.p, r["p"]), f"level {l}: p differs"
    assert gi["op_cmplx"] == oi["op_cmplx"]


HIER_CASES = {
    "poisson7_32": lambda: wl.poisson(7, 32, 32, 32),
    "poisson27_20": lambda: wl.poisson(27, 20, 20, 20),
    "fv2d_128": lambda: wl.fv2d(128, 128, seed=2),
    "rgg_30000": lambda: wl.rgg(30000, seed=11),
}


@pytest.mark.parametrize("case", sorted(HIER_CASES))
def test_hierarchy_and_solve_parity(case):
    A = HIER_CASES[case]()
    p = c1_params()
    b = wl.vector(1, 1, A.n)
    with bc.Handle(A, p) as h:
        o = orc.OracleHandle(A, p)
        compare_hierarchies(h, o)
        x, info = h.solve(b)
    xo, oi, st = o.solve(b)
    assert st == 0 and oi["converged"] and info.converged
    assert abs(info.iters - oi["iters"]) <= 1, (info.iters, oi["iters"])
    assert np.linalg.norm(x - xo) / np.linalg.norm(xo) < 1e-6
    r = b - A.to_scipy() @ x
    assert np.linalg.norm(r) / np.linalg.norm(b) <= 1.05 * p.rtol
    assert info.true_rel_residual <= 1.05 * p.rtol


@pytest.mark.parametrize("solver_type", [0, 1, 2])
@pytest.mark.parametrize("cycle_type", [0, 1, 2])
def test_bootstrap_composites_cycles(solver_type, cycle_type):
    A = wl.fv2d(64, 64, seed=2)
    p = c1_params()
    p.solver_type, p.cycle_type, p.max_hrc, p.conv_ratio = solver_type, cycle_type, 3, 0.1
    p.relax_type, p.coarse_solver = 0, 4
    b = wl.vector(2, 2, A.n)
    with bc.Handle(A, p) as h:
        o = orc.OracleHandle(A, p)
        nh, est = h.num_hierarchies()
        onh, oest = o.num_hierarchies()
        assert nh == onh == 3
        assert abs(est - oest) <= 1e-9 * abs(oest)
        # Hierarchies 1 and 2 come from w = 1: bit-exact.  Hierarchy 3 comes
        # from the w of 15 composite cycles, whose sums round differently on
        # the GPU: w within 1e-10, and the hierarchy bit-exact when the oracle
        # coarsens from the GPU's w.
        compare_hierarchies(h, o, 0)
        compare_hierarchies(h, o, 1)
        gw = h.level(2, 0).w
        np.testing.assert_allclose(gw, o.level(2, 0)["w"], rtol=1e-10,
                                   atol=1e-12 * np.abs(gw).max())
        compare_hierarchies(h, orc.OracleHandle(A, p, w=gw), 2, 0)
        # one preconditioner application from a nonzero guess
        r0, z0 = wl.vector(1, 5, A.n), wl.vector(1, 6, A.n)
        rt, zt = dev(r0), dev(z0)
        h.precond_apply_device(rt.data_ptr(), zt.data_ptr())
        zo = o.precond_apply(r0, z0)
        np.testing.assert_allclose(zt.cpu().numpy(), zo, rtol=1e-10,
                                   atol=1e-12 * np.abs(zo).max())
        x, info = h.solve(b)
    xo, oi, st = o.solve(b)
    assert info.converged and abs(info.iters - oi["iters"]) <= 1
    assert np.linalg.norm(x - xo) / np.linalg.norm(xo) < 1e-6


def test_setup_is_deterministic():
    A = wl.rgg(20000, seed=3)
    p = c1_params()
    with bc.Handle(A, p) as h1, bc.Handle(A, p) as h2:
        L = h1.hierarchy_info()["num_levels"]
        assert h2.hierarchy_info()["num_levels"] == L
        for l in range(L):
            a, b = h1.level(0, l), h2.level(0, l)
            assert np.array_equal(a.A.val, b.A.val) and np.array_equal(a.A.col, b.A.col)
        x1, _ = h1.solve(np.ones(A.n))
        x2, _ = h2.solve(np.ones(A.n))
        assert np.array_equal(x1, x2)


def test_edge_cases():
    p = c1_params()
    # 1x1 system
    A = bc.CsrMatrix(1, np.array([0, 1]), np.array([0]), np.array([4.0]))
    x, info = bc.solve(A, p, np.array([2.0]))
    assert abs(x[0] - 0.5) < 1e-14
    # diagonal matrix: no edges, every vertex a singleton aggregate
    n = 50
    D = bc.CsrMatrix(n, np.arange(n + 1), np.arange(n), np.linspace(1, 2, n))
    x, info = bc.solve(D, p, np.ones(n))
    np.testing.assert_allclose(x, 1 / np.linspace(1, 2, n), rtol=1e-12)
    # zero right-hand side: already converged
    B = wl.poisson(7, 8, 8, 8)
    x, info = bc.solve(B, p, np.zeros(B.n))
    assert info.iters == 0 and np.all(x == 0)


def test_errors():
    p = c1_params()
    bad = bc.CsrMatrix(2, np.array([0, 1, 2]), np.array([1, 0]), np.array([1.0, 1.0]))
    with pytest.raises(bc.BcmgError, match="INVALID_MATRIX"):
        bc.Handle(bad, p)


def test_cli_matches_reference_format(tmp_path):
    A = wl.poisson(7, 10, 10, 10)
    mtx = tmp_path / "a.mtx"
    bc.write_matrix_mm(str(mtx), A)
    settings = tmp_path / "settings"
    settings.write_text("0 % solver_type\n1 % max_hrc\n0.8 % rho\n2 % aggr_sweeps\n"
                        "0 % aggr_type\n20 % max_levels\n0 % cycle_type\n4 % coarse\n"
                        "4 % relax\n16 % coarse sweeps\n4 % pre\n4 % post\n1000 % itnlim\n"
                        "1.e-8 % rtol\n")
    cli = os.path.join(os.path.dirname(bc.LIB_PATH), "bcmg_cli")
    out = subprocess.run([cli, str(mtx), str(settings), str(tmp_path / "x.txt")],
                         capture_output=True, text=True, check=True)
    assert "#META sol;num_iteration int" in out.stdout
    lines = (tmp_path / "x.txt").read_text().splitlines()
    assert len(lines) == A.n and all("e" in s for s in lines[:3])
    x = np.array([float(s) for s in lines])
    xo, _, _ = orc.OracleHandle(A, bc.Params.init_from_file(str(settings))).solve(np.ones(A.n))
    assert np.linalg.norm(x - xo) / np.linalg.norm(xo) < 1e-6


@pytest.mark.parametrize("prec", [bc.PREC_FP64, bc.PREC_MIXED])
def test_kcycle_matches_oracle(prec):
    """cycle_type 3 (K-cycle, GAMG_cycle.cu:88-100 + inneritkcycle,
    FCG.cu:633-723) on the GPU against the oracle's: same hierarchy, the
    solution within 1e-6 and the outer iteration count within one.  The FCG
    loop with the K-cycle runs as a captured graph (inner scalars on the
    device, the second inner step an IF node): a repeated solve launches a
    fraction of the host-driven loop's kernels and gives the host-driven
    solution (same iterations, within 1e-10).  Batched solves refuse the
    K-cycle."""
    from bootcmatchg_b200._lib import lib
    A = wl.poisson(27, 20, 20, 20)
    p = c1_params()
    p.cycle_type = 3
    b = wl.vector(1, 11, A.n)
    ext = bc.Extensions(precision=prec, replace_every=10 if prec else 0)
    with bc.Handle(A, p, ext) as h:
        x, info = h.solve(b)
        n0 = lib.bcmg_kernel_launches()
        x2, info2 = h.solve(b)
        graph_launches = lib.bcmg_kernel_launches() - n0
        with pytest.raises(bc.BcmgError, match="UNSUPPORTED"):
            h.solve_batch(np.asfortranarray(np.stack([b, b], axis=1)))
    ext_host = bc.Extensions(precision=prec, replace_every=10 if prec else 0, use_graphs=0)
    with bc.Handle(A, p, ext_host) as hh:
        n0 = lib.bcmg_kernel_launches()
        xh, ih = hh.solve(b)
        host_launches = lib.bcmg_kernel_launches() - n0
    assert info2.iters == info.iters and np.array_equal(x2, x)
    assert ih.iters == info.iters, (ih.iters, info.iters)
    assert np.linalg.norm(xh - x) / np.linalg.norm(xh) < 1e-10
    assert graph_launches * 3 < host_launches, (graph_launches, host_launches)
    o = orc.OracleHandle(A, p)
    xo, oi, st = o.solve(b)
    assert st == 0 and oi["converged"] and info.converged
    assert abs(info.iters - oi["iters"]) <= 1
    assert np.linalg.norm(x - xo) / np.linalg.norm(xo) < 1e-6
    assert info.true_rel_residual <= 1.05 * p.rtol


def test_hierarchy_file_roundtrip(tmp_path):
    """bcmg_save / bcmg_load: the loaded handle has the same levels bit for bit
    and solves to the same bits; a hierarchy saved from an FP64 setup also
    loads for mixed-precision solves."""
    A = wl.fv2d(64, 64, seed=2)
    p = c1_params()
    p.max_hrc, p.conv_ratio, p.solver_type = 2, 0.1, 0
    b = wl.vector(2, 4, A.n)
    path = tmp_path / "h.bcmg"
    with bc.Handle(A, p) as h:
        x0, i0 = h.solve(b)
        nh0 = h.num_hierarchies()[0]
        info0 = h.hierarchy_info(nh0 - 1)
        lv0 = h.level(nh0 - 1, 1)
        h.save(path)
    with bc.Handle.load(path) as h2:
        assert h2.num_hierarchies()[0] == nh0
        assert h2.params.max_hrc == 2
        lv = h2.level(nh0 - 1, 1)
        assert h2.hierarchy_info(nh0 - 1)["num_levels"] == info0["num_levels"]
        for a, b_ in ((lv.A.val, lv0.A.val), (lv.A.col, lv0.A.col), (lv.D, lv0.D),
                      (lv.agg, lv0.agg), (lv.p, lv0.p)):
            assert np.array_equal(a, b_)
        x1, i1 = h2.solve(b)
    assert i1.iters == i0.iters and np.array_equal(x1, x0)
    ext = bc.Extensions(precision=bc.PREC_MIXED, replace_every=10)
    with bc.Handle.load(path, ext) as h3:
        x2, i2 = h3.solve(b)
    assert i2.converged and np.linalg.norm(x2 - x0) / np.linalg.norm(x0) < 1e-6


def test_hierarchy_file_roundtrip_smoothed(tmp_path):
    """Hierarchy files with smoothed aggregation (aggrtype 1): the file also
    holds every level's smoothed prolongator; the loaded handle has the same
    coarse matrices bit for bit and solves to the same bits in FP64, and the
    same file serves a mixed-precision solve."""
    A = wl.poisson(27, 12, 12, 12)
    p = c1_params()
    p.aggrtype = 1
    b = wl.vector(1, 9, A.n)
    path = tmp_path / "sa.bcmg"
    with bc.Handle(A, p) as h:
        x0, i0 = h.solve(b)
        nl = h.hierarchy_info(0)["num_levels"]
        lv0 = [h.level(0, l) for l in range(nl)]
        h.save(path)
    with bc.Handle.load(path) as h2:
        assert h2.params.aggrtype == 1
        assert h2.hierarchy_info(0)["num_levels"] == nl
        for l in range(nl):
            lv = h2.level(0, l)
            for a, b_ in ((lv.A.row, lv0[l].A.row), (lv.A.col, lv0[l].A.col),
                          (lv.A.val, lv0[l].A.val), (lv.D, lv0[l].D), (lv.M, lv0[l].M)):
                assert np.array_equal(a, b_)
        x1, i1 = h2.solve(b)
    assert i0.converged and i1.iters == i0.iters and np.array_equal(x1, x0)
    ext = bc.Extensions(precision=bc.PREC_MIXED, replace_every=10)
    with bc.Handle.load(path, ext) as h3:
        x2, i2 = h3.solve(b)
    assert i2.converged and np.linalg.norm(x2 - x0) / np.linalg.norm(x0) < 1e-6


SMOOTHED_CASES = {
    "poisson7_20": lambda: wl.poisson(7, 20, 20, 20),
    "poisson27_12": lambda: wl.poisson(27, 12, 12, 12),
    "fv2d_64": lambda: wl.fv2d(64, 64, seed=2),
    "rgg_20000": lambda: wl.rgg(20000, seed=11),
}


@pytest.mark.parametrize("case", sorted(SMOOTHED_CASES))
def test_smoothed_aggregation_matches_oracle(case):
    """aggrtype 1 (matchingAggregation.cu:353-390): the smoothed coarse
    matrices, their D and M, and the operator complexity bit for bit against
    the oracle's (the products sum in the same canonical order); FP64 and
    mixed solves within 1e-6 of the oracle's solution, iterations within one.
    A batched solve of two right-hand sides (the smoothed P and R applied to
    both columns at once) converges on both, its first column within 1e-5 of
    the oracle's solution (the batched kernels sum in another order)."""
    A = SMOOTHED_CASES[case]()
    p = c1_params()
    p.aggrtype = 1
    b = wl.vector(1, 7, A.n)
    o = orc.OracleHandle(A, p)
    xo, oi, st = o.solve(b)
    assert st == 0 and oi["converged"]
    B2 = np.asfortranarray(np.stack([b, wl.vector(1, 8, A.n)], axis=1))
    for prec in (bc.PREC_FP64, bc.PREC_MIXED):
        ext = bc.Extensions(precision=prec, replace_every=10 if prec else 0)
        with bc.Handle(A, p, ext) as h:
            compare_hierarchies(h, o)
            x, info = h.solve(b)
            Xb, ib = h.solve_batch(B2)
        assert info.converged and abs(info.iters - oi["iters"]) <= 1, (info.iters, oi["iters"])
        assert np.linalg.norm(x - xo) / np.linalg.norm(xo) < 1e-6
        assert info.true_rel_residual <= 1.05 * p.rtol
        for j in range(2):
            assert ib[j].converged and ib[j].true_rel_residual <= 1.05 * p.rtol, ib[j]
        assert abs(ib[0].iters - oi["iters"]) <= 2, (ib[0].iters, oi["iters"])
        assert np.linalg.norm(Xb[:, 0] - xo) / np.linalg.norm(xo) < 1e-5


def test_spgemm_tiers_match_oracle():
    """bcmg_k_spgemm bit for bit against the oracle's canonical-order product,
    with product rows in every tier of the kernel: up to 512 distinct
    columns (a warp, shared memory), up to 2,048 (a block, shared memory)
    and beyond (a block, global memory), plus empty and one-entry rows."""
    from test_cpu_oracle import rows_with_lengths
    rng = np.random.default_rng(8)
    lengths = rng.choice([0, 1, 10, 60, 300], size=240, p=[0.05, 0.05, 0.3, 0.3, 0.3])
    X = rows_with_lengths(lengths, 4000, 9)
    Y = rows_with_lengths([25] * 4000, 6000, 10)
    crow_o, ccol_o, cval_o = orc.spgemm(X, Y, 6000)
    assert np.diff(crow_o).max() > 2048 and np.diff(crow_o).min() == 0
    xr, xc, xv = dev(X.row), dev(X.col), dev(X.val)
    yr, yc, yv = dev(Y.row), dev(Y.col), dev(Y.val)
    crow = torch.zeros(X.n + 1, dtype=torch.int32, device="cuda")
    nnz = C.c_int32()
    args = (X.n, 6000, X.nnz, P(xr), P(xc), P(xv), Y.n, Y.nnz, P(yr), P(yc), P(yv), P(crow),
            C.byref(nnz))
    check(lib.bcmg_k_spgemm(*args, None, None, None), "spgemm")
    ccol = torch.zeros(nnz.value, dtype=torch.int32, device="cuda")
    cval = torch.zeros(nnz.value, dtype=torch.float64, device="cuda")
    check(lib.bcmg_k_spgemm(*args, P(ccol), P(cval), None), "spgemm")
    assert np.array_equal(crow.cpu().numpy(), crow_o)
    assert np.array_equal(ccol.cpu().numpy(), ccol_o)
    assert np.array_equal(cval.cpu().numpy(), cval_o)
