"""Shared helpers for the test suite (workload settings, random inputs)."""
import numpy as np


def c1_params():
    """Settings of the 7-point Poisson 32^3 workload (single hierarchy,
    aggrsweeps 2, unsmoothed, V-cycle, l1 smoother 4/4, 16 coarse sweeps,
    itnlim 1000, rtol 1e-8)."""
    import bootcmatchg_b200 as bc
    p = bc.Params.default()
    p.solver_type, p.max_hrc, p.conv_ratio = 0, 1, 0.8
    p.aggrsweeps, p.aggrtype, p.max_levels, p.cycle_type = 2, 0, 20, 0
    p.relax_type, p.coarse_solver = 4, 4
    p.prerelax_sweeps, p.postrelax_sweeps, p.relaxnumber_coarse = 4, 4, 16
    p.itnlim, p.rtol = 1000, 1e-8
    return p


def random_sym_graph(n, deg, seed, int_weights=True, diag_shift=1.0):
    """Random symmetric matrix with a dominant diagonal; integer-valued
    off-diagonals produce many exactly tied matching weights."""
    import bootcmatchg_b200 as bc
    import scipy.sparse as sp
    rng = np.random.default_rng(seed)
    m = n * deg // 2
    i = rng.integers(0, n, m)
    j = rng.integers(0, n, m)
    keep = i != j
    i, j = i[keep], j[keep]
    if int_weights:
        v = -rng.integers(1, 4, i.shape[0]).astype(float)
    else:
        v = -rng.uniform(0.5, 2.0, i.shape[0])
    a = sp.coo_matrix((v, (i, j)), shape=(n, n)).tocsr()
    a = a + a.T
    a.sum_duplicates()
    a = a.tocsr()
    d = np.asarray(abs(a).sum(axis=1)).ravel() + diag_shift
    a = a + sp.diags(d)
    a = a.tocsr()
    a.sort_indices()
    return bc.CsrMatrix.from_scipy(a)
