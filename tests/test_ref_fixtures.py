"""Pins the oracle to BootCMatchG's own CUDA code.

The fixtures in tests/golden/ are outputs of the reference's unmodified
kernels (built by oracle/ref/Makefile, generated on a B200 by
tests/golden/make_ref_fixtures.py).  On the same inputs the oracle must give:
  - matching weights W within 4 ulps (device vs host log);
  - the same symmetric matching;
  - the same aggregates as a partition of the vertices (the reference numbers
    aggregates with atomicAdd, so its numbering is relabelled canonically:
    ascending smallest member, which is the oracle's numbering);
  - prolongator values within 2 ulps (the reference is compiled with FMA
    contraction, the oracle without);
  - the same number of Galerkin entries per row as nsparse's symbolic phase
    (row pointers recorded in the committed fixture by the run that made it).
    The values nsparse's numeric phase returned on the B200 are not usable
    (2213 of 5472 slots zero, 331 entries at columns that P^T A P does not
    have; whether nsparse's hash-table kernels or the cuSPARSE transposition
    of the build's compatibility shim is at fault was not established), so
    the oracle's Galerkin values are checked against scipy's P^T A P of the
    same P instead.

The suitor_*.npz fixtures pin the matching rule on more inputs (a random
geometric graph Laplacian, a 2-D anisotropic FV matrix, a 7-point grid, each
with a random smooth vector): the reference's sequential suitor matcher
(approx_match_cpu_suitor, src/AMG/suitor.cu:455-526, a host loop) run on the
oracle's weights.  That matcher compares with an absolute tolerance, so the
inputs were kept only where the weights within each row are more than ten
times that tolerance apart; on them its result is the exact rule's, and the
oracle's matching must equal it.

Only pair_poisson7_12 exercises the reference's kernels: on the next input (27-point Poisson 8^3) the
reference's matching-and-aggregation call did not finish within 900 s on a
B200, and its
stock solve() stopped with an illegal memory access (src/matrix/CSR.cu:140),
so its GPU code is not run again and the remaining cases have no fixture.
"""
import glob
import os

import numpy as np
import pytest

import bootcmatchg_b200 as bc
import workloads as wl
from oracle import oracle as orc

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
PAIR = sorted(glob.glob(os.path.join(GOLDEN, "pair_*.npz")))


def ulps(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    sp = np.spacing(np.maximum(np.abs(a), np.abs(b)))
    return np.where(a == b, 0.0, np.abs(a - b) / sp)


def canonical(agg):
    """Relabels aggregates by ascending smallest member."""
    nc = agg.max() + 1
    first = np.full(nc, agg.shape[0])
    np.minimum.at(first, agg, np.arange(agg.shape[0]))
    order = np.argsort(first)
    rank = np.empty(nc, np.int64)
    rank[order] = np.arange(nc)
    return rank[agg]


SUITOR = sorted(glob.glob(os.path.join(GOLDEN, "suitor_*.npz")))


def test_fixtures_present():
    assert len(PAIR) >= 1
    assert len(SUITOR) >= 3


@pytest.mark.parametrize("path", PAIR, ids=[os.path.basename(p)[5:-4] for p in PAIR])
def test_oracle_matches_reference_kernels(path):
    f = np.load(path)
    n = f["w"].shape[0]
    A = bc.CsrMatrix(n, f["row"], f["col"], f["val"])
    o = orc.pair_aggregate(A, f["w"])
    # W: the reference stores AH without the diagonal
    off = np.ones(A.nnz, bool)
    for i in range(n):
        seg = slice(A.row[i], A.row[i + 1])
        off[seg] = A.col[seg] != i
    assert ulps(o["W"][off], f["W"]).max() <= 4
    assert np.array_equal(o["match"], f["match"]), "matching differs from the reference"
    assert o["nc"] == int(f["nc"])
    assert np.array_equal(canonical(f["agg"]), o["agg"]), "aggregates differ"
    assert ulps(o["p"], f["p"]).max() <= 2
    # Galerkin with the reference's own numbering
    nc = int(f["nc"])
    crow, ccol, cval = orc.galerkin(A, f["agg"], f["p"], nc)
    if "crow" in f.files:
        # nsparse's row pointers, recorded by the run that made the fixture
        assert np.array_equal(crow, f["crow"]), "entries per Galerkin row differ"
    import scipy.sparse as sp
    P = sp.csr_matrix((f["p"], (np.arange(n), f["agg"])), shape=(n, nc))
    ref = (P.T @ A.to_scipy() @ P).toarray()
    ours = sp.csr_matrix((cval, ccol, crow), shape=(nc, nc)).toarray()
    assert np.abs(ours - ref).max() <= 1e-13 * np.abs(ref).max()



def _fixture_cases():
    """The generator's case table (tests/golden/make_ref_fixtures.py)."""
    import importlib.util
    spec = importlib.util.spec_from_file_location(
        "make_ref_fixtures", os.path.join(GOLDEN, "make_ref_fixtures.py"))
    mk = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mk)
    return mk


@pytest.mark.parametrize("path", SUITOR, ids=[os.path.basename(p)[7:-4] for p in SUITOR])
def test_oracle_matching_equals_reference_suitor(path):
    """suitor[v] of the reference = the vertex whose offer v holds.  The
    input is rebuilt from the seeded generators (checked against the
    fixture's checksum) and W from the oracle; every held offer is mutual
    (the matching), and the pairs are the oracle's: its greedy rule on W and
    its suitor restatement on (A, w)."""
    mk = _fixture_cases()
    f = np.load(path)
    name = os.path.basename(path)[:-4]
    make, wseed = {c[0]: (c[1], c[2]) for c in mk.SUITOR_CASES}[name]
    A = make()
    assert A.nnz == int(f["nnz"]) and float(A.val.sum()) == float(f["val_sum"])
    assert wseed == int(f["wseed"])
    w = np.abs(wl.vector(1, wseed, A.n)) + 0.1
    o = orc.pair_aggregate(A, w)
    wrow, _, wval = mk.off_diagonal(A, o["W"])
    assert mk.min_row_gap(wrow, wval) > mk.MIN_ROW_GAP  # no tie the tolerance could blur
    n = A.n
    s = f["suitor"]
    assert s.shape == (n,) and s.min() >= -1 and s.max() < n
    held = s >= 0
    assert np.array_equal(s[s[held]], np.arange(n)[held]), "an offer is not mutual"
    ref_match = np.where(held, s, -1)
    assert np.array_equal(orc.greedy_match(A, o["W"]), ref_match), "greedy differs"
    assert np.array_equal(o["match"], ref_match), "oracle matching differs from the reference"
