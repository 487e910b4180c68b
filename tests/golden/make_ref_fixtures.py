"""Generates the golden fixture that pins the CPU oracle.

The fixture is the output of BootCMatchG's own CUDA code -- the unmodified
reference sources built by oracle/ref/Makefile into oracle/_ref/libref.so --
on one seeded input from this repository's generators:

  pair_poisson7_12.npz  one matching + aggregation sweep (Matching::makeAH,
                        toMaximumProductMatrix, the suitor kernel, unsymFix,
                        _aggregate_symmetric) on the 7-point Poisson 12^3
                        matrix with w = 1: W, the symmetric matching, the
                        coarse index map, the prolongator values and the
                        number of aggregates.

This is the only input on which the reference's GPU code finished on a B200.
On the next one (27-point Poisson 8^3) the same call did not return within
900 s, and the reference's stock solve() stopped with an illegal memory
access, so the script runs this one case and nothing else.  The committed file
also holds crow/ccol/cval, the row pointers, columns and values of nsparse's
Galerkin product R (A P) of the same P, written by the run that made it; the
values came back corrupted, only the row pointers are used, and the harness no
longer exports that product, so this script does not write those arrays.

  suitor_*.npz          the reference's sequential suitor matching
                        (approx_match_cpu_suitor, src/AMG/suitor.cu:455-526, a
                        host loop that takes and returns device arrays) on the
                        matching weights W the oracle computes for a seeded
                        matrix and a seeded positive smooth vector w.  That
                        matcher compares weights with an absolute tolerance,
                        so only inputs whose weights within each row are
                        more than ten times that tolerance apart are kept (a
                        weight difference is exact to about 1e-15): on them
                        it follows the exact rule.  The file holds the
                        reference's suitor array and a checksum of the input
                        (nnz and the sum of the values); the test rebuilds A
                        and w from the same seeded generators and W with the
                        oracle.

Run on a GPU box (the reference tree is not needed there):
    python tests/golden/make_ref_fixtures.py OUTDIR            (pair case)
    python tests/golden/make_ref_fixtures.py OUTDIR --case suitor
TEST INFRASTRUCTURE ONLY.
"""
from __future__ import annotations

import ctypes as C
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import workloads as wl  # noqa: E402  (host generators only)

REF = os.path.join(ROOT, "oracle", "_ref", "libref.so")


def ptr(a):
    return C.c_void_p(a.ctypes.data)


def main():
    outdir = sys.argv[1] if len(sys.argv) > 1 else os.path.dirname(os.path.abspath(__file__))
    os.makedirs(outdir, exist_ok=True)
    lib = C.CDLL(REF)
    lib.ref_pair_aggregate.restype = C.c_int
    A = wl.poisson(7, 12, 12, 12)
    w = np.ones(A.n)
    n, nnz = A.n, A.nnz
    agg = np.zeros(n, np.int32)
    p = np.zeros(n)
    match = np.zeros(n, np.int32)
    W = np.zeros(nnz - n)
    nc = C.c_int()
    st = lib.ref_pair_aggregate(n, nnz, ptr(A.row), ptr(A.col), ptr(A.val), ptr(w), ptr(agg),
                                ptr(p), C.byref(nc), ptr(match), ptr(W))
    assert st == 0, f"CUDA error {st}"
    np.savez_compressed(os.path.join(outdir, "pair_poisson7_12.npz"), row=A.row, col=A.col,
                        val=A.val, w=w, W=W, match=match, agg=agg, p=p, nc=nc.value)
    print(f"pair_poisson7_12: n={n} nnz={nnz} nc={nc.value} matched={(match >= 0).sum()}")


# (name, matrix, seed of w): a random geometric graph Laplacian, a 2-D
# anisotropic FV matrix and a 7-point Poisson grid, each with a random w.
SUITOR_CASES = [
    ("suitor_rgg_20000", lambda: wl.rgg(20000, 21), 22),
    ("suitor_fv2d_64", lambda: wl.fv2d(64, 64, 24), 25),
    ("suitor_poisson7_16", lambda: wl.poisson(7, 16, 16, 16), 26),
]
MIN_ROW_GAP = 3.9e-9  # ten times the reference's tolerance, 3.9e-10 (suitor.cu:458)


def off_diagonal(A, W):
    """W over A's pattern (0 on the diagonal) as an n x n CSR without the
    diagonal, as Matching::makeAH stores it (src/AMG/matching.cu:293-317)."""
    rows = np.repeat(np.arange(A.n), np.diff(A.row))
    keep = A.col != rows
    counts = np.bincount(rows[keep], minlength=A.n)
    wrow = np.zeros(A.n + 1, np.int32)
    np.cumsum(counts, out=wrow[1:])
    return wrow, np.ascontiguousarray(A.col[keep]), np.ascontiguousarray(W[keep])


def min_row_gap(wrow, wval):
    gap = np.inf
    for i in range(len(wrow) - 1):
        v = np.sort(wval[wrow[i]:wrow[i + 1]])
        if v.size > 1:
            gap = min(gap, float(np.diff(v).min()))
    return gap


def suitor_cases(outdir):
    from oracle import oracle as orc
    lib = C.CDLL(REF)
    lib.ref_cpu_suitor.restype = C.c_int
    for name, make, wseed in SUITOR_CASES:
        A = make()
        w = np.abs(wl.vector(1, wseed, A.n)) + 0.1
        W = orc.pair_aggregate(A, w)["W"]
        wrow, wcol, wval = off_diagonal(A, W)
        gap = min_row_gap(wrow, wval)
        if not gap > MIN_ROW_GAP:
            print(f"{name}: weights within a row only {gap:.3g} apart; skipped")
            continue
        s = np.full(A.n, -2, np.int32)
        st = lib.ref_cpu_suitor(A.n, int(wval.size), ptr(wrow), ptr(wcol), ptr(wval), ptr(s))
        assert st == 0, f"CUDA error {st}"
        np.savez_compressed(os.path.join(outdir, name + ".npz"), suitor=s, nnz=A.nnz,
                            val_sum=float(A.val.sum()), wseed=wseed)
        print(f"{name}: n={A.n} weights={wval.size} row gap {gap:.3g} "
              f"held offers={(s >= 0).sum()}")


if __name__ == "__main__":
    if "--case" in sys.argv and sys.argv[sys.argv.index("--case") + 1] == "suitor":
        sys.argv = [a for a in sys.argv if a not in ("--case", "suitor")]
        out = sys.argv[1] if len(sys.argv) > 1 else os.path.dirname(os.path.abspath(__file__))
        os.makedirs(out, exist_ok=True)
        suitor_cases(out)
    else:
        main()
