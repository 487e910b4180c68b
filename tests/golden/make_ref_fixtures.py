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

Run on a GPU box (the reference tree is not needed there):
    python tests/golden/make_ref_fixtures.py OUTDIR
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


if __name__ == "__main__":
    main()
