"""Generates the golden fixtures that pin the CPU oracle.

The fixtures are outputs of BootCMatchG's own CUDA code -- the unmodified
reference sources built by oracle/ref/Makefile into oracle/_ref/libref.so --
on seeded inputs from this repository's generators:

  pair_<case>.npz   one matching + aggregation sweep (Matching::makeAH,
                    toMaximumProductMatrix, the suitor kernel, unsymFix,
                    _aggregate_symmetric): W, symmetric matching, coarse index
                    map, prolongator values, number of aggregates; and the
                    Galerkin product R (A P) of that P computed by nsparse.
  solve_<case>.npz  the stock solve(A, p, rhs): solution and #META output.

Run on a GPU box (the reference tree is not needed there):
    python tests/golden/make_ref_fixtures.py OUTDIR
On a B200 only pair_poisson7_12 finished: the next case's matching call did
not return within 900 s and the stock solve() faulted, so the reference's GPU
code is not run again and this script is kept as the record of how the
committed fixture was made.
TEST INFRASTRUCTURE ONLY.
"""
from __future__ import annotations

import ctypes as C
import os
import re
import subprocess
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import bootcmatchg_b200 as bc  # noqa: E402  (host generators only)

REF = os.path.join(ROOT, "oracle", "_ref", "libref.so")

# Inputs: (generator call, smooth vector); small enough to commit.
PAIR_CASES = {
    "poisson7_12": (lambda: bc.poisson(7, 12, 12, 12), None),
    "poisson27_8": (lambda: bc.poisson(27, 8, 8, 8), None),
    "poisson5_30": (lambda: bc.poisson(5, 30, 30), None),
    "fv2d_32": (lambda: bc.fv2d(32, 32, seed=2), None),
    "rgg_3000": (lambda: bc.rgg(3000, seed=4), None),
    "rgg_3000_w": (lambda: bc.rgg(3000, seed=4), ("normal", 9)),
    "fv2d_32_w": (lambda: bc.fv2d(32, 32, seed=5), ("uniform", 3)),
}

SOLVE_CASES = {
    "poisson7_16": lambda: bc.poisson(7, 16, 16, 16),
}


def smooth_vector(spec, n):
    if spec is None:
        return np.ones(n)
    kind, seed = spec
    return bc.vector(1 if kind == "normal" else 2, seed, n)


def c1_params():
    # solver_type, max_hrc, aggrsweeps, aggrtype, max_levels, cycle_type,
    # coarse_solver, relax_type, relaxnumber_coarse, prerelax, postrelax, itnlim
    prm = np.array([0, 1, 2, 0, 20, 0, 4, 4, 16, 4, 4, 1000], np.int32)
    dprm = np.array([0.8, 1e-8])
    return prm, dprm


def ptr(a):
    return C.c_void_p(a.ctypes.data)


def pair_fixture(lib, name, make, wspec, outdir):
    A = make()
    w = smooth_vector(wspec, A.n)
    n, nnz = A.n, A.nnz
    agg = np.zeros(n, np.int32)
    p = np.zeros(n)
    match = np.zeros(n, np.int32)
    W = np.zeros(nnz - n)
    nc = C.c_int()
    st = lib.ref_pair_aggregate(n, nnz, ptr(A.row), ptr(A.col), ptr(A.val), ptr(w), ptr(agg),
                                ptr(p), C.byref(nc), ptr(match), ptr(W))
    assert st == 0, f"{name}: CUDA error {st}"
    crow = np.zeros(nc.value + 1, np.int32)
    cnnz = C.c_int()
    st = lib.ref_galerkin(n, nnz, ptr(A.row), ptr(A.col), ptr(A.val), nc.value, ptr(agg),
                          ptr(p), ptr(crow), C.byref(cnnz), None, None)
    assert st == 0
    ccol = np.zeros(cnnz.value, np.int32)
    cval = np.zeros(cnnz.value)
    st = lib.ref_galerkin(n, nnz, ptr(A.row), ptr(A.col), ptr(A.val), nc.value, ptr(agg),
                          ptr(p), ptr(crow), C.byref(cnnz), ptr(ccol), ptr(cval))
    assert st == 0
    np.savez_compressed(os.path.join(outdir, f"pair_{name}.npz"), row=A.row, col=A.col,
                        val=A.val, w=w, W=W, match=match, agg=agg, p=p, nc=nc.value,
                        crow=crow, ccol=ccol, cval=cval)
    print(f"pair_{name}: n={n} nnz={nnz} nc={nc.value} matched={(match >= 0).sum()}")


def solve_fixture(name, make, outdir):
    """Runs the stock solve() in a child process to capture its #META lines."""
    A = make()
    b = np.ones(A.n)
    tmp = os.path.join(outdir, f"_{name}_inputs.npz")
    np.savez(tmp, row=A.row, col=A.col, val=A.val, b=b)
    code = (
        "import ctypes as C, numpy as np, sys\n"
        f"lib = C.CDLL({REF!r})\n"
        f"d = np.load({tmp!r})\n"
        "row, col, val, b = [np.ascontiguousarray(d[k]) for k in ('row','col','val','b')]\n"
        f"prm = np.array({c1_params()[0].tolist()}, np.int32)\n"
        f"dprm = np.array({c1_params()[1].tolist()})\n"
        "x = np.zeros(b.shape[0])\n"
        "P = lambda a: C.c_void_p(a.ctypes.data)\n"
        "st = lib.ref_solve(b.shape[0], col.shape[0], P(row), P(col), P(val), P(prm), P(dprm), P(b), P(x))\n"
        "sys.stdout.flush()\n"
        f"np.save({tmp!r} + '.x.npy', x)\n"
        "sys.exit(st)\n")
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True,
                         timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    meta = dict(re.findall(r"#META (\S+) \w+ (\S+)", out.stdout))
    x = np.load(tmp + ".x.npy")
    os.remove(tmp + ".x.npy")
    os.remove(tmp)
    np.savez_compressed(os.path.join(outdir, f"solve_{name}.npz"), x=x,
                        iters=int(meta["sol;num_iteration"]),
                        residual=float(meta["sol;residual"]),
                        levels_meta=out.stdout[-4000:])
    print(f"solve_{name}: iters={meta['sol;num_iteration']} residual={meta['sol;residual']}")


def main():
    outdir = sys.argv[1] if len(sys.argv) > 1 else os.path.dirname(os.path.abspath(__file__))
    os.makedirs(outdir, exist_ok=True)
    lib = C.CDLL(REF)
    lib.ref_pair_aggregate.restype = C.c_int
    lib.ref_galerkin.restype = C.c_int
    for name, (make, wspec) in PAIR_CASES.items():
        pair_fixture(lib, name, make, wspec, outdir)
    for name, make in SOLVE_CASES.items():
        solve_fixture(name, make, outdir)


if __name__ == "__main__":
    main()
