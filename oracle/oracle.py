"""ctypes binding of the CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py.  The product library never loads it.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_PATH = os.path.join(_HERE, "liboracle.so")

vp = C.c_void_p
i32 = C.c_int32
i32p = C.POINTER(C.c_int32)


def _ptr(a):
    return None if a is None else C.c_void_p(a.ctypes.data)


class _Csr(C.Structure):
    _fields_ = [("n", i32), ("m", i32), ("nnz", i32), ("row", i32p), ("col", i32p),
                ("val", C.POINTER(C.c_double))]


class _Params(C.Structure):
    _fields_ = [("solver_type", C.c_int), ("max_hrc", C.c_int), ("conv_ratio", C.c_double),
                ("matchtype", C.c_int), ("aggrsweeps", C.c_int), ("aggrtype", C.c_int),
                ("max_levels", C.c_int), ("cycle_type", C.c_int), ("coarse_solver", C.c_int),
                ("relax_type", C.c_int), ("prerelax_sweeps", C.c_int),
                ("postrelax_sweeps", C.c_int), ("itnlim", C.c_int), ("rtol", C.c_double),
                ("relaxnumber_coarse", C.c_int)]


class _Info(C.Structure):
    _fields_ = [("iters", C.c_int), ("converged", C.c_int), ("residual", C.c_double),
                ("rel_residual", C.c_double), ("true_rel_residual", C.c_double),
                ("setup_ms", C.c_double), ("solve_ms", C.c_double), ("num_hrc", C.c_int),
                ("estimated_ratio", C.c_double)]


_SIG = {
    "orc_set_threads": (None, [C.c_int]),
    "orc_get_threads": (C.c_int, []),
    "orc_setup": (C.c_int, [C.POINTER(_Csr), C.POINTER(_Params), C.POINTER(vp)]),
    "orc_setup_from_w": (C.c_int, [C.POINTER(_Csr), C.POINTER(_Params), vp, C.POINTER(vp)]),
    "orc_solve": (C.c_int, [vp, vp, vp, C.POINTER(_Info)]),
    "orc_fcg_sample": (C.c_int, [vp, vp, vp, C.c_int, C.POINTER(C.c_double)]),
    "orc_precond_apply": (C.c_int, [vp, vp, vp]),
    "orc_destroy": (None, [vp]),
    "orc_hierarchy_count": (C.c_int, [vp, C.POINTER(C.c_int), C.POINTER(C.c_double)]),
    "orc_hierarchy_info": (C.c_int, [vp, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_double),
                                     C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "orc_level_info": (C.c_int, [vp, C.c_int, C.c_int, i32p, i32p, i32p]),
    "orc_level_copy": (C.c_int, [vp, C.c_int, C.c_int, vp, vp, vp, vp, vp, vp, vp, vp]),
    "orc_pair_aggregate": (C.c_int, [i32, i32, vp, vp, vp, vp, vp, vp, i32p, vp, vp, vp]),
    "orc_galerkin": (C.c_int, [i32, i32, vp, vp, vp, i32, vp, vp, vp, i32p, vp, vp]),
    "orc_relax": (C.c_int, [i32, vp, vp, vp, vp, vp, vp, C.c_int]),
    "orc_spgemm": (C.c_int, [i32, i32, vp, vp, vp, i32, i32, i32, vp, vp, vp, vp, i32p, vp, vp]),
    "orc_spmv": (C.c_int, [i32, vp, vp, vp, C.c_double, vp, C.c_double, vp]),
    "orc_greedy_match": (C.c_int, [i32, vp, vp, vp, vp]),
    "orc_max_coarse_size": (i32, [i32]),
    "orc_grid_sweeps": (C.c_int, [C.c_int, C.c_int, vp]),
}


def _load():
    if not os.path.exists(ORACLE_PATH):
        raise ImportError(f"{ORACLE_PATH} missing: run make -C oracle")
    lib = C.CDLL(ORACLE_PATH)
    for k, (r, a) in _SIG.items():
        f = getattr(lib, k)
        f.restype = r
        f.argtypes = a
    return lib


olib = _load()


def set_threads(n: int) -> None:
    olib.orc_set_threads(n)


def get_threads() -> int:
    return olib.orc_get_threads()


def _check(st, where):
    if st != 0:
        raise RuntimeError(f"oracle {where} failed with status {st}")


def _csr(A):
    c = _Csr()
    c.n, c.m, c.nnz = A.n, A.m, A.nnz
    c.row = A.row.ctypes.data_as(i32p)
    c.col = A.col.ctypes.data_as(i32p)
    c.val = A.val.ctypes.data_as(C.POINTER(C.c_double))
    return c


def _params(p):
    q = _Params()
    for f, _ in _Params._fields_:
        setattr(q, f, getattr(p, f))
    return q


class OracleHandle:
    """FP64 host setup + solve of the same method (parity oracle)."""

    def __init__(self, A, params, w=None):
        """Bootstrap setup; with w, a single hierarchy coarsened from w."""
        self._h = C.c_void_p()
        self._A = A
        c, p = _csr(A), _params(params)
        if w is None:
            _check(olib.orc_setup(C.byref(c), C.byref(p), C.byref(self._h)), "setup")
        else:
            self._w = np.ascontiguousarray(w, dtype=np.float64)
            _check(olib.orc_setup_from_w(C.byref(c), C.byref(p), _ptr(self._w),
                                         C.byref(self._h)), "setup_from_w")
        self.n = A.n

    def close(self):
        if self._h and self._h.value:
            olib.orc_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def solve(self, b, x0=None):
        b = np.ascontiguousarray(b, dtype=np.float64)
        x = np.zeros(self.n) if x0 is None else np.array(x0, dtype=np.float64, copy=True)
        info = _Info()
        st = olib.orc_solve(self._h, _ptr(b), _ptr(x), C.byref(info))
        return x, {f: getattr(info, f) for f, _ in _Info._fields_}, st

    def fcg_sample(self, b, iters):
        b = np.ascontiguousarray(b, dtype=np.float64)
        x = np.zeros(self.n)
        secs = C.c_double()
        _check(olib.orc_fcg_sample(self._h, _ptr(b), _ptr(x), iters, C.byref(secs)), "sample")
        return secs.value

    def precond_apply(self, r, z):
        r = np.ascontiguousarray(r, dtype=np.float64)
        z = np.array(z, dtype=np.float64, copy=True)
        _check(olib.orc_precond_apply(self._h, _ptr(r), _ptr(z)), "precond")
        return z

    def num_hierarchies(self):
        nh, est = C.c_int(), C.c_double()
        _check(olib.orc_hierarchy_count(self._h, C.byref(nh), C.byref(est)), "count")
        return nh.value, est.value

    def hierarchy_info(self, hrc=0):
        nl, oc, ow, ac = C.c_int(), C.c_double(), C.c_double(), C.c_double()
        _check(olib.orc_hierarchy_info(self._h, hrc, C.byref(nl), C.byref(oc), C.byref(ow),
                                       C.byref(ac)), "hinfo")
        return {"num_levels": nl.value, "op_cmplx": oc.value, "op_wcmplx": ow.value,
                "avg_cratio": ac.value}

    def level(self, hrc, level):
        n, nnz, nc = C.c_int32(), C.c_int32(), C.c_int32()
        _check(olib.orc_level_info(self._h, hrc, level, C.byref(n), C.byref(nnz),
                                   C.byref(nc)), "linfo")
        n, nnz, nc = n.value, nnz.value, nc.value
        out = {"n": n, "nnz": nnz, "n_coarse": nc,
               "row": np.zeros(n + 1, np.int32), "col": np.zeros(nnz, np.int32),
               "val": np.zeros(nnz), "D": np.zeros(n), "M": np.zeros(n), "w": np.zeros(n),
               "agg": np.zeros(n, np.int32) if nc else None,
               "p": np.zeros(n) if nc else None}
        _check(olib.orc_level_copy(self._h, hrc, level, _ptr(out["row"]), _ptr(out["col"]),
                                   _ptr(out["val"]), _ptr(out["D"]), _ptr(out["M"]),
                                   _ptr(out["agg"]), _ptr(out["p"]), _ptr(out["w"])), "lcopy")
        return out


def pair_aggregate(A, w):
    n = A.n
    agg, p = np.zeros(n, np.int32), np.zeros(n)
    W, s, m = np.zeros(A.nnz), np.zeros(n, np.int32), np.zeros(n, np.int32)
    nc = C.c_int32()
    w = np.ascontiguousarray(w, dtype=np.float64)
    _check(olib.orc_pair_aggregate(n, A.nnz, _ptr(A.row), _ptr(A.col), _ptr(A.val), _ptr(w),
                                   _ptr(agg), _ptr(p), C.byref(nc), _ptr(W), _ptr(s), _ptr(m)),
           "pair_aggregate")
    return {"agg": agg, "p": p, "nc": nc.value, "W": W, "suitor": s, "match": m}


def galerkin(A, agg, p, nc):
    agg = np.ascontiguousarray(agg, dtype=np.int32)
    p = np.ascontiguousarray(p, dtype=np.float64)
    crow = np.zeros(nc + 1, np.int32)
    cnnz = C.c_int32()
    _check(olib.orc_galerkin(A.n, A.nnz, _ptr(A.row), _ptr(A.col), _ptr(A.val), nc, _ptr(agg),
                             _ptr(p), _ptr(crow), C.byref(cnnz), None, None), "galerkin")
    ccol, cval = np.zeros(cnnz.value, np.int32), np.zeros(cnnz.value)
    _check(olib.orc_galerkin(A.n, A.nnz, _ptr(A.row), _ptr(A.col), _ptr(A.val), nc, _ptr(agg),
                             _ptr(p), _ptr(crow), C.byref(cnnz), _ptr(ccol), _ptr(cval)),
           "galerkin")
    return crow, ccol, cval


def spgemm(X, Y, m):
    """C = X Y (Y has m columns) in the canonical summation order."""
    crow = np.zeros(X.n + 1, np.int32)
    cnnz = C.c_int32()
    args = (X.n, X.nnz, _ptr(X.row), _ptr(X.col), _ptr(X.val), Y.n, m, Y.nnz, _ptr(Y.row),
            _ptr(Y.col), _ptr(Y.val), _ptr(crow), C.byref(cnnz))
    _check(olib.orc_spgemm(*args, None, None), "spgemm")
    ccol, cval = np.zeros(cnnz.value, np.int32), np.zeros(cnnz.value)
    _check(olib.orc_spgemm(*args, _ptr(ccol), _ptr(cval)), "spgemm")
    return crow, ccol, cval


def relax(A, d, f, u, k):
    u = np.array(u, dtype=np.float64, copy=True)
    d = np.ascontiguousarray(d, dtype=np.float64)
    f = np.ascontiguousarray(f, dtype=np.float64)
    _check(olib.orc_relax(A.n, _ptr(A.row), _ptr(A.col), _ptr(A.val), _ptr(d), _ptr(f), _ptr(u),
                          k), "relax")
    return u


def greedy_match(A, W):
    W = np.ascontiguousarray(W, dtype=np.float64)
    m = np.zeros(A.n, np.int32)
    _check(olib.orc_greedy_match(A.n, _ptr(A.row), _ptr(A.col), _ptr(W), _ptr(m)), "greedy")
    return m
