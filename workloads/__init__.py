"""Seeded synthetic inputs for the solve path (libworkloads.so).

The reference ships no test matrices, so every workload of the tests and of
bench.py comes from these generators (splitmix64 uniforms, Box-Muller
normals, fixed seeds):

  poisson(stencil, nx, ny, nz)  7/27-point 3-D or 5-point 2-D Poisson,
                                Dirichlet unknowns eliminated, x-fastest rows
  fv2d(nx, ny, seed, aniso)     2-D cell-centred FV -div(K grad u), K = exp(2g)
  rgg(n, seed, ...)             random geometric graph Laplacian + shift I
  vector(kind, seed, n)         ones / standard normal / uniform [-1, 1]

This library is neither the product (libbcmg.so) nor the oracle: both the GPU
path and the CPU baseline read the same bytes from it.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
WORKLOADS_PATH = os.path.join(_HERE, "libworkloads.so")

i32 = C.c_int32
i32p = C.POINTER(C.c_int32)


class _Csr(C.Structure):
    _fields_ = [("n", i32), ("m", i32), ("nnz", i32), ("row", i32p), ("col", i32p),
                ("val", C.POINTER(C.c_double))]


def _load():
    if not os.path.exists(WORKLOADS_PATH):
        raise ImportError(f"{WORKLOADS_PATH} missing: run make -C workloads")
    lib = C.CDLL(WORKLOADS_PATH)
    sig = {
        "wl_poisson": (C.c_int, [C.c_int, i32, i32, i32, C.POINTER(_Csr)]),
        "wl_fv2d": (C.c_int, [i32, i32, C.c_uint64, C.c_double, C.POINTER(_Csr)]),
        "wl_rgg": (C.c_int, [i32, C.c_uint64, C.c_double, C.c_double, C.c_double,
                             C.c_double, C.POINTER(_Csr)]),
        "wl_vector": (C.c_int, [C.c_int, C.c_uint64, i32, C.c_void_p]),
        "wl_csr_free": (None, [C.POINTER(_Csr)]),
        "wl_last_error": (C.c_char_p, []),
    }
    for k, (r, a) in sig.items():
        f = getattr(lib, k)
        f.restype = r
        f.argtypes = a
    return lib


_lib = _load()


@dataclass
class Matrix:
    """Host CSR matrix: 0-based int32 row pointers / columns, FP64 values
    (the same fields as bootcmatchg_b200.CsrMatrix, which accepts it)."""

    n: int
    row: np.ndarray
    col: np.ndarray
    val: np.ndarray
    m: int = -1

    def __post_init__(self):
        if self.m < 0:
            self.m = self.n

    @property
    def nnz(self) -> int:
        return int(self.col.shape[0])

    def to_scipy(self):
        import scipy.sparse as sp
        return sp.csr_matrix((self.val, self.col, self.row), shape=(self.n, self.m))


def _check(st: int, what: str) -> None:
    if st != 0:
        raise ValueError(f"{what}: {_lib.wl_last_error().decode()}")


def _take(c: _Csr) -> Matrix:
    n, nnz = c.n, c.nnz
    row = np.ctypeslib.as_array(c.row, shape=(n + 1,)).copy()
    col = np.ctypeslib.as_array(c.col, shape=(nnz,)).copy() if nnz else np.zeros(0, np.int32)
    val = np.ctypeslib.as_array(c.val, shape=(nnz,)).copy() if nnz else np.zeros(0)
    _lib.wl_csr_free(C.byref(c))
    return Matrix(n, row, col, val, c.m)


def poisson(stencil: int, nx: int, ny: int, nz: int = 1) -> Matrix:
    c = _Csr()
    _check(_lib.wl_poisson(stencil, nx, ny, nz, C.byref(c)), "poisson")
    return _take(c)


def fv2d(nx: int, ny: int, seed: int = 2, aniso: float = 1e-3) -> Matrix:
    c = _Csr()
    _check(_lib.wl_fv2d(nx, ny, seed, aniso, C.byref(c)), "fv2d")
    return _take(c)


def rgg(n: int, seed: int, mean_degree: float = 12.0, wlo: float = 0.5, whi: float = 2.0,
        shift: float = 1e-3) -> Matrix:
    c = _Csr()
    _check(_lib.wl_rgg(n, seed, mean_degree, wlo, whi, shift, C.byref(c)), "rgg")
    return _take(c)


def vector(kind: int, seed: int, n: int) -> np.ndarray:
    """kind 0: ones, 1: standard normal, 2: uniform [-1, 1]."""
    out = np.zeros(n)
    _check(_lib.wl_vector(kind, seed, n, C.c_void_p(out.ctypes.data)), "vector")
    return out
