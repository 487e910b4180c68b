"""Python mirror of the reference's host interface for the solve path.

    reference (BootCMatchG)                      here
    readMatrixFromFile  src/matrix/matrixIO.cu:4 read_matrix_from_file
    AMG::Params::initFromFile  src/AMG/AMG.cu:480 Params.init_from_file
    solve(A_host, p, rhs)  src/SOLVER/solver.cu:20 solve
    (setup inside solve(), solver.cu:37-62)      Handle(A, params) / Handle.solve

Everything runs in libbcmg.so through its C ABI; this module only moves
numpy arrays across it.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from ._lib import Csr, Ext, Params as _CParams, SolveInfo, check, lib

ERR_PARAM, ERR_ALLOC, ERR_PENDING = 1, 3, 11
PREC_FP64 = 0
PREC_MIXED = 1
STORE_FP32, STORE_BF16, STORE_FP16 = 0, 1, 2


@dataclass
class CsrMatrix:
    """Host CSR matrix: 0-based int32 row pointers / columns, FP64 values."""

    n: int
    row: np.ndarray
    col: np.ndarray
    val: np.ndarray
    m: int = -1

    def __post_init__(self):
        self.row = np.ascontiguousarray(self.row, dtype=np.int32)
        self.col = np.ascontiguousarray(self.col, dtype=np.int32)
        self.val = np.ascontiguousarray(self.val, dtype=np.float64)
        if self.m < 0:
            self.m = self.n

    @property
    def nnz(self) -> int:
        return int(self.col.shape[0])

    def as_c(self) -> Csr:
        c = Csr()
        c.n, c.m, c.nnz = self.n, self.m, self.nnz
        c.row = self.row.ctypes.data_as(C.POINTER(C.c_int32))
        c.col = self.col.ctypes.data_as(C.POINTER(C.c_int32))
        c.val = self.val.ctypes.data_as(C.POINTER(C.c_double))
        return c

    def to_scipy(self):
        import scipy.sparse as sp
        return sp.csr_matrix((self.val, self.col, self.row), shape=(self.n, self.m))

    @staticmethod
    def of(A) -> "CsrMatrix":
        """A itself, or a CsrMatrix over the n/row/col/val(/m) fields of any
        host CSR object (no copy when the arrays already have the dtypes)."""
        if isinstance(A, CsrMatrix):
            return A
        return CsrMatrix(A.n, A.row, A.col, A.val, getattr(A, "m", -1))

    @staticmethod
    def from_scipy(a) -> "CsrMatrix":
        a = a.tocsr()
        a.sort_indices()
        return CsrMatrix(a.shape[0], a.indptr, a.indices, a.data, a.shape[1])


def _take(c: Csr) -> CsrMatrix:
    """Copies a library-allocated bcmg_csr into numpy and frees it."""
    n, nnz = c.n, c.nnz
    row = np.ctypeslib.as_array(c.row, shape=(n + 1,)).copy()
    col = np.ctypeslib.as_array(c.col, shape=(nnz,)).copy() if nnz else np.zeros(0, np.int32)
    val = np.ctypeslib.as_array(c.val, shape=(nnz,)).copy() if nnz else np.zeros(0)
    m = c.m
    lib.bcmg_csr_free(C.byref(c))
    return CsrMatrix(n, row, col, val, m)


def read_matrix_from_file(path: str, m_type: int = 0) -> CsrMatrix:
    """readMatrixFromFile(path, m_type, loadOnDevice=false)."""
    c = Csr()
    check(lib.bcmg_read_matrix(path.encode(), m_type, C.byref(c)), "read_matrix_from_file")
    return _take(c)


def write_matrix_mm(path: str, A: CsrMatrix) -> None:
    c = CsrMatrix.of(A).as_c()
    check(lib.bcmg_write_matrix_mm(path.encode(), C.byref(c)), "write_matrix_mm")


@dataclass
class Params:
    """The 14 settings of struct params (src/AMG/AMG.cu:20-37)."""

    solver_type: int = 0
    max_hrc: int = 1
    conv_ratio: float = 0.8
    aggrsweeps: int = 2
    aggrtype: int = 0
    max_levels: int = 39
    cycle_type: int = 0
    coarse_solver: int = 4
    relax_type: int = 4
    relaxnumber_coarse: int = 20
    prerelax_sweeps: int = 1
    postrelax_sweeps: int = 1
    itnlim: int = 200000
    rtol: float = 1e-6
    matchtype: int = 3

    @staticmethod
    def init_from_file(path: str) -> "Params":
        p = _CParams()
        check(lib.bcmg_params_from_file(path.encode(), C.byref(p)), "Params.init_from_file")
        return Params._from_c(p)

    @staticmethod
    def default() -> "Params":
        p = _CParams()
        lib.bcmg_params_default(C.byref(p))
        return Params._from_c(p)

    @staticmethod
    def _from_c(p: _CParams) -> "Params":
        return Params(**{f: getattr(p, f) for f, _ in _CParams._fields_})

    def to_c(self) -> _CParams:
        p = _CParams()
        for f, _ in _CParams._fields_:
            setattr(p, f, getattr(self, f))
        return p

    def check(self) -> None:
        p = self.to_c()
        check(lib.bcmg_params_check(C.byref(p)), "Params.check")


@dataclass
class Extensions:
    precision: int = PREC_FP64
    coarse_storage: int = STORE_FP32
    replace_every: int = 0
    use_graphs: int = 1
    device: int = 0
    verbose: int = 0
    max_device_seconds: float = 2.0  # bound on each pipelined-pass wait
    match_step_limit: int = 0  # per-thread matching step bound (0: 8 nnz + 1024)
    stream: int = 0  # cudaStream_t as an integer (0: the handle makes its own)
    sliced: int = 1  # solve on the sliced copies of the levels
    autotune: int = 1  # batched solves: time the row-kernel shapes per level
    narrow_values: int = 1  # store solve-phase values narrower when exact

    def to_c(self) -> Ext:
        e = Ext()
        for f, _ in Ext._fields_:
            v = getattr(self, f)
            setattr(e, f, C.c_void_p(v) if f == "stream" else v)
        return e


@dataclass
class SolveResult:
    iters: int
    converged: bool
    residual: float
    rel_residual: float
    true_rel_residual: float
    setup_ms: float
    solve_ms: float
    num_hrc: int
    estimated_ratio: float

    @staticmethod
    def from_c(i: SolveInfo) -> "SolveResult":
        return SolveResult(i.iters, bool(i.converged), i.residual, i.rel_residual,
                           i.true_rel_residual, i.setup_ms, i.solve_ms, i.num_hrc,
                           i.estimated_ratio)


@dataclass
class LevelData:
    n: int
    nnz: int
    n_coarse: int
    A: CsrMatrix
    D: np.ndarray
    M: np.ndarray
    w: np.ndarray
    agg: np.ndarray | None = None
    p: np.ndarray | None = None


def _ptr(a: np.ndarray) -> C.c_void_p:
    return C.c_void_p(a.ctypes.data)


class Handle:
    """A set-up solver (bootstrap hierarchies on the device)."""

    def __init__(self, A: CsrMatrix, params: Params, ext: Extensions | None = None):
        self._h = C.c_void_p()
        ext = ext or Extensions()
        A = CsrMatrix.of(A)
        c = A.as_c()
        p = params.to_c()
        e = ext.to_c()
        check(lib.bcmg_setup(C.byref(c), C.byref(p), C.byref(e), C.byref(self._h)),
              "bcmg_setup")
        self.n = A.n
        self.params = params

    @classmethod
    def from_device(cls, n: int, nnz: int, row_ptr: int, col_ptr: int, val_ptr: int,
                    params: Params, ext: Extensions | None = None) -> "Handle":
        self = cls.__new__(cls)
        self._h = C.c_void_p()
        p = params.to_c()
        e = (ext or Extensions()).to_c()
        check(lib.bcmg_setup_device(n, nnz, C.c_void_p(row_ptr), C.c_void_p(col_ptr),
                                    C.c_void_p(val_ptr), C.byref(p), C.byref(e),
                                    C.byref(self._h)), "bcmg_setup_device")
        self.n = n
        self.params = params
        return self

    @classmethod
    def load(cls, path: str, ext: Extensions | None = None) -> "Handle":
        """A handle from a hierarchy file written by save(); no setup runs."""
        self = cls.__new__(cls)
        self._h = C.c_void_p()
        e = (ext or Extensions()).to_c()
        check(lib.bcmg_load(str(path).encode(), C.byref(e), C.byref(self._h)), "bcmg_load")
        n, nnz, nc = C.c_int32(), C.c_int32(), C.c_int32()
        check(lib.bcmg_level_info(self._h, 0, 0, C.byref(n), C.byref(nnz), C.byref(nc)),
              "level_info")
        p = _CParams()
        check(lib.bcmg_get_params(self._h, C.byref(p)), "bcmg_get_params")
        self.n = n.value
        self.params = Params._from_c(p)
        return self

    def save(self, path: str) -> None:
        """Writes the hierarchies to a file bcmg_load / Handle.load reads."""
        check(lib.bcmg_save(self._h, str(path).encode()), "bcmg_save")

    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            lib.bcmg_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def ptr(self) -> C.c_void_p:
        return self._h

    def solve(self, b: np.ndarray, x0: np.ndarray | None = None) -> tuple[np.ndarray, SolveResult]:
        b = np.ascontiguousarray(b, dtype=np.float64)
        x = np.zeros(self.n) if x0 is None else np.array(x0, dtype=np.float64, copy=True)
        info = SolveInfo()
        check(lib.bcmg_solve(self._h, _ptr(b), _ptr(x), 0, C.byref(info)), "bcmg_solve")
        return x, SolveResult.from_c(info)

    def solve_device(self, b_ptr: int, x_ptr: int) -> SolveResult:
        info = SolveInfo()
        check(lib.bcmg_solve(self._h, C.c_void_p(b_ptr), C.c_void_p(x_ptr), 1,
                             C.byref(info)), "bcmg_solve")
        return SolveResult.from_c(info)

    def precond_apply_device(self, r_ptr: int, z_ptr: int) -> None:
        check(lib.bcmg_precond_apply(self._h, C.c_void_p(r_ptr), C.c_void_p(z_ptr)),
              "bcmg_precond_apply")

    def solve_batch(self, B: np.ndarray, X0: np.ndarray | None = None
                    ) -> tuple[np.ndarray, list[SolveResult]]:
        """Solves A X = B for the columns of B (n x nrhs) on the shared
        hierarchy; returns X and one SolveResult per column."""
        B = np.asfortranarray(B, dtype=np.float64)
        if B.ndim != 2 or B.shape[0] != self.n:
            raise ValueError(f"B must be {self.n} x nrhs")
        nrhs = B.shape[1]
        X = (np.zeros((self.n, nrhs), order="F") if X0 is None
             else np.array(X0, dtype=np.float64, order="F", copy=True))
        infos = (SolveInfo * nrhs)()
        st = lib.bcmg_solve_batch(self._h, nrhs, _ptr(B), self.n, _ptr(X), self.n, 0, infos)
        check(st, "bcmg_solve_batch")
        return X, [SolveResult.from_c(i) for i in infos]

    def solve_batch_device(self, nrhs: int, b_ptr: int, ldb: int, x_ptr: int, ldx: int
                           ) -> list[SolveResult]:
        infos = (SolveInfo * nrhs)()
        check(lib.bcmg_solve_batch(self._h, nrhs, C.c_void_p(b_ptr), ldb, C.c_void_p(x_ptr),
                                   ldx, 1, infos), "bcmg_solve_batch")
        return [SolveResult.from_c(i) for i in infos]

    def precond_apply_batch_device(self, nrhs: int, r_ptr: int, ldr: int, z_ptr: int,
                                   ldz: int) -> None:
        check(lib.bcmg_precond_apply_batch(self._h, nrhs, C.c_void_p(r_ptr), ldr,
                                           C.c_void_p(z_ptr), ldz), "bcmg_precond_apply_batch")

    def batch_config(self, nrhs: int, hrc: int, level: int) -> dict:
        w, v, t, ms = C.c_int32(), C.c_int32(), C.c_int32(), C.c_double()
        check(lib.bcmg_batch_config(self._h, nrhs, hrc, level, C.byref(w), C.byref(v),
                                    C.byref(t), C.byref(ms)), "bcmg_batch_config")
        return {"width": w.value, "cols_per_lane": v.value, "threads": t.value,
                "tune_ms": ms.value}

    def device_bytes(self) -> int:
        b = C.c_uint64()
        check(lib.bcmg_device_bytes(self._h, C.byref(b)), "bcmg_device_bytes")
        return b.value

    def set_max_device_seconds(self, seconds: float) -> None:
        """Bound on each wait of the handle's pipelined row passes."""
        check(lib.bcmg_set_max_device_seconds(self._h, seconds),
              "bcmg_set_max_device_seconds")

    def set_stream(self, stream_ptr: int) -> None:
        check(lib.bcmg_set_stream(self._h, C.c_void_p(stream_ptr)), "bcmg_set_stream")

    def num_hierarchies(self) -> tuple[int, float]:
        nh, est = C.c_int(), C.c_double()
        check(lib.bcmg_hierarchy_count(self._h, C.byref(nh), C.byref(est)), "count")
        return nh.value, est.value

    def hierarchy_info(self, hrc: int = 0) -> dict:
        nl, oc, ow, ac = C.c_int(), C.c_double(), C.c_double(), C.c_double()
        check(lib.bcmg_hierarchy_info(self._h, hrc, C.byref(nl), C.byref(oc), C.byref(ow),
                                      C.byref(ac)), "hierarchy_info")
        return {"num_levels": nl.value, "op_cmplx": oc.value, "op_wcmplx": ow.value,
                "avg_cratio": ac.value}

    def level(self, hrc: int, level: int) -> LevelData:
        n, nnz, nc = C.c_int32(), C.c_int32(), C.c_int32()
        check(lib.bcmg_level_info(self._h, hrc, level, C.byref(n), C.byref(nnz),
                                  C.byref(nc)), "level_info")
        n, nnz, nc = n.value, nnz.value, nc.value
        row = np.zeros(n + 1, np.int32)
        col = np.zeros(nnz, np.int32)
        val = np.zeros(nnz)
        D, M, w = np.zeros(n), np.zeros(n), np.zeros(n)
        last = nc == 0
        agg = None if last else np.zeros(n, np.int32)
        p = None if last else np.zeros(n)
        check(lib.bcmg_level_copy(self._h, hrc, level, _ptr(row), _ptr(col), _ptr(val),
                                  _ptr(D), _ptr(M), None if last else _ptr(agg),
                                  None if last else _ptr(p), _ptr(w)), "level_copy")
        return LevelData(n, nnz, nc, CsrMatrix(n, row, col, val), D, M, w, agg, p)


@dataclass
class RequestResult:
    solve: SolveResult
    latency_ms: float
    queue_ms: float
    group: int
    cache_hit: bool


class Server:
    """Solve server (bcmg_server_*): continuous batching of solve requests
    with a hierarchy cache and memory-capped admission on one GPU."""

    def __init__(self, params: Params, ext: Extensions | None = None, slots: int = 4,
                 mem_cap_gb: float = 150.0, cache_cap_gb: float = 60.0, max_batch: int = 32,
                 device: int = 0):
        o = _lib.ServerOpts()
        lib.bcmg_server_opts_default(C.byref(o))
        o.device, o.slots, o.mem_cap_gb = device, slots, mem_cap_gb
        o.cache_cap_gb, o.max_batch = cache_cap_gb, max_batch
        o.params = params.to_c()
        o.ext = (ext or Extensions(device=device)).to_c()
        self._s = C.c_void_p()
        check(lib.bcmg_server_create(C.byref(o), C.byref(self._s)), "bcmg_server_create")
        self._live = {}  # ticket -> objects that must outlive the request

    def submit(self, A: CsrMatrix, b: np.ndarray, key: int = 0) -> int:
        A = CsrMatrix.of(A)
        c = A.as_c()
        b = np.ascontiguousarray(b, dtype=np.float64)
        x = np.zeros(A.n)
        t = C.c_uint64()
        check(lib.bcmg_server_submit(self._s, C.byref(c), key, _ptr(b), _ptr(x), C.byref(t)),
              "bcmg_server_submit")
        self._live[t.value] = (c, A, x)
        return t.value

    def wait(self, ticket: int, timeout: float = -1.0) -> tuple[np.ndarray, RequestResult]:
        info = _lib.RequestInfo()
        st = lib.bcmg_server_wait(self._s, ticket, timeout, C.byref(info))
        if st == ERR_PENDING:
            raise TimeoutError(f"request {ticket} pending")
        _, _, x = self._live.pop(ticket, (None, None, None))
        check(st, "bcmg_server_wait")
        return x, RequestResult(SolveResult.from_c(info.solve), info.latency_ms, info.queue_ms,
                                info.group, bool(info.cache_hit))

    def stats(self) -> dict:
        s = _lib.ServerStats()
        check(lib.bcmg_server_stats_get(self._s, C.byref(s)), "bcmg_server_stats_get")
        return {f: getattr(s, f) for f, _ in _lib.ServerStats._fields_}

    def close(self) -> None:
        if getattr(self, "_s", None) and self._s.value:
            lib.bcmg_server_destroy(self._s)
            self._s = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def solve(A: CsrMatrix, params: Params, rhs: np.ndarray,
          ext: Extensions | None = None) -> tuple[np.ndarray, SolveResult]:
    """solve(A_host, p, rhs) (src/SOLVER/solver.cu:20-129): setup, FCG from
    x0 = 0, teardown."""
    rhs = np.ascontiguousarray(rhs, dtype=np.float64)
    x = np.zeros(A.n)
    c = CsrMatrix.of(A).as_c()
    p = params.to_c()
    e = (ext or Extensions()).to_c()
    info = SolveInfo()
    check(lib.bcmg_solve_legacy(C.byref(c), C.byref(p), C.byref(e), _ptr(rhs), _ptr(x),
                                C.byref(info)), "solve")
    return x, SolveResult.from_c(info)
