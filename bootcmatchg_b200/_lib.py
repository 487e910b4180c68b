"""ctypes bindings to libbcmg.so (the product's C ABI, include/bcmg.h).

The library is loaded from this package's lib/ folder.  There is no Python or
CPU fallback: if the shared object is missing the import fails loudly.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_DIR = os.path.join(_HERE, "lib")
LIB_PATH = os.path.join(LIB_DIR, "libbcmg.so")

i32 = C.c_int32
i32p = C.POINTER(C.c_int32)
f64p = C.POINTER(C.c_double)
vp = C.c_void_p


class Csr(C.Structure):
    """bcmg_csr (include/bcmg.h)."""

    _fields_ = [("n", i32), ("m", i32), ("nnz", i32), ("row", i32p), ("col", i32p),
                ("val", f64p)]


class Params(C.Structure):
    """bcmg_params: same field order as the reference's struct params
    (src/AMG/AMG.cu:20-37)."""

    _fields_ = [("solver_type", C.c_int), ("max_hrc", C.c_int), ("conv_ratio", C.c_double),
                ("matchtype", C.c_int), ("aggrsweeps", C.c_int), ("aggrtype", C.c_int),
                ("max_levels", C.c_int), ("cycle_type", C.c_int), ("coarse_solver", C.c_int),
                ("relax_type", C.c_int), ("prerelax_sweeps", C.c_int),
                ("postrelax_sweeps", C.c_int), ("itnlim", C.c_int), ("rtol", C.c_double),
                ("relaxnumber_coarse", C.c_int)]


class Ext(C.Structure):
    """bcmg_ext: extensions beyond the reference's settings."""

    _fields_ = [("precision", C.c_int), ("coarse_storage", C.c_int),
                ("replace_every", C.c_int), ("use_graphs", C.c_int), ("device", C.c_int),
                ("verbose", C.c_int), ("max_device_seconds", C.c_double),
                ("stream", C.c_void_p), ("sliced", C.c_int), ("autotune", C.c_int),
                ("narrow_values", C.c_int), ("match_step_limit", C.c_int64)]


class SolveInfo(C.Structure):
    _fields_ = [("iters", C.c_int), ("converged", C.c_int), ("residual", C.c_double),
                ("rel_residual", C.c_double), ("true_rel_residual", C.c_double),
                ("setup_ms", C.c_double), ("solve_ms", C.c_double), ("num_hrc", C.c_int),
                ("estimated_ratio", C.c_double)]


class ServerOpts(C.Structure):
    _fields_ = [("device", C.c_int), ("slots", C.c_int), ("mem_cap_gb", C.c_double),
                ("cache_cap_gb", C.c_double), ("max_batch", C.c_int), ("params", Params),
                ("ext", Ext)]


class RequestInfo(C.Structure):
    _fields_ = [("solve", SolveInfo), ("latency_ms", C.c_double), ("queue_ms", C.c_double),
                ("group", C.c_int), ("cache_hit", C.c_int)]


class ServerStats(C.Structure):
    _fields_ = [(k, C.c_uint64) for k in ("submitted", "completed", "failed", "setups",
                                          "cache_hits", "batches", "evictions",
                                          "peak_resident_bytes", "resident_bytes")] + \
               [("cached_hierarchies", C.c_int), ("queued", C.c_int), ("running", C.c_int)]


# name -> (restype, argtypes); every symbol include/bcmg.h declares.
SIGNATURES = {
    "bcmg_last_error": (C.c_char_p, []),
    "bcmg_status_string": (C.c_char_p, [C.c_int]),
    "bcmg_version": (C.c_char_p, []),
    "bcmg_kernel_launches": (C.c_ulonglong, []),
    "bcmg_set_max_device_seconds": (C.c_int, [vp, C.c_double]),
    "bcmg_debug_fail_alloc": (C.c_int, [C.c_int64]),
    "bcmg_wait_selftest": (C.c_int, [C.c_int, C.c_double]),
    "bcmg_debug_alloc_stats": (C.c_int, [C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
    "bcmg_read_matrix": (C.c_int, [C.c_char_p, C.c_int, C.POINTER(Csr)]),
    "bcmg_write_matrix_mm": (C.c_int, [C.c_char_p, C.POINTER(Csr)]),
    "bcmg_csr_free": (None, [C.POINTER(Csr)]),
    "bcmg_csr_check": (C.c_int, [C.POINTER(Csr)]),
    "bcmg_params_default": (None, [C.POINTER(Params)]),
    "bcmg_params_from_file": (C.c_int, [C.c_char_p, C.POINTER(Params)]),
    "bcmg_params_check": (C.c_int, [C.POINTER(Params)]),
    "bcmg_ext_default": (None, [C.POINTER(Ext)]),
    "bcmg_setup": (C.c_int, [C.POINTER(Csr), C.POINTER(Params), C.POINTER(Ext),
                             C.POINTER(vp)]),
    "bcmg_setup_device": (C.c_int, [i32, i32, vp, vp, vp, C.POINTER(Params),
                                    C.POINTER(Ext), C.POINTER(vp)]),
    "bcmg_solve": (C.c_int, [vp, vp, vp, C.c_int, C.POINTER(SolveInfo)]),
    "bcmg_solve_legacy": (C.c_int, [C.POINTER(Csr), C.POINTER(Params), C.POINTER(Ext), vp,
                                    vp, C.POINTER(SolveInfo)]),
    "bcmg_destroy": (C.c_int, [vp]),
    "bcmg_set_stream": (C.c_int, [vp, vp]),
    "bcmg_precond_apply": (C.c_int, [vp, vp, vp]),
    "bcmg_solve_batch": (C.c_int, [vp, i32, vp, C.c_int64, vp, C.c_int64, C.c_int,
                                   C.POINTER(SolveInfo)]),
    "bcmg_precond_apply_batch": (C.c_int, [vp, i32, vp, C.c_int64, vp, C.c_int64]),
    "bcmg_level_relax_batch": (C.c_int, [vp, C.c_int, C.c_int, i32, vp, vp, C.c_int]),
    "bcmg_save": (C.c_int, [vp, C.c_char_p]),
    "bcmg_get_params": (C.c_int, [vp, C.POINTER(Params)]),
    "bcmg_load": (C.c_int, [C.c_char_p, C.POINTER(Ext), C.POINTER(vp)]),
    "bcmg_device_bytes": (C.c_int, [vp, C.POINTER(C.c_uint64)]),
    "bcmg_server_opts_default": (None, [C.POINTER(ServerOpts)]),
    "bcmg_server_create": (C.c_int, [C.POINTER(ServerOpts), C.POINTER(vp)]),
    "bcmg_server_submit": (C.c_int, [vp, C.POINTER(Csr), C.c_uint64, vp, vp,
                                     C.POINTER(C.c_uint64)]),
    "bcmg_server_wait": (C.c_int, [vp, C.c_uint64, C.c_double, C.POINTER(RequestInfo)]),
    "bcmg_server_stats_get": (C.c_int, [vp, C.POINTER(ServerStats)]),
    "bcmg_server_destroy": (C.c_int, [vp]),
    "bcmg_batch_config": (C.c_int, [vp, i32, C.c_int, C.c_int, i32p, i32p, i32p,
                                    C.POINTER(C.c_double)]),
    "bcmg_hierarchy_count": (C.c_int, [vp, C.POINTER(C.c_int), C.POINTER(C.c_double)]),
    "bcmg_hierarchy_info": (C.c_int, [vp, C.c_int, C.POINTER(C.c_int),
                                      C.POINTER(C.c_double), C.POINTER(C.c_double),
                                      C.POINTER(C.c_double)]),
    "bcmg_level_info": (C.c_int, [vp, C.c_int, C.c_int, i32p, i32p, i32p]),
    "bcmg_level_copy": (C.c_int, [vp, C.c_int, C.c_int, vp, vp, vp, vp, vp, vp, vp, vp]),
    "bcmg_level_relax": (C.c_int, [vp, C.c_int, C.c_int, vp, vp, C.c_int]),
    "bcmg_level_format": (C.c_int, [vp, C.c_int, C.c_int, C.POINTER(C.c_int64),
                                    C.POINTER(C.c_int64), i32p, i32p]),
    "bcmg_k_pair_aggregate": (C.c_int, [i32, i32, vp, vp, vp, vp, vp, vp, i32p, vp, vp,
                                        vp, vp]),
    "bcmg_k_spgemm": (C.c_int, [i32, i32, i32, vp, vp, vp, i32, i32, vp, vp, vp, vp, i32p,
                                vp, vp, vp]),
    "bcmg_k_galerkin": (C.c_int, [i32, i32, vp, vp, vp, i32, vp, vp, vp, i32p, vp, vp,
                                  vp]),
    "bcmg_k_relax": (C.c_int, [i32, i32, vp, vp, vp, vp, vp, vp, C.c_int, vp]),
    "bcmg_k_relax_noalloc": (C.c_int, [i32, i32, vp, vp, vp, vp, vp, vp, C.c_int, vp]),
    "bcmg_k_spmv": (C.c_int, [i32, i32, vp, vp, vp, C.c_double, vp, C.c_double, vp, vp]),
}


def _load() -> C.CDLL:
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build the CUDA library first "
            "(python -c 'import __graft_entry__ as g; g.build()' or make -C "
            "bootcmatchg_b200/csrc)")
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()


class BcmgError(RuntimeError):
    def __init__(self, status: int, where: str):
        self.status = status
        name = lib.bcmg_status_string(status).decode()
        msg = (lib.bcmg_last_error() or b"").decode()
        super().__init__(f"{where}: {name}: {msg}")


def check(status: int, where: str) -> None:
    if status != 0:
        raise BcmgError(status, where)
