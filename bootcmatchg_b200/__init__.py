"""B200-native alpha-AMG + flexible CG: the BootCMatchG solve path on sm_100a.

The product is libbcmg.so (C ABI in include/bcmg.h); this package binds it.
"""
from .api import (CsrMatrix, Extensions, Handle, LevelData, Params, RequestResult, Server,
                  SolveResult, ERR_ALLOC, ERR_PARAM, ERR_PENDING,
                  PREC_FP64, PREC_MIXED, STORE_BF16, STORE_FP16, STORE_FP32,
                  read_matrix_from_file, solve, write_matrix_mm)
from ._lib import LIB_PATH, BcmgError, lib

__all__ = [
    "CsrMatrix", "Extensions", "Handle", "LevelData", "Params", "RequestResult", "Server",
    "SolveResult", "ERR_ALLOC", "ERR_PARAM", "ERR_PENDING",
    "PREC_FP64", "PREC_MIXED", "STORE_BF16", "STORE_FP16", "STORE_FP32",
    "read_matrix_from_file", "solve", "write_matrix_mm",
    "LIB_PATH", "BcmgError", "lib",
]
