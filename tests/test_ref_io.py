"""Pins host-side parts of the path to BootCMatchG's own host code.

oracle/ref/Makefile compiles the reference's unmodified src/matrix/matrixIO.cu
into oracle/_ref/libref.so; its reader (readMatrixFromFile with m_type 0 into
host memory, src/matrix/matrixIO.cu:4-192) and writer (CSRMatrixPrintMM,
matrixIO.cu:290-333) are plain host code, so these tests run them on the CPU
next to bcmg_read_matrix and bcmg_write_matrix_mm on the same files:
  - the reader gives the same row pointers and, row by row, the same
    (column, value) pairs bit for bit; the reference keeps each row in file
    order while bcmg_read_matrix sorts it, so rows are compared sorted;
    symmetric files are expanded the same way;
  - the writer produces the same bytes;
  - bcmg_params_from_file reads a settings file into the same 15 fields as
    AMG::Params::initFromFile (src/AMG/AMG.cu:480-526);
  - the oracle's coarsest-size rule and grid-sweep table equal
    BuildData::setMaxCoarseSize and ApplyData::setGridSweeps
    (src/AMG/AMG.cu:309-311, 371-394).
The library is built where the reference tree is present (this build
container); elsewhere the tests skip.
"""
import ctypes as C
import os

import numpy as np
import pytest

import bootcmatchg_b200 as bc
import workloads as wl

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBREF = os.path.join(ROOT, "oracle", "_ref", "libref.so")


@pytest.fixture(scope="module")
def ref():
    if not os.path.exists(LIBREF):
        pytest.skip("the reference's own build (oracle/_ref/libref.so) is not here")
    lib = C.CDLL(LIBREF)
    ip = C.POINTER(C.c_int)
    lib.ref_read_mm.argtypes = [C.c_char_p, ip, ip, ip, C.POINTER(ip), C.POINTER(ip),
                                C.POINTER(C.POINTER(C.c_double))]
    lib.ref_write_mm.argtypes = [C.c_int, C.c_int, C.c_int, ip, ip, C.POINTER(C.c_double),
                                 C.c_char_p]
    lib.ref_free.argtypes = [C.c_void_p]
    lib.ref_params_from_file.argtypes = [C.c_char_p, C.c_void_p]
    lib.ref_max_coarse_size.argtypes = [C.c_int]
    lib.ref_grid_sweeps.argtypes = [C.c_int, C.c_int, C.c_void_p]
    return lib


def ref_read(lib, path):
    n, m, nnz = C.c_int(), C.c_int(), C.c_int()
    row, col = C.POINTER(C.c_int)(), C.POINTER(C.c_int)()
    val = C.POINTER(C.c_double)()
    assert lib.ref_read_mm(str(path).encode(), C.byref(n), C.byref(m), C.byref(nnz),
                           C.byref(row), C.byref(col), C.byref(val)) == 0
    r = np.ctypeslib.as_array(row, shape=(n.value + 1,)).copy()
    c = np.ctypeslib.as_array(col, shape=(nnz.value,)).copy()
    v = np.ctypeslib.as_array(val, shape=(nnz.value,)).copy()
    for p in (row, col, val):
        lib.ref_free(C.cast(p, C.c_void_p))
    return n.value, m.value, r, c, v


def ref_write(lib, A, path):
    row = np.ascontiguousarray(A.row, dtype=np.int32)
    col = np.ascontiguousarray(A.col, dtype=np.int32)
    val = np.ascontiguousarray(A.val, dtype=np.float64)
    ip = C.POINTER(C.c_int)
    lib.ref_write_mm(A.n, A.m if A.m > 0 else A.n, len(val), row.ctypes.data_as(ip),
                     col.ctypes.data_as(ip), val.ctypes.data_as(C.POINTER(C.c_double)),
                     str(path).encode())


def random_entries(n, seed, symmetric):
    """Distinct (i, j, v) with a full diagonal; v spans many magnitudes and
    signs (a negative zero and subnormal-sized values included)."""
    rng = np.random.default_rng(seed)
    pairs = {(i, i) for i in range(n)}
    while len(pairs) < 5 * n:
        i, j = (int(x) for x in rng.integers(0, n, 2))
        if symmetric and j > i:
            i, j = j, i
        pairs.add((i, j))
    pairs = sorted(pairs)
    rng.shuffle(pairs)  # file order is not row order
    vals = rng.standard_normal(len(pairs)) * 10.0 ** rng.integers(-300, 300, len(pairs))
    vals[0] = -0.0
    return [(i, j, float(v)) for (i, j), v in zip(pairs, vals)]


def write_file(path, n, entries, symmetric):
    with open(path, "w") as f:
        kind = "symmetric" if symmetric else "general"
        f.write(f"%%MatrixMarket matrix coordinate real {kind}\n")
        f.write("% written by the test\n")
        f.write(f"{n} {n} {len(entries)}\n")
        for i, j, v in entries:
            f.write(f"{i + 1} {j + 1} {v!r}\n")


def assert_same_rows(A, n, row, col, val):
    assert A.n == n
    assert np.array_equal(A.row, row)
    for i in range(n):
        a, b = row[i], row[i + 1]
        o = np.argsort(col[a:b], kind="stable")
        assert np.array_equal(A.col[a:b], col[a:b][o]), i
        assert np.array_equal(A.val[a:b].view(np.int64), val[a:b][o].view(np.int64)), i


@pytest.mark.parametrize("symmetric", [False, True])
def test_reader_matches_reference(ref, tmp_path, symmetric):
    n = 40
    path = tmp_path / "a.mtx"
    write_file(path, n, random_entries(n, 3 + symmetric, symmetric), symmetric)
    rn, rm, row, col, val = ref_read(ref, path)
    assert rm == n
    A = bc.read_matrix_from_file(str(path))
    assert_same_rows(A, rn, row, col, val)


def test_reader_matches_reference_on_a_written_stencil(ref, tmp_path):
    """A 7-point Poisson matrix written by the reference's writer reads back
    the same through both readers (and equals the generator's matrix)."""
    P = wl.poisson(7, 6, 5, 4)
    path = tmp_path / "p.mtx"
    ref_write(ref, bc.CsrMatrix(P.n, P.row, P.col, P.val), path)
    rn, _, row, col, val = ref_read(ref, path)
    A = bc.read_matrix_from_file(str(path))
    assert_same_rows(A, rn, row, col, val)
    assert np.array_equal(A.col, P.col) and np.array_equal(A.val, P.val)


def test_writer_matches_reference_bytes(ref, tmp_path):
    n = 30
    src = tmp_path / "src.mtx"
    write_file(src, n, random_entries(n, 11, False), False)
    A = bc.read_matrix_from_file(str(src))
    ours, theirs = tmp_path / "ours.mtx", tmp_path / "theirs.mtx"
    bc.write_matrix_mm(str(ours), A)
    ref_write(ref, A, theirs)
    assert ours.read_bytes() == theirs.read_bytes()


SETTINGS = [
    # the reference's base file, values with its comments
    ["0 % solver_type", "1 % max_hrc", "0.8 % rho", "2 % aggr_sweeps", "0 % aggr_type",
     "39 % max_levels", "0 % cycle_type", "4 % coarsest_solver_type", "4 % relax_type",
     "20 % coarserelax_sweeps", "1 % prerelax_sweeps", "1 % postrelax_sweeps",
     "200000 % itnlim", "1.e-6 % rtol"],
    # the settings of the benchmarks' 7-point Poisson case, no comments
    ["0", "1", "0.8", "2", "0", "20", "0", "4", "4", "16", "4", "4", "1000", "1e-8"],
    # bootstrap composites, smoothed aggregation, W-cycle, Jacobi
    ["2", "3", "0.5", "1", "1", "10", "2", "0", "0", "7", "2", "3", "50",
     "2.5e-10   % tight"],
    ["1", "2", "0.25", "3", "0", "5", "1", "4", "0", "1", "0", "2", "7", "0.125"],
]


@pytest.mark.parametrize("case", range(len(SETTINGS)))
def test_settings_file_matches_reference(ref, tmp_path, case):
    from bootcmatchg_b200._lib import Params as CParams
    from bootcmatchg_b200._lib import check, lib
    path = tmp_path / "settings"
    path.write_text("\n".join(SETTINGS[case]) + "\n")
    ours, theirs = CParams(), CParams()
    check(lib.bcmg_params_from_file(str(path).encode(), C.byref(ours)), "params_from_file")
    assert ref.ref_params_from_file(str(path).encode(), C.byref(theirs)) == C.sizeof(CParams)
    # field by field (the padding bytes of the reference's struct, returned
    # by value, are not defined); doubles bit for bit
    import struct
    for name, ctype in CParams._fields_:
        a, b = getattr(ours, name), getattr(theirs, name)
        if ctype is C.c_double:
            a, b = struct.pack("<d", a), struct.pack("<d", b)
        assert a == b, (name, a, b)


def test_coarsest_size_rule_matches_reference(ref):
    from oracle import oracle as orc
    sizes = [1, 2, 7, 8, 26, 27, 63, 64, 125, 1000, 1728, 4096, 32768, 884736, 1000000,
             2097152, 4194304, 2000000, 2 ** 31 - 1]
    for n in sizes:
        assert orc.olib.orc_max_coarse_size(n) == ref.ref_max_coarse_size(n), n


def test_grid_sweeps_match_reference(ref):
    from oracle import oracle as orc
    for cycle_type in (0, 1, 2):
        for max_levels in range(1, 41):
            a = np.zeros(64, np.int32)
            b = np.zeros(64, np.int32)
            ka = orc.olib.orc_grid_sweeps(cycle_type, max_levels, C.c_void_p(a.ctypes.data))
            kb = ref.ref_grid_sweeps(cycle_type, max_levels, C.c_void_p(b.ctypes.data))
            assert ka == kb == max_levels - 1
            assert np.array_equal(a[:ka], b[:kb]), (cycle_type, max_levels)
