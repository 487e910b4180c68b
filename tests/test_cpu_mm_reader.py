"""The Matrix-Market reader and writer (bcmg_read_matrix / bcmg_write_matrix_mm,
io.cpp; readMTXDouble and CSRMatrixPrintMM, src/matrix/matrixIO.cu:33-192,
292-335) on their edge cases, against a plain-Python reading of the same
rules: each of the nz lines after the size line is one record "i j [v]" read
as sscanf("%lld %lld %lf") reads it (white space of any kind between fields,
signs, any strtod number, trailing text ignored), symmetric storage mirrored
off the diagonal, each row sorted by column with duplicates summed in file
order.  The large cases are several megabytes, so the records are split
over the reader's threads (and chunk boundaries fall inside rows).
"""
import numpy as np
import pytest

import bootcmatchg_b200 as bc

HEAD = "%%MatrixMarket matrix coordinate {field} {sym}\n"


def expected_csr(n, records, symmetric):
    """records: (i, j, v) 1-based in file order."""
    rows = [dict() for _ in range(n)]
    order = [[] for _ in range(n)]

    def add(i, j, v):
        if j in rows[i]:
            rows[i][j] = rows[i][j] + v
        else:
            rows[i][j] = v
            order[i].append(j)

    for i, j, v in records:
        add(i - 1, j - 1, v)
        if symmetric and i != j:
            add(j - 1, i - 1, v)
    row, col, val = [0], [], []
    for i in range(n):
        for j in sorted(rows[i]):
            col.append(j)
            val.append(rows[i][j])
        row.append(len(col))
    return np.array(row), np.array(col), np.array(val)


def check(A, n, records, symmetric=False):
    row, col, val = expected_csr(n, records, symmetric)
    assert A.n == n
    assert np.array_equal(A.row, row) and np.array_equal(A.col, col)
    assert np.array_equal(A.val, val)


def read(tmp_path, text, name="m.mtx"):
    p = tmp_path / name
    p.write_bytes(text.encode())
    return bc.read_matrix_from_file(str(p))


def test_record_syntax(tmp_path):
    body = ("  1\t1   2.5\r\n"          # CRLF, tabs, leading blanks
            "+2 +1 +1e3\n"              # plus signs
            "1 2 -.5E-2 trailing\n"     # text after the value is ignored
            "2 2 0x1p3\n"               # hexadecimal float (strtod syntax)
            "3 3 5.\n"
            "3 1 1.5abc\n"              # the number ends where strtod stops
            "1 3 7")                    # no newline at the end
    A = read(tmp_path, HEAD.format(field="real", sym="general") + "% comment\n3 3 7\n" + body)
    check(A, 3, [(1, 1, 2.5), (2, 1, 1e3), (1, 2, -0.005), (2, 2, 8.0), (3, 3, 5.0),
                 (3, 1, 1.5), (1, 3, 7.0)])


def test_lines_after_the_records_are_ignored(tmp_path):
    A = read(tmp_path, HEAD.format(field="real", sym="general") +
             "2 2 2\n1 1 1\n2 2 2\nnot a record\n\n")
    check(A, 2, [(1, 1, 1.0), (2, 2, 2.0)])


@pytest.mark.parametrize("bad_line,index", [("\n", 1), ("1 +-2 3\n", 1), ("1 2\n", 1),
                                             ("1.0 2 3\n", 1), ("x\n", 1)])
def test_malformed_record_is_named(tmp_path, bad_line, index):
    text = HEAD.format(field="real", sym="general") + "2 2 3\n1 1 1\n" + bad_line + "2 2 2\n"
    with pytest.raises(bc.BcmgError, match=f"malformed record {index}"):
        read(tmp_path, text)


def test_missing_records(tmp_path):
    with pytest.raises(bc.BcmgError, match="error reading record 2 of 4"):
        read(tmp_path, HEAD.format(field="real", sym="general") + "2 2 4\n1 1 1\n2 2 2\n")


def test_pattern_integer_and_symmetric(tmp_path):
    A = read(tmp_path, HEAD.format(field="pattern", sym="general") + "2 2 2\n1 2\n2 1\n")
    check(A, 2, [(1, 2, 1.0), (2, 1, 1.0)])
    A = read(tmp_path, HEAD.format(field="integer", sym="symmetric") +
             "3 3 4\n1 1 4\n2 1 -1\n3 2 -2\n3 3 5\n")
    check(A, 3, [(1, 1, 4.0), (2, 1, -1.0), (3, 2, -2.0), (3, 3, 5.0)], symmetric=True)


def random_records(n, count, seed):
    rng = np.random.default_rng(seed)
    i = rng.integers(1, n + 1, size=count)
    j = rng.integers(1, n + 1, size=count)
    v = rng.standard_normal(count)
    return list(zip(i.tolist(), j.tolist(), v.tolist()))


@pytest.mark.parametrize("symmetric", [False, True])
def test_large_files_split_over_threads(tmp_path, symmetric):
    """About 8 MB of records in random order with duplicates (and, when
    symmetric, diagonal and off-diagonal records): the same CSR as a
    sequential reading."""
    n, count = 3000, 300_000
    recs = random_records(n, count, 5 + symmetric)
    if symmetric:
        recs = [(max(i, j), min(i, j), v) for i, j, v in recs]
    lines = "".join(f"{i} {j} {v!r}\n" for i, j, v in recs)
    text = HEAD.format(field="real", sym="symmetric" if symmetric else "general")
    text += f"{n} {n} {count}\n" + lines
    assert len(text) > 6 << 20  # more than one 4 MB share: several threads
    A = read(tmp_path, text)
    check(A, n, recs, symmetric)


def test_malformed_record_in_a_late_chunk(tmp_path):
    n, count = 1000, 250_000
    recs = random_records(n, count, 9)
    lines = [f"{i} {j} {v!r}\n" for i, j, v in recs]
    lines[200_123] = "1 2 oops\n"
    text = HEAD.format(field="real", sym="general") + f"{n} {n} {count}\n" + "".join(lines)
    with pytest.raises(bc.BcmgError, match="malformed record 200123"):
        read(tmp_path, text)


def test_written_file_reads_back_exactly(tmp_path):
    n, count = 2000, 200_000
    recs = random_records(n, count, 13)
    row, col, val = expected_csr(n, recs, False)
    A = bc.CsrMatrix(n, row.astype(np.int32), col.astype(np.int32), val)
    p = tmp_path / "w.mtx"
    bc.write_matrix_mm(str(p), A)
    head, size, first = p.read_text().split("\n", 3)[:3]
    assert head == "%%MatrixMarket matrix coordinate real general"
    assert size == f"{n}  {n} {A.nnz} "
    r0 = int(np.nonzero(np.diff(row))[0][0])
    assert first == "%d   %d  %.18e" % (r0 + 1, col[row[r0]] + 1, val[row[r0]])
    B = bc.read_matrix_from_file(str(p))
    assert np.array_equal(B.row, row) and np.array_equal(B.col, col)
    assert np.array_equal(B.val, val)


# The plain COO list (readMTX2Double, matrixIO.cu:194-289): "n nnz", then nnz
# row indices, nnz column indices and nnz values, 1-based, separated by any
# white space; each number is read from where the previous one stopped.
def test_coo_list_syntax_and_errors(tmp_path):
    def coo(text):
        p = tmp_path / "a.coo"
        p.write_text(text)
        return bc.read_matrix_from_file(str(p), m_type=1)

    A = coo("3 4\n1\t2 3 3\r\n1 1 3 1\n+2.5 -1e-1 0x1p2 7 trailing text\n")
    check(A, 3, [(1, 1, 2.5), (2, 1, -0.1), (3, 3, 4.0), (3, 1, 7.0)])
    for text, what in [("2 3\n1 2\n", "short row list"), ("2 2\n1 2\n1\n", "short column list"),
                       ("2 2\n1 2\n1 2\n3.0 x\n", "short value list"),
                       ("2 1000000000000\n1 2\n", "short row list"), ("0 1\n", "bad COO header"),
                       ("2\n", "bad COO header")]:
        with pytest.raises(bc.BcmgError, match=what):
            coo(text)


def test_coo_list_large(tmp_path):
    n, count = 5000, 200_000
    recs = random_records(n, count, 21)
    text = f"{n} {count}\n" + " ".join(str(i) for i, _, _ in recs) + "\n" + \
        " ".join(str(j) for _, j, _ in recs) + "\n" + " ".join(repr(v) for _, _, v in recs) + "\n"
    p = tmp_path / "b.coo"
    p.write_text(text)
    check(bc.read_matrix_from_file(str(p), m_type=1), n, recs)
