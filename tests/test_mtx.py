"""Matrix Market loader (trl_csr_read_mtx) against the oracle's restatement of the
reference loader (examples/sycl/csrevp.hh:26-124), bit for bit, on files written here."""
import os

import numpy as np
import pytest

from trl_b200 import problems as P

native = pytest.importorskip("trl_b200.native")


def _lib_or_skip():
    if not os.path.exists(native.SOLVER_LIB):
        pytest.skip("solver library needs the reference headers at build time")


def _write(path, header, size, entries, fmt="{r} {c} {v}", comments=("% written by the loader test",)):
    with open(path, "w") as f:
        f.write(header + "\n")
        for c in comments:
            f.write(c + "\n")
        f.write(size + "\n")
        for r, c, v in entries:
            f.write(fmt.format(r=r, c=c, v=v) + "\n")


def _same(path, oracle, threads=0):
    A = native.read_mtx(path, threads)
    rows, cols, rp, ci, va = oracle.read_mtx(path)
    assert A.n == rows == cols
    assert np.array_equal(A.rowptr, rp)
    assert np.array_equal(A.colind, ci)
    assert np.array_equal(A.values, va)
    return A


def test_general_real_file_with_comments_and_duplicates(tmp_path, oracle):
    _lib_or_skip()
    rng = np.random.default_rng(1)
    n = 50
    ent = [(int(r), int(c), repr(float(v))) for r, c, v in zip(rng.integers(1, n + 1, 300), rng.integers(1, n + 1, 300), rng.standard_normal(300))]
    ent += ent[:5]  # duplicates are kept
    p = tmp_path / "general.mtx"
    _write(p, "%%MatrixMarket matrix coordinate real general", f"{n} {n} {len(ent)}", ent, fmt="  {r}\t{c}   {v}  ",
           comments=("% a comment", "", "%another"))
    _same(str(p), oracle)


def test_symmetric_lower_triangle_is_mirrored(tmp_path, oracle):
    _lib_or_skip()
    A = P.laplace2d(12)
    rows = A.row_indices()
    low = [(int(r) + 1, int(c) + 1, f"{v:.17g}") for r, c, v in zip(rows, A.colind, A.values) if c <= r]
    p = tmp_path / "sym.mtx"
    _write(p, "%%MatrixMarket MATRIX Coordinate Real SYMMETRIC", f"{A.n} {A.n} {len(low)}", low)
    B = _same(str(p), oracle)
    assert np.array_equal(B.to_dense(), A.to_dense())


def test_pattern_and_integer_files(tmp_path, oracle):
    _lib_or_skip()
    p = tmp_path / "pattern.mtx"
    _write(p, "%%MatrixMarket matrix coordinate pattern symmetric", "4 4 4", [(1, 1, ""), (2, 1, ""), (4, 3, ""), (3, 3, "")], fmt="{r} {c}")
    B = _same(str(p), oracle)
    assert B.nnz == 6 and np.all(B.values == 1.0)
    p = tmp_path / "integer.mtx"
    _write(p, "%%MatrixMarket matrix coordinate integer general", "3 3 3", [(1, 2, "+7"), (3, 1, "-2"), (2, 2, "5")])
    B = _same(str(p), oracle)
    assert B.values.tolist() == [7.0, 5.0, -2.0]


def test_parallel_parse_matches_serial(tmp_path, oracle):
    _lib_or_skip()
    A = P.zipf_symmetric(20_000, cap=64, seed=3)
    rows = A.row_indices()
    low = [(int(r) + 1, int(c) + 1, f"{v:.17g}") for r, c, v in zip(rows, A.colind, A.values) if c <= r]
    p = tmp_path / "big.mtx"
    _write(p, "%%MatrixMarket matrix coordinate real symmetric", f"{A.n} {A.n} {len(low)}", low)
    assert os.path.getsize(p) > 3 << 20  # several threads get a range (1 MiB each at least)
    one = native.read_mtx(str(p), 1)
    many = _same(str(p), oracle, threads=8)
    assert np.array_equal(one.rowptr, many.rowptr) and np.array_equal(one.colind, many.colind) and np.array_equal(one.values, many.values)
    assert np.array_equal(np.sort(many.values), np.sort(A.values))


@pytest.mark.parametrize("header,size,lines", [
    ("%%MatrixMarket matrix coordinate real general", "3 3 2", ["1 1 1.0"]),             # fewer entries than declared
    ("%%MatrixMarket matrix coordinate real general", "3 3 1", ["4 1 1.0"]),             # row out of range
    ("%%MatrixMarket matrix coordinate real general", "3 3 1", ["1 x 1.0"]),             # not a number
    ("%%MatrixMarket matrix array real general", "3 3", ["1.0"]),                         # dense format
    ("%%MatrixMarket matrix coordinate complex general", "3 3 1", ["1 1 1.0 0.0"]),      # complex field
])
def test_malformed_files_are_rejected(tmp_path, header, size, lines):
    _lib_or_skip()
    p = tmp_path / "bad.mtx"
    with open(p, "w") as f:
        f.write("\n".join([header, size, *lines]) + "\n")
    with pytest.raises(native.TrlError) as e:
        native.read_mtx(str(p))
    assert e.value.status == native.TRL_EINVAL


def test_missing_file_is_rejected(tmp_path):
    _lib_or_skip()
    with pytest.raises(native.TrlError):
        native.read_mtx(str(tmp_path / "absent.mtx"))
