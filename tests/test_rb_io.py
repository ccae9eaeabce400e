"""Rutherford-Boeing input boundary (ReadHB_PARA restated)."""
import os

import numpy as np

from sympack_b200 import DistSparseMatrix, generators as G

HERE = os.path.dirname(os.path.abspath(__file__))


def test_roundtrip_cfg1(tmp_path):
    n, cp, ri, v = G.laplacian_2d(64, 64)
    A = DistSparseMatrix.from_lower_csc(n, cp, ri, v)
    p = str(tmp_path / "lap2d_64.rb")
    A.write_rb(p, "2D 5-point Laplacian 64x64")
    B = DistSparseMatrix.from_rb(p)
    assert B.size == n and np.array_equal(B.colptr, cp) and np.array_equal(B.rowind, ri)
    assert np.array_equal(B.nzvalLocal, v)
    lines = open(p).read().splitlines()
    assert lines[3].split() == ["(8I10)", "(8I10)", "(4E20.12)"]
    assert all(len(l) == 80 for l in lines[4:4 + (n + 1) // 8])


def test_roundtrip_random_values(tmp_path):
    n, cp, ri, v = G.stencil27(5, 4, 3, 1e-2, seed=3)
    p = str(tmp_path / "s.rb")
    DistSparseMatrix.from_lower_csc(n, cp, ri, v).write_rb(p)
    B = DistSparseMatrix.from_rb(p)
    assert np.array_equal(B.rowind, ri)
    assert np.allclose(B.nzvalLocal, v, rtol=1e-12, atol=0)


def test_reader_sorts_rows_and_accepts_d_exponent():
    B = DistSparseMatrix.from_rb(os.path.join(HERE, "golden", "tiny_unsorted.rb"))
    assert B.size == 5 and B.nnz == 9
    assert list(B.colptr) == [1, 4, 6, 8, 9, 10]
    assert list(B.rowind) == [1, 2, 3, 2, 4, 3, 5, 4, 5]
    assert list(B.nzvalLocal[:3]) == [4.0, -1.0, -1.0]


def test_parallel_fixed_width_and_free_layout_agree(tmp_path):
    """A file in the writer's fixed-width layout is split among threads by the
    reference's offset arithmetic; the same data with other spacing, 'D' exponents and
    CRLF line ends goes through the sequential parser: both give the same arrays."""
    n, cp, ri, v = G.stencil27(40, 40, 40, 1e-2, seed=4)  # ~870k entries: several threads
    p = str(tmp_path / "fixed.rb")
    DistSparseMatrix.from_lower_csc(n, cp, ri, v).write_rb(p)
    A = DistSparseMatrix.from_rb(p)
    assert np.array_equal(A.colptr, cp) and np.array_equal(A.rowind, ri)
    assert np.allclose(A.nzvalLocal, v, rtol=1e-12, atol=0)
    lines = open(p).read().split("\n")
    head, body = lines[:4], lines[4:]
    body = [" ".join(l.split()).replace("E", "D") for l in body]
    q = str(tmp_path / "free.rb")
    with open(q, "w", newline="") as f:
        f.write("\r\n".join(head + body))
    B = DistSparseMatrix.from_rb(q)
    assert np.array_equal(B.colptr, A.colptr) and np.array_equal(B.rowind, A.rowind)
    assert np.array_equal(B.nzvalLocal, A.nzvalLocal)


def test_d_exponents_in_fixed_width_fields(tmp_path):
    n, cp, ri, v = G.laplacian_2d(9, 7)
    p = str(tmp_path / "d.rb")
    DistSparseMatrix.from_lower_csc(n, cp, ri, v).write_rb(p)
    text = open(p).read().split("\n")
    nhead = 4 + (n + 1 + 7) // 8 + (len(ri) + 7) // 8
    text = text[:nhead] + [l.replace("E", "D") for l in text[nhead:]]
    open(p, "w").write("\n".join(text))
    B = DistSparseMatrix.from_rb(p)
    assert np.allclose(B.nzvalLocal, v, rtol=1e-12, atol=0)


def test_row_index_out_of_range_is_rejected(tmp_path):
    import pytest
    n, cp, ri, v = G.laplacian_2d(4, 4)
    bad = ri.copy()
    bad[3] = n + 5
    p = str(tmp_path / "bad.rb")
    DistSparseMatrix.from_lower_csc(n, cp, bad, v).write_rb(p)
    with pytest.raises(Exception):
        DistSparseMatrix.from_rb(p)
