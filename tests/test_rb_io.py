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
