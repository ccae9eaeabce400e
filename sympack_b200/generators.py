"""Seeded synthetic SPD matrices of the shapes the benchmarks and tests use.

Every generator returns the lower triangle, diagonal included, as 1-based CSC
(colptr int64, rowind int32 sorted per column, nzval float64) — the input
convention of symPACK's DistSparseMatrix.  Grid points are numbered x fastest.
"""
from __future__ import annotations

import numpy as np


def _coo_to_lower_csc(n, rows, cols, vals):
    """rows >= cols (0-based) -> 1-based lower CSC with rows sorted per column."""
    order = np.lexsort((rows, cols))
    rows, cols, vals = rows[order], cols[order], vals[order]
    colptr = np.zeros(n + 1, np.int64)
    np.add.at(colptr, cols + 1, 1)
    colptr = np.cumsum(colptr) + 1
    colptr[0] = 1
    return colptr.astype(np.int64), (rows + 1).astype(np.int32), vals.astype(np.float64)


def _grid_edges(dims, offsets):
    """Pairs (i, j), i < j, of grid points joined by one of the given offsets.
    dims = (nx, ny[, nz]); offsets are (dx, dy[, dz]) tuples."""
    dims = tuple(int(d) for d in dims) + (1,) * (3 - len(dims))
    nx, ny, nz = dims
    idx = np.arange(nx * ny * nz, dtype=np.int64).reshape(nz, ny, nx)
    pi, pj = [], []
    for off in offsets:
        off = tuple(off) + (0,) * (3 - len(off))
        src, dst = [], []
        for d, size in ((off[2], nz), (off[1], ny), (off[0], nx)):
            if d >= 0:
                src.append(slice(0, size - d))
                dst.append(slice(d, size))
            else:
                src.append(slice(-d, size))
                dst.append(slice(0, size + d))
        a, b = idx[tuple(src)].ravel(), idx[tuple(dst)].ravel()
        pi.append(np.minimum(a, b))
        pj.append(np.maximum(a, b))
    if not pi:
        return np.empty(0, np.int64), np.empty(0, np.int64)
    return np.concatenate(pi), np.concatenate(pj)


def _forward_offsets(ndim, full):
    """Half of the stencil's neighbour offsets (one of each +/- pair)."""
    rng = (-1, 0, 1)
    offs = []
    if ndim == 2:
        cand = [(dx, dy) for dy in rng for dx in rng]
    else:
        cand = [(dx, dy, dz) for dz in rng for dy in rng for dx in rng]
    for o in cand:
        if not any(o):
            continue
        if not full and sum(abs(v) for v in o) != 1:
            continue
        # keep the lexicographically positive representative of +/- o
        rev = tuple(reversed(o))
        if rev > tuple(0 for _ in o):
            offs.append(o)
    return offs


def laplacian_2d(nx: int, ny: int, shift: float = 0.0):
    """5-point Dirichlet Laplacian: diagonal 4 + shift, neighbours -1."""
    n = nx * ny
    i, j = _grid_edges((nx, ny), _forward_offsets(2, False))
    rows = np.concatenate([np.arange(n), j])
    cols = np.concatenate([np.arange(n), i])
    vals = np.concatenate([np.full(n, 4.0 + shift), -np.ones(len(i))])
    return (n, *_coo_to_lower_csc(n, rows, cols, vals))


def laplacian_3d(nx: int, ny: int, nz: int, shift: float = 0.0):
    """7-point Dirichlet Laplacian: diagonal 6 + shift, neighbours -1."""
    n = nx * ny * nz
    i, j = _grid_edges((nx, ny, nz), _forward_offsets(3, False))
    rows = np.concatenate([np.arange(n), j])
    cols = np.concatenate([np.arange(n), i])
    vals = np.concatenate([np.full(n, 6.0 + shift), -np.ones(len(i))])
    return (n, *_coo_to_lower_csc(n, rows, cols, vals))


def _dominant(n, i, j, off, delta):
    absum = np.zeros(n)
    np.add.at(absum, i, np.abs(off))
    np.add.at(absum, j, np.abs(off))
    diag = absum * (1.0 + delta)
    diag[diag == 0] = 1.0
    rows = np.concatenate([np.arange(n), j])
    cols = np.concatenate([np.arange(n), i])
    vals = np.concatenate([diag, off])
    return (n, *_coo_to_lower_csc(n, rows, cols, vals))


def stencil27(nx: int, ny: int, nz: int, delta: float, seed: int = 0):
    """27-point stencil: off-diagonals U[-1, 0) from seed, diagonal = |row sum| (1 + delta)."""
    n = nx * ny * nz
    i, j = _grid_edges((nx, ny, nz), _forward_offsets(3, True))
    rng = np.random.default_rng(seed)
    off = -rng.uniform(0.0, 1.0, size=len(i))  # in (-1, 0]
    off[off == 0.0] = -0.5
    return _dominant(n, i, j, off, delta)


def random_graph_spd(n: int, avg_degree: float = 10.0, dominance: float = 1.05, seed: int = 0):
    """Random sparse graph, off-diagonals U[-1, 0), diagonal = dominance * |row sum|."""
    rng = np.random.default_rng(seed)
    m = int(n * avg_degree / 2)
    a = rng.integers(0, n, size=m)
    b = rng.integers(0, n, size=m)
    keep = a != b
    a, b = a[keep], b[keep]
    lo, hi = np.minimum(a, b), np.maximum(a, b)
    key = np.unique(lo.astype(np.int64) * n + hi)
    lo, hi = key // n, key % n
    off = -rng.uniform(0.0, 1.0, size=len(lo))
    off[off == 0.0] = -0.5
    return _dominant(n, lo, hi, off, dominance - 1.0)


def quasi_definite_3d(nx: int, ny: int, nz: int, frac_negative: float = 0.3, delta: float = 1e-2, seed: int = 0):
    """Symmetric indefinite, quasi-definite matrix on a 27-point grid graph: a seeded
    fraction of the vertices is 'negative'.  Couplings between vertices of the same
    sign are U[-1, 0) (positive block) or U(0, 1] (negative block), couplings across
    signs U[-1, 1); the diagonal is sign x (1 + delta) x (sum of |same-sign couplings|),
    or sign x 1 with none.  So the matrix is [H B^T; B -G] with H, G symmetric
    diagonally dominant: it has an LDL^T factorization without pivoting in every
    symmetric ordering, with as many negative pivots as negative vertices.
    Not positive definite (the Cholesky path rejects it)."""
    n = nx * ny * nz
    i, j = _grid_edges((nx, ny, nz), _forward_offsets(3, True))
    rng = np.random.default_rng(seed)
    sign = np.where(rng.uniform(size=n) < frac_negative, -1.0, 1.0)
    same = sign[i] == sign[j]
    mag = rng.uniform(0.0, 1.0, size=len(i))
    mag[mag == 0.0] = 0.5
    off = np.where(same, -sign[i] * mag, rng.uniform(-1.0, 1.0, size=len(i)))
    absum = np.zeros(n)
    np.add.at(absum, i[same], mag[same])
    np.add.at(absum, j[same], mag[same])
    diag = sign * np.where(absum > 0, absum * (1.0 + delta), 1.0)
    rows = np.concatenate([np.arange(n), j])
    cols = np.concatenate([np.arange(n), i])
    vals = np.concatenate([diag, off])
    return (n, *_coo_to_lower_csc(n, rows, cols, vals))


def config_matrix(name: str, **kw):
    """Named workloads: 'lap2d_64' (n=4096), 'lap3d_60' (n=216,000, shift 1e-3),
    'st27_80' (n=512,000, delta from kw), plus scaled-down variants 'lap3d_<k>', 'st27_<k>'."""
    if name.startswith("lap2d_"):
        k = int(name.split("_")[1])
        return laplacian_2d(k, k)
    if name.startswith("lap3d_"):
        k = int(name.split("_")[1])
        return laplacian_3d(k, k, k, shift=kw.get("shift", 1e-3))
    if name.startswith("st27_"):
        k = int(name.split("_")[1])
        return stencil27(k, k, k, delta=kw.get("delta", 1e-2), seed=kw.get("seed", 0))
    raise ValueError(name)


def batch_systems(count: int, n_min: int = 500, n_max: int = 20000, seed: int = 0):
    """Independent SPD systems of uneven size, n log-uniform in [n_min, n_max].

    Even-numbered systems are Laplacians on random grids (2D 5-point or 3D
    7-point, shift 1e-3), odd-numbered ones random sparse graphs of average
    degree 10 with off-diagonals U[-1, 0) and diagonal dominance 1.05.  The
    grid systems get the grid size closest to the drawn n.  Returns a list of
    (n, colptr, rowind, nzval)."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        target = int(round(np.exp(rng.uniform(np.log(n_min), np.log(n_max)))))
        if k % 2 == 0:
            if rng.uniform() < 0.5:
                ar = rng.uniform(0.5, 2.0)
                nx = max(2, int(round(np.sqrt(target * ar))))
                ny = max(2, int(round(target / nx)))
                out.append(laplacian_2d(nx, ny, 1e-3))
            else:
                a1, a2 = rng.uniform(0.7, 1.4, size=2)
                base = (target / (a1 * a2)) ** (1.0 / 3.0)
                nx = max(2, int(round(base * a1)))
                ny = max(2, int(round(base * a2)))
                nz = max(2, int(round(target / (nx * ny))))
                out.append(laplacian_3d(nx, ny, nz, 1e-3))
        else:
            out.append(random_graph_spd(target, 10.0, 1.05, seed=int(rng.integers(1 << 31))))
    return out


def block_diagonal(systems):
    """Stack systems [(n, colptr, rowind, nzval), ...] into one block-diagonal
    lower CSC.  Returns (n, colptr, rowind, nzval, sys_offsets) with 0-based
    system offsets (sys_offsets[k] = first row of system k, last = n)."""
    offs = np.zeros(len(systems) + 1, np.int32)
    for k, s in enumerate(systems):
        offs[k + 1] = offs[k] + s[0]
    n = int(offs[-1])
    cps, ris, vals = [np.ones(1, np.int64)], [], []
    base = 0
    for k, (nk, cp, ri, v) in enumerate(systems):
        cps.append(np.asarray(cp[1:], np.int64) - 1 + base + 1)
        ris.append(np.asarray(ri, np.int32) + offs[k])
        vals.append(np.asarray(v, np.float64))
        base += len(ri)
    return (n, np.concatenate(cps), np.concatenate(ris).astype(np.int32), np.concatenate(vals), offs)
