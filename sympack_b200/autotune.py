"""Tile-shape autotuner for the factorization plan.

Three plan parameters shape the kernel sequence of a factorization:

* ``small_max_w`` — supernodes up to this many columns (and 96 KB of panel) are
  factored whole in shared memory by one CTA each, one launch per level;
  wider ones go through the blocked POTRF / TRSM / update path.
* ``big_tile_rows`` — update products with at least this many rows use
  128 x 128 tensor-core tiles, smaller ones 64 x 64 tiles.
* ``outer_nb`` — columns per outer block of a wide panel: its trailing columns
  are updated once per outer block (256 or 512; larger blocks halve the
  trailing-matrix traffic of the update tiles but lengthen the in-block chain).

Which values are fastest depends on the supernode-size distribution of the
matrix (a batch of many small systems favours wide shared-memory panels and
small tiles; one large 3D problem the opposite).  ``tune`` times every
(small_max_w, big_tile_rows) candidate on the device with the real values, keeps the
fastest, then tries its outer block at 512 columns against 256; results are
cached in a JSON file keyed by the input structure, the relaxation and
precision options and the GPU name, so that a structure seen before is planned
without timing.  The cache lives at ``$SPB_AUTOTUNE_CACHE`` or
``~/.cache/sympack_b200/autotune.json``.
"""
from __future__ import annotations

import hashlib
import json
import os
import time

import numpy as np

from .solver import DistSparseMatrix, symPACKMatrix2D

CANDIDATES = [(w, r) for w in (16, 32, 48) for r in (96, 128, 256)]
OUTER_CANDIDATES = (256, 512)


def cache_path() -> str:
    return os.environ.get("SPB_AUTOTUNE_CACHE") or os.path.join(os.path.expanduser("~"), ".cache", "sympack_b200",
                                                                "autotune.json")


def _gpu_name(device: int) -> str:
    import torch  # device properties only
    return torch.cuda.get_device_name(device)


def structure_key(M: symPACKMatrix2D, A: DistSparseMatrix, sys_offsets=None) -> str:
    """Hash of everything the plan depends on: input structure, batch offsets,
    ordering / relaxation / precision options and the GPU."""
    o = M.options
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(A.colptr, np.int64).tobytes())
    h.update(np.ascontiguousarray(A.rowind, np.int32).tobytes())
    if sys_offsets is not None:
        h.update(np.ascontiguousarray(sys_offsets, np.int32).tobytes())
    r = o.relax
    h.update(repr((o.orderingStr, o.precision, r.nrelax0, r.nrelax1, r.nrelax2, r.maxSize, r.zrelax0, r.zrelax1,
                   r.zrelax2)).encode())
    h.update(_gpu_name(o.device).encode())
    return h.hexdigest()


def _load(path):
    try:
        with open(path) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _store(path, table):
    os.makedirs(os.path.dirname(path) or ".", exist_ok=True)
    tmp = f"{path}.{os.getpid()}.tmp"
    with open(tmp, "w") as f:
        json.dump(table, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


def time_candidate(M: symPACKMatrix2D, A: DistSparseMatrix, w: int, r: int, reps: int = 3, outer: int = 0) -> float:
    """Best-of-reps factorization time (seconds) with plan (w, r, outer); the first
    factorization (graph capture) is not timed."""
    M.Replan(w, r, outer)
    best = float("inf")
    for k in range(reps + 1):
        M.DistributeMatrix(A)
        t0 = time.perf_counter()
        M.Factorize()
        dt = time.perf_counter() - t0
        if k:
            best = min(best, dt)
    return best


def tune(M: symPACKMatrix2D, A: DistSparseMatrix, sys_offsets=None, candidates=None, reps: int = 3,
         use_cache: bool = True) -> dict:
    """Pick the plan of M (after its symbolic factorization) and leave M
    replanned with it and A distributed, ready for Factorize.

    Returns {"small_max_w", "big_tile_rows", "outer_nb", "seconds", "cached", "times"}."""
    path = cache_path()
    key = structure_key(M, A, sys_offsets)
    table = _load(path) if use_cache else {}
    if key in table and "outer_nb" in table[key]:
        e = table[key]
        M.Replan(e["small_max_w"], e["big_tile_rows"], e["outer_nb"])
        M.DistributeMatrix(A)
        return dict(e, cached=True)
    times = {}
    for w, r in candidates or CANDIDATES:
        times[f"{w},{r},{OUTER_CANDIDATES[0]}"] = time_candidate(M, A, w, r, reps, OUTER_CANDIDATES[0])
    best = min(times, key=times.get)
    w, r, _ = (int(x) for x in best.split(","))
    for o in OUTER_CANDIDATES[1:]:
        times[f"{w},{r},{o}"] = time_candidate(M, A, w, r, reps, o)
    best = min(times, key=times.get)
    w, r, o = (int(x) for x in best.split(","))
    e = {"small_max_w": w, "big_tile_rows": r, "outer_nb": o, "seconds": times[best], "times": times}
    if use_cache:
        table = _load(path)
        table[key] = e
        _store(path, table)
    M.Replan(w, r, o)
    M.DistributeMatrix(A)
    return dict(e, cached=False)
