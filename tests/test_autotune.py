"""Tile-shape autotuner, host side: picks the fastest candidate plan, caches it by
structure / options / GPU, and a cached entry is applied without timing.  The
numeric handle is a stand-in whose Factorize time depends on the plan."""
import json
import time

import numpy as np
import pytest

from sympack_b200 import autotune, generators as G
from sympack_b200.solver import DistSparseMatrix, symPACKOptions


class FakeM:
    def __init__(self):
        self.options = symPACKOptions(device=0)
        self.plan = None
        self.factorizations = 0
        self.calls = []

    def Replan(self, w, r, outer=0):
        self.plan = (w, r)
        self.outer = outer
        self.calls.append(("replan", w, r, outer))

    def DistributeMatrix(self, A):
        self.calls.append(("distribute",))

    def Factorize(self):
        self.factorizations += 1
        # fastest plan: (32, 128); the others are slower in proportion to their distance
        w, r = self.plan
        time.sleep(0.002 + 0.0005 * (abs(w - 32) / 16 + abs(r - 128) / 32) - 0.0003 * (self.outer == 512))


@pytest.fixture
def env(tmp_path, monkeypatch):
    monkeypatch.setenv("SPB_AUTOTUNE_CACHE", str(tmp_path / "tune.json"))
    monkeypatch.setattr(autotune, "_gpu_name", lambda device: "fake-gpu")
    n, cp, ri, v = G.laplacian_2d(12, 12)
    return tmp_path / "tune.json", DistSparseMatrix.from_lower_csc(n, cp, ri, v)


def test_tune_picks_fastest_and_caches(env):
    path, A = env
    M = FakeM()
    r = autotune.tune(M, A, reps=1)
    assert (r["small_max_w"], r["big_tile_rows"], r["outer_nb"]) == (32, 128, 512) and not r["cached"]
    assert M.plan == (32, 128) and M.outer == 512 and M.calls[-1] == ("distribute",)
    table = json.loads(path.read_text())
    assert len(table) == 1 and len(next(iter(table.values()))["times"]) == len(autotune.CANDIDATES) + 1
    M2 = FakeM()
    r2 = autotune.tune(M2, A, reps=1)
    assert r2["cached"] and M2.plan == (32, 128) and M2.outer == 512 and M2.factorizations == 0


def test_key_depends_on_structure_options_and_offsets(env):
    _, A = env
    M = FakeM()
    k1 = autotune.structure_key(M, A)
    k2 = autotune.structure_key(M, A, sys_offsets=np.array([0, A.size], np.int32))
    M.options = symPACKOptions(device=0, precision="FP32_IR")
    k3 = autotune.structure_key(M, A)
    n, cp, ri, v = G.laplacian_2d(12, 13)
    k4 = autotune.structure_key(FakeM(), DistSparseMatrix.from_lower_csc(n, cp, ri, v))
    assert len({k1, k2, k3, k4}) == 4


def test_old_cache_entry_without_outer_block_is_retuned(env):
    """An entry written before the outer block was tuned is timed again (and replaced)."""
    path, A = env
    M = FakeM()
    key = autotune.structure_key(M, A)
    path.write_text(json.dumps({key: {"small_max_w": 48, "big_tile_rows": 256, "seconds": 1.0, "times": {}}}))
    r = autotune.tune(M, A, reps=1)
    assert not r["cached"] and r["outer_nb"] in autotune.OUTER_CANDIDATES
    assert "outer_nb" in json.loads(path.read_text())[key]
