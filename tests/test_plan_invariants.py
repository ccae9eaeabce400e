"""Host-side invariants of the device plan, compiled from the library's own plan and
symbolic sources with g++ (no GPU): the tile shapes the tensor-core engines rely on (FP64
tiles cut from even rows for the 16-byte bulk copies, FP32 tiles in whole 32-column TMA
chunks), the persistent factorization's dispatch order (run one task at a time in that
order, no task ever waits), the tiny-leaf solve batches (first forward, last backward,
every tiny leaf in exactly one), the forward solve's arrival counts (what the tasks
signal equals what each supernode waits for), and both solve sweeps run one task at a time
in dispatch order with the kernels' wait targets and signals (no task waits for one handed
out after it, and every supernode ends done), the relative indices of the external updates
(filled by host threads on large plans) against a merge of the row lists, and the task
order re-built from measured durations (same tasks, waits and signals; still never
waiting for a later task).  The matrices: 7- and 27-point grids, and a
block-diagonal batch merged as the batch analysis merges its systems (grids, a dense block,
a path, one-column systems), each planned in FP64, FP32 and with small blocks."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "sympack_b200", "csrc")


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_plan_invariants_on_grid_matrices_and_a_batch(tmp_path):
    exe = tmp_path / "plan_invariants"
    srcs = [os.path.join(ROOT, "tests", "native", "plan_invariants.cpp")]
    srcs += [os.path.join(CSRC, f) for f in ("plan.cpp", "symbolic.cpp", "amd.cpp")]
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", CSRC, *srcs, "-o", str(exe)], check=True,
                   capture_output=True, text=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert r.stdout.startswith("ok")
