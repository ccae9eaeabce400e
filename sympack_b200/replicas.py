"""Replica coordination for runs on several GPUs of one node.

One factorization does not shard (its exchanges follow the elimination tree level by
level), so N GPUs run N independent replicas of the same workload: one process per GPU,
no data-path collective.  What the processes share is the timing: every timed region is
bracketed by a barrier, each rank measures its own device time, and the reported time is
the maximum over the ranks (the whole job is done when the slowest replica is), while the
work is the sum over the ranks.  These helpers hold that logic so that it is the same in
bench.py and in the multi-process tests (which run it over the gloo backend on CPU).
"""
from __future__ import annotations

import os


def world_info() -> tuple[int, int, int]:
    """(world size, rank, local rank) from the launcher's environment (1, 0, 0 alone)."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def max_over_ranks(values, device=None, dist=None):
    """Element-wise maximum of a list of floats over all ranks of the default process
    group (the values themselves when there is no group)."""
    import torch
    if dist is None:
        import torch.distributed as dist
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t.cpu()]


def job_rate(units_per_rank: float, world: int, max_ms: float) -> float:
    """Whole-job throughput: the work of every replica over the slowest replica's time
    (units per second)."""
    return world * units_per_rank / (max_ms * 1e-3)


def barrier(dist=None, sync=None):
    """Barrier over the ranks (if any), then the caller's device synchronisation."""
    if dist is None:
        import torch.distributed as dist
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.barrier()
    if sync is not None:
        sync()
