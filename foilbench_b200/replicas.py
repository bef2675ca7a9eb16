"""Multi-GPU host logic: one process per GPU, no data-path collective.

A single Stable Fluids solve does not shard (its row transforms would need an all-to-all
transpose and every CG iteration global dot products), so N GPUs run N independent
replicas of a single-solve workload, or split a set of independent scenarios (the batched and
served configurations) between them. The only collectives are the timing reduction (maximum
device time over ranks) and the throughput sum, over whatever process group is given (NCCL on
GPUs, gloo in the CPU tests).
"""

from __future__ import annotations

from typing import Sequence


def partition(weights: Sequence[float], world: int) -> list[list[int]]:
    """Split item indices between `world` ranks, largest weight first onto the least loaded
    rank (LPT). Every rank gets a list (possibly empty); the result is deterministic."""
    if world < 1:
        raise ValueError("world must be >= 1")
    loads = [0.0] * world
    out: list[list[int]] = [[] for _ in range(world)]
    for i in sorted(range(len(weights)), key=lambda k: (-float(weights[k]), k)):
        r = min(range(world), key=lambda q: (loads[q], q))
        out[r].append(i)
        loads[r] += float(weights[i])
    for lst in out:
        lst.sort()
    return out


def max_over_ranks(value: float, group=None, device=None) -> float:
    """Maximum of `value` over the ranks of `group` (the job's time is its slowest rank's)."""
    import torch
    import torch.distributed as dist

    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size(group) == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


def sum_over_ranks(value: float, group=None, device=None) -> float:
    import torch
    import torch.distributed as dist

    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size(group) == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return float(t.item())


def job_throughput(local_units: float, local_seconds: float, group=None, device=None) -> float:
    """Whole-job rate: all ranks' units divided by the slowest rank's time."""
    units = sum_over_ranks(local_units, group, device)
    seconds = max_over_ranks(local_seconds, group, device)
    return units / seconds if seconds > 0 else float("nan")
