"""Scenes across GPUs: one process per GPU, each stepping its own share of independent scenes.

Scenes never interact, so the step has no data-path collective: a multi-GPU run partitions the scene list
(:func:`partition_scenes`), every rank steps its part with ``rb_step`` on its own device, and only the
measurements meet -- the timed region's device time as the maximum over ranks and the counts as sums
(:func:`max_over_ranks`, :func:`sum_over_ranks`).  These work with any ``torch.distributed`` backend (NCCL
between GPUs, gloo on the host).
"""
import numpy as np


def partition_scenes(costs, world_size):
    """Split scene indices into `world_size` parts of near-equal total cost (longest processing time first:
    each scene, largest first, goes to the part with the least cost so far; ties to the lower rank).
    Returns one ascending index array per rank; together they cover every scene exactly once."""
    costs = np.asarray(costs, dtype=np.float64)
    if world_size < 1:
        raise ValueError("world_size must be positive")
    order = np.argsort(-costs, kind="stable")
    load = np.zeros(world_size)
    parts = [[] for _ in range(world_size)]
    for i in order:
        r = int(np.argmin(load))
        parts[r].append(int(i))
        load[r] += costs[i]
    return [np.array(sorted(p), dtype=np.int64) for p in parts]


def _reduce(value, op, device):
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=op)
    return float(t.item())


def max_over_ranks(value, device="cpu"):
    """The largest `value` of all ranks (a no-op without an initialised process group)."""
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    return _reduce(value, dist.ReduceOp.MAX, device)


def sum_over_ranks(value, device="cpu"):
    """The sum of `value` over all ranks (a no-op without an initialised process group)."""
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    return _reduce(value, dist.ReduceOp.SUM, device)
