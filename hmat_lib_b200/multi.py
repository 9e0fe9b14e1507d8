"""Several GPUs of one node, one process per GPU.

A single HODLR product does not shard without an exchange, so the engine
runs replicas; the instances of a batch of independent trees are instead
partitioned across the ranks, with no collective on the data path.  Timings
(and error sums) are combined with one small all-reduce per quantity, taken
by every rank in the same order.
"""
from __future__ import annotations


def partition(count: int, rank: int, world: int) -> list:
    """Instances of a batch owned by `rank`: every world-th one, so uneven
    sizes drawn in sequence spread evenly."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} of {world}")
    return list(range(rank, count, world))


def _reduce(value: float, dist, device, op_name: str) -> float:
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=getattr(dist.ReduceOp, op_name))
    return float(t.item())


def max_over_ranks(value: float, dist=None, device=None) -> float:
    """The job's time is its slowest rank's."""
    return _reduce(value, dist, device, "MAX")


def sum_over_ranks(value: float, dist=None, device=None) -> float:
    return _reduce(value, dist, device, "SUM")
