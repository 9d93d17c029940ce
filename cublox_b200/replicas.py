"""Map-sharded replicas across GPUs (one process per GPU).

Robots' maps are independent: a scan touches only its own map, so maps are
partitioned across ranks and every rank integrates its share with no data
exchange.  The only collective is the timing reduction that turns per-rank
times into a whole-job rate (the slowest rank bounds the job).
"""
from __future__ import annotations


def shard(n_maps: int, rank: int, world: int) -> range:
    """Contiguous block of map indices owned by `rank` (sizes differ by at
    most one, lower ranks take the extra)."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError("rank must be in [0, world)")
    base, extra = divmod(n_maps, world)
    start = rank * base + min(rank, extra)
    return range(start, start + base + (1 if rank < extra else 0))


def max_over_ranks(value: float, dist=None, device=None) -> float:
    """The maximum of a per-rank float over all ranks (identity without a
    process group)."""
    if dist is None:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value: float, dist=None, device=None) -> float:
    if dist is None:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def job_rate(units: float, seconds: float, dist=None, device=None) -> float:
    """Whole-job throughput: all ranks' units over the slowest rank's time."""
    return sum_over_ranks(units, dist, device) / max_over_ranks(seconds, dist, device)
