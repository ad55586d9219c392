"""Multi-GPU sharding of frame batches (one process per GPU).

Frames are independent, so a job of F frames splits into contiguous ranges,
one per rank, with no data-path collective. Each rank generates (or receives)
its own frames: the frame generator's counter is offset by the rank's first
frame so that shards never overlap. The only exchange is the reduction of a
few counters (frame errors, bit errors, iterations) and the max of the timings.
"""
from __future__ import annotations


def shard_range(total_frames: int, rank: int, world: int):
    """[first, count) of rank's contiguous share; the first ranks take one
    more frame when total_frames does not divide evenly."""
    if world < 1 or not (0 <= rank < world):
        raise ValueError("bad rank/world")
    base, extra = divmod(total_frames, world)
    first = rank * base + min(rank, extra)
    return first, base + (1 if rank < extra else 0)


def reduce_counters(values, device=None):
    """Sum a list of counters over all ranks (torch.distributed, any backend)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor(values, dtype=torch.float64, device=device)
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(t)
    return t.tolist()


def max_over_ranks(value: float, device=None) -> float:
    import torch
    import torch.distributed as dist
    t = torch.tensor([value], dtype=torch.float64, device=device)
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
