"""Independent solver replicas, one per GPU.

A FLUPS solve does not shard across devices here: independent solves
(batched right-hand sides, served requests) are the unit of work, so N GPUs
run N replicas with no data-path collective.  This module holds the host
logic shared by the benchmark and the serving loop: which device a rank
uses, how work items are split over ranks, and how a per-rank device time
becomes the job's time (the maximum over ranks).
"""
import os


def rank_info():
    """(rank, world_size, local_rank) from the torchrun environment (1 process if unset)."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def split_items(n_items, rank, world):
    """Contiguous, balanced share [start, stop) of n_items for this rank."""
    base, extra = divmod(n_items, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def max_over_ranks(value, group=None, device=None):
    """Job time = slowest rank (all ranks must call this in the same order)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size(group) == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


def sum_over_ranks(value, group=None, device=None):
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size(group) == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return float(t.item())
