"""Row sharding across ranks (one process per GPU) and the gathers that turn
per-rank results back into one network's result.

The inference of different input rows is independent, so a batch is split
into contiguous row ranges, one per rank, with no collective on the data
path (the reference splits the batch over GPUs the same way with one OpenMP
thread per GPU, src/cospdnn.cpp:150-184).  After the run, categories (global
row ids), per-layer survivor counts and the run time are combined with
torch.distributed: categories are concatenated in rank order (ranges are
contiguous and ascending, so the result stays sorted), survivor counts are
summed, times take the max over ranks.
"""
import numpy as np


def shard_rows(total, world, rank):
    """Contiguous near-equal range [row0, row1) of rank `rank`."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError("bad world/rank")
    return total * rank // world, total * (rank + 1) // world


def _dist():
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized():
        raise RuntimeError("torch.distributed is not initialized")
    return dist


def gather_categories(local, row0, group=None):
    """Global categories from each rank's local ones (row ids within its
    shard, ascending) and its first row; the same array on every rank."""
    dist = _dist()
    world = dist.get_world_size(group)
    mine = (np.asarray(local, np.int64) + int(row0)).tolist()
    parts = [None] * world
    dist.all_gather_object(parts, mine, group=group)
    return np.asarray([r for p in parts for r in p], np.int64)


def sum_alive(alive, group=None, device=None):
    """Per-layer survivor counts summed over ranks."""
    import torch
    dist = _dist()
    t = torch.as_tensor(np.asarray(alive, np.int64), device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return t.cpu().numpy()


def max_over_ranks(x, group=None, device=None):
    """Max of a per-rank scalar (a device-measured time) over ranks."""
    import torch
    dist = _dist()
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())
