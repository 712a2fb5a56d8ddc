"""Multi-GPU form of the engine: independent replicas, one process per GPU.

A scene does not shard without a spatial decomposition (two halo exchanges
per IISPH sweep), while scenes are independent; N GPUs therefore run N
replicas (the 1M benchmark scene on every GPU, or disjoint shares of a scene
sweep) and nothing crosses between them on the data path. The only
collective is the end-of-run aggregation of the timing scalars: whole-job
units are summed and the device time is the maximum over ranks.
"""
from __future__ import annotations


def aggregate(local_ms: float, local_units: float, device=None):
    """(max over ranks of local_ms, sum over ranks of local_units); the
    identity without an initialized process group of more than one rank."""
    import torch
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(local_ms), float(local_units)
    t_max = torch.tensor([float(local_ms)], dtype=torch.float64, device=device)
    t_sum = torch.tensor([float(local_units)], dtype=torch.float64, device=device)
    dist.all_reduce(t_max, op=dist.ReduceOp.MAX)
    dist.all_reduce(t_sum, op=dist.ReduceOp.SUM)
    return float(t_max.item()), float(t_sum.item())


def share(items, rank: int, world_size: int):
    """This rank's share of a request list: every world_size-th item starting
    at rank (disjoint, covering, arrival order kept)."""
    if world_size < 1 or not 0 <= rank < world_size:
        raise ValueError("rank must lie in [0, world_size)")
    return list(items)[rank::world_size]
