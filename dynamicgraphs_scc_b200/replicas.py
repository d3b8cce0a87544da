"""Replica runs over several GPUs, one process per GPU.

A decomposition of one graph does not shard: FW-BW needs reachability over the
whole graph, with no partition that exchanges once.  Several GPUs therefore
run independent replicas (weak scaling) and the only collective is the
reduction of their timings: the job's time is the slowest rank's, its work
the sum of the ranks' edges."""
from __future__ import annotations


def reduce_replicas(ms: float, edges: int, dist=None, device=None):
    """(slowest rank's ms, total edges over ranks); the local values when not distributed."""
    if dist is None or not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(ms), int(edges)
    import torch
    t_ms = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    t_e = torch.tensor([float(edges)], dtype=torch.float64, device=device)
    dist.all_reduce(t_ms, op=dist.ReduceOp.MAX)
    dist.all_reduce(t_e, op=dist.ReduceOp.SUM)
    return float(t_ms.item()), int(round(t_e.item()))
