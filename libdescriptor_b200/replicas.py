"""Whole-job throughput of independent replicas (one process per GPU).

The descriptor path has no exchange step: every centre depends only on its
own neighbours, so N GPUs run N independent batches and only the timing is
combined.  Each rank times its own work on the device; the job's time is the
slowest rank's, and its throughput is all ranks' units over that time.
"""
from __future__ import annotations


def replica_throughput(units: float, ms: float, dist=None, device=None) -> tuple[float, float, float]:
    """(units per second of the whole job, the job's milliseconds = max over
    ranks, all ranks' units).  ``dist`` is ``torch.distributed`` (or None for
    one process); the reduction runs on ``device`` (a CUDA device for NCCL,
    the CPU for gloo)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return units / (ms * 1e-3), ms, units
    import torch

    t = torch.tensor([ms], dtype=torch.float64, device=device)
    u = torch.tensor([units], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.all_reduce(u, op=dist.ReduceOp.SUM)
    ms_max, total = float(t.item()), float(u.item())
    return total / (ms_max * 1e-3), ms_max, total
