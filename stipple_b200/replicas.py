"""Replica arithmetic for N independent copies of a workload, one process per
GPU: images are independent, so ranks exchange nothing but one timing scalar
(the slowest rank's time sets the job's time)."""
from __future__ import annotations


def max_over_ranks(value: float) -> float:
    """The largest `value` over the default process group (itself without one).
    The scalar travels on the device for NCCL and on the host for gloo."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(units_per_rank: float, world: int, slowest_ms: float) -> float:
    """Whole-job units per second: every rank's units over the slowest rank's time."""
    return world * units_per_rank / (slowest_ms / 1e3)
