"""Multi-GPU policy of this library: replicas only.

The transposition has no exchange step (TTC's own multi-device mode runs whole replicas,
transposeGenerator.py:459-478 in the TTC project), so N GPUs run N independent seeded workloads:
rank r draws its problems from its own seed, no collective touches the data, and the only
collective is the max over ranks of each rank's device time, taken once per timed region
(weak scaling: the job's throughput is all ranks' bytes over the slowest rank's time).
"""
from __future__ import annotations

SEED_STRIDE = 1000  # rank r uses seed + r * SEED_STRIDE


def rank_seed(seed: int, rank: int) -> int:
    """The seed of rank `rank`'s independent workload."""
    return seed + SEED_STRIDE * rank


def max_over_ranks(value: float, device=None) -> float:
    """The maximum of `value` over all ranks of the default process group (the value itself when no
    group is initialised or it has one rank). `device` is where the reduction tensor lives: a CUDA
    device for NCCL, the CPU for gloo."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device if device is not None else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_throughput(bytes_per_rank: int, world: int, slowest_ms: float) -> float:
    """Whole-job GB/s: every rank moved `bytes_per_rank` in at most `slowest_ms`."""
    return bytes_per_rank * world / (slowest_ms / 1e3) / 1e9
