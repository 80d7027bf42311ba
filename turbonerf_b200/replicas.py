"""Data-parallel replicas: one independent trainer per rank, no data-path collective.

The reference trains one scene on one GPU (src/services/device-manager.cuh:26-32). Scenes are
independent, so N GPUs run N replicas, each with its own seed; the only collectives are the
barrier around the timed region and the reduction of its result: the job's time is the
slowest rank's and its work is the sum of all ranks' work (weak scaling).
"""
from __future__ import annotations


def replica_seed(base: int, rank: int) -> int:
    """Seed of the replica on `rank`: distinct per rank, the base itself on rank 0."""
    return (int(base) + 7919 * int(rank)) & 0xFFFFFFFF


def barrier() -> None:
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.barrier()


def job_throughput(local_ms: float, local_units: float, device=None) -> tuple[float, float, float]:
    """Whole-job throughput of a timed region: (units per second, slowest rank's ms, total
    units). Every rank calls it with its own time and work; with one process, or none
    initialised, it is the local ratio. `device` is where the reduction tensors live (the CUDA
    device for NCCL, the CPU for gloo). A rank that has left makes the reduction fail with the
    process group's error after its timeout, on every rank still in it."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(local_ms)], dtype=torch.float64, device=device)
    u = torch.tensor([float(local_units)], dtype=torch.float64, device=device)
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dist.all_reduce(u, op=dist.ReduceOp.SUM)
    ms, units = float(t.item()), float(u.item())
    return units / (ms / 1e3) if ms > 0 else 0.0, ms, units
