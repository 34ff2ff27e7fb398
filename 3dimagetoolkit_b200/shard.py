"""Spreading independent volumes over ranks (one process per GPU).

Volumes of a batch are independent, so the batch shards with no data-path collective:
rank r takes volumes r, r + W, r + 2W, ... (W ranks). The only collectives are the
ones that report a job-wide figure: the total voxel-iterations (sum) over the slowest
rank's device time (max).
"""
from __future__ import annotations


def volume_shard(n_volumes: int, rank: int, world: int) -> list[int]:
    """Indices of the volumes rank `rank` of `world` processes."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside a world of {world}")
    return list(range(rank, n_volumes, world))


def job_throughput(local_vox_iters: float, local_seconds: float, group=None) -> tuple[float, float]:
    """(job voxel-iterations, job seconds): sum over ranks and max over ranks.

    Uses torch.distributed when it is initialised (any backend), else returns the
    local figures."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()):
        return local_vox_iters, local_seconds
    dev = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend(group) == "nccl" \
        else torch.device("cpu")
    s = torch.tensor([local_vox_iters], dtype=torch.float64, device=dev)
    m = torch.tensor([local_seconds], dtype=torch.float64, device=dev)
    dist.all_reduce(s, op=dist.ReduceOp.SUM, group=group)
    dist.all_reduce(m, op=dist.ReduceOp.MAX, group=group)
    return float(s.item()), float(m.item())
