"""Replica plumbing for running one tracker per GPU (one process per GPU).

Every ROI is independent and each bead's Z-LUT lives with its tracker, so multi-GPU use is
replication: rank r localizes its own ROIs on GPU r with no data-path collective (as the
reference's UseAll mode gives each device its own streams and LUT copy,
cudatrack/QueuedCUDATracker.cu:111-136,810-819). The only collectives are the timing
barrier and the max-over-ranks reduction of elapsed times, on the process group that
torchrun sets up (NCCL on GPUs, gloo on CPU).
"""
from __future__ import annotations

import os
from dataclasses import dataclass


@dataclass
class RankInfo:
    world_size: int
    rank: int
    local_rank: int


def env() -> RankInfo:
    return RankInfo(int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
                    int(os.environ.get("LOCAL_RANK", "0")))


def shard(n_total: int, rank: int, world_size: int) -> tuple[int, int]:
    """Contiguous share of n_total units for `rank`: (start, count); shares differ by at most 1."""
    base, extra = divmod(n_total, world_size)
    start = rank * base + min(rank, extra)
    return start, base + (1 if rank < extra else 0)


def init(backend: str, timeout_s: float = 300.0, device=None) -> RankInfo:
    """Join the process group torchrun describes (no-op for a single process)."""
    info = env()
    if info.world_size > 1:
        import datetime

        import torch.distributed as dist

        if not dist.is_initialized():
            kw = {"timeout": datetime.timedelta(seconds=timeout_s)}
            if device is not None:
                kw["device_id"] = device
            dist.init_process_group(backend, **kw)
    return info


def barrier() -> None:
    import torch.distributed as dist

    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.barrier()


def reduce_max(x: float, device=None) -> float:
    """Max of x over ranks (x on a single process)."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_rate(units_per_rank: int, world_size: int, seconds_max: float) -> float:
    """Whole-job throughput of weak-scaled replicas: all ranks' units over the slowest rank's time."""
    return units_per_rank * world_size / seconds_max


def finalize() -> None:
    import torch.distributed as dist

    if dist.is_available() and dist.is_initialized():
        dist.barrier()
        dist.destroy_process_group()
