"""One process per GPU, independent replicas of the single-GPU count.

The count is a single-GPU path: no exchange step exists, so several GPUs run
independent replicas (each rank counts its own graph) and only the timing is
combined. torch.distributed carries the barrier and the max-over-ranks of
device-measured times; there is no data-path collective.
"""
from __future__ import annotations

import datetime
import os

import torch
import torch.distributed as dist


def env_ranks() -> tuple[int, int, int]:
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", str(rank)))
    return rank, world, local


def init(backend: str = "nccl", timeout_s: float = 300.0) -> tuple[int, int, int]:
    """Join the process group when launched by torchrun with WORLD_SIZE > 1."""
    rank, world, local = env_ranks()
    if world > 1 and not dist.is_initialized():
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        kw = {}
        if backend == "nccl":
            torch.cuda.set_device(local)
            kw["device_id"] = torch.device("cuda", local)
        dist.init_process_group(backend=backend, timeout=datetime.timedelta(seconds=timeout_s), **kw)
    return rank, world, local


def _device() -> torch.device:
    if dist.is_initialized() and dist.get_backend() == "nccl":
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device("cpu")


def barrier() -> None:
    if dist.is_initialized():
        if dist.get_backend() == "nccl":
            dist.barrier(device_ids=[torch.cuda.current_device()])
        else:
            dist.barrier()


def reduce_max(x: float) -> float:
    if not dist.is_initialized():
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=_device())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def reduce_sum(x: float) -> float:
    if not dist.is_initialized():
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=_device())
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def aggregate(per_rank_units: float, per_rank_seconds: float) -> tuple[float, float, float]:
    """Whole-job throughput: units all ranks processed / the slowest rank's time.
    Returns (value, total_units, max_seconds)."""
    total = reduce_sum(per_rank_units)
    tmax = reduce_max(per_rank_seconds)
    return (total / tmax if tmax > 0 else 0.0), total, tmax


def finish() -> None:
    if dist.is_initialized():
        barrier()
        dist.destroy_process_group()
