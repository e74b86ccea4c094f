"""Independent replicas across GPUs: one process per GPU, no data-path collective.

Global placement of one design does not shard at the sizes the engine targets
(the whole working set of a 210k-cell design is ~100 MB), so multi-GPU runs are
replicas: every rank places its own design instance on its own GPU, and only
timing is combined -- the slowest rank's device time bounds the whole job.
"""
from __future__ import annotations

import datetime
import os

import torch
import torch.distributed as dist


def world() -> tuple[int, int, int]:
    """(rank, world size, local rank) from the torchrun environment (1 process when absent)."""
    rank = int(os.environ.get("RANK", "0"))
    size = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", str(rank)))
    return rank, size, local


def init(backend: str | None = None, timeout_s: float = 120.0) -> bool:
    """Joins the process group when launched with more than one rank; returns whether it did."""
    _, size, _ = world()
    if size <= 1 or dist.is_initialized():
        return dist.is_initialized()
    if backend is None:
        backend = "nccl" if torch.cuda.is_available() else "gloo"
    os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
    kwargs = {"backend": backend, "timeout": datetime.timedelta(seconds=timeout_s)}
    if backend == "nccl":
        kwargs["device_id"] = torch.device("cuda", world()[2])
    dist.init_process_group(**kwargs)
    return True


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


def reduce_max(value: float) -> float:
    """Maximum of `value` over ranks (the job's time is its slowest rank's)."""
    if not dist.is_initialized():
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=_device())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def reduce_sum(value: float) -> float:
    if not dist.is_initialized():
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=_device())
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def shutdown() -> None:
    if dist.is_initialized():
        dist.destroy_process_group()


def replica_seed(base_seed: int, rank: int) -> int:
    """Instance i of a replicated workload uses seed base + i."""
    return int(base_seed) + int(rank)
