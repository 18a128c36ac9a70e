"""Multi-GPU as independent replicas (one process per GPU, no data-path collective).

A scan fits one B200, and independent scans shard with no exchange, so the
only collectives are for measurement: a barrier before and after a timed
region and the maximum of the ranks' times. Launched by
``torch.distributed.run`` (RANK / WORLD_SIZE / LOCAL_RANK / MASTER_* from the
environment); NCCL on GPUs, gloo for CPU tests.
"""

from __future__ import annotations

import datetime
import os

import torch
import torch.distributed as dist


def env_rank() -> tuple[int, int, int]:
    """(rank, world size, local rank) from the launcher's environment."""
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("LOCAL_RANK", "0"))


def init(backend: str = "nccl", timeout_s: float = 300.0) -> None:
    """Join the process group when launched with more than one rank."""
    if env_rank()[1] > 1 and not dist.is_initialized():
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))


def barrier() -> None:
    """All ranks reach this point (and, on GPUs, their work is complete)."""
    if dist.is_initialized() and dist.get_world_size() > 1:
        dist.barrier()
    if torch.cuda.is_available() and torch.cuda.is_initialized():
        torch.cuda.synchronize()


def max_over_ranks(value: float) -> float:
    """The largest value any rank holds (float64 all-reduce)."""
    if not (dist.is_initialized() and dist.get_world_size() > 1):
        return float(value)
    dev = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend() == "nccl" else torch.device("cpu")
    t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def shard(items: list, rank: int | None = None, world: int | None = None) -> list:
    """The items this rank processes when independent work is split across ranks
    (round robin, so uneven item costs spread evenly)."""
    r, w, _ = env_rank()
    r = r if rank is None else rank
    w = w if world is None else world
    return items[r::w]


def finish() -> None:
    """Leave the process group."""
    if dist.is_initialized():
        dist.destroy_process_group()


__all__ = ["barrier", "env_rank", "finish", "init", "max_over_ranks", "shard"]
