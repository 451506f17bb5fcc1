"""Replica plumbing for multi-GPU runs: one process per GPU, no data-path collective.

Trajectories are independent, so N GPUs solve N independent ensembles (each
rank its own seeded trajectory range).  The only collectives are the harness's:
a barrier around timed regions and the max over ranks of a measured duration.
Both work on any torch.distributed backend (NCCL on GPUs, gloo in the CPU tests).
"""

from __future__ import annotations

import datetime
import os

import torch


def env_rank_world():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(
        os.environ.get("LOCAL_RANK", "0"))


def init(backend: str = "nccl", timeout_s: float = 120.0):
    """Join the process group when launched with more than one rank."""
    import torch.distributed as dist

    rank, world, local = env_rank_world()
    if world > 1 and not dist.is_initialized():
        kw = {}
        if backend == "nccl":
            torch.cuda.set_device(local)
            kw["device_id"] = torch.device("cuda", local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s), **kw)
    elif backend == "nccl":
        torch.cuda.set_device(0)
    return rank, world, local


def _device_for_collectives():
    import torch.distributed as dist

    if dist.get_backend() == "nccl":
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device("cpu")


def max_over_ranks(x: float, world: int) -> float:
    if world == 1:
        return float(x)
    import torch.distributed as dist

    t = torch.tensor([float(x)], dtype=torch.float64, device=_device_for_collectives())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()
    if torch.cuda.is_available() and torch.cuda.is_initialized():
        torch.cuda.synchronize()


def shard_seed(base_seed: int, rank: int) -> int:
    """Each rank's ensemble is drawn from its own seed (weak scaling, disjoint data)."""
    return base_seed + rank


def finalize(world: int):
    if world > 1:
        import torch.distributed as dist

        if dist.is_initialized():
            dist.destroy_process_group()
