"""Replicas over the GPUs of one node: the VELO path has no exchange step (events are
independent), so every rank reconstructs its own events and only the timing is combined.

Launched one process per GPU (torchrun); RANK / WORLD_SIZE / LOCAL_RANK / MASTER_* come from
the environment.  The rates are whole-job aggregates: every rank processes the same number of
events, and the job's time is the slowest rank's (max over ranks), measured on the device.
"""
from __future__ import annotations

import datetime
import os


def dist_env() -> tuple[int, int, int]:
    """(world size, rank, local rank) from the launcher's environment; (1, 0, 0) without one."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def init(backend: str = "nccl", timeout_s: float = 600.0) -> tuple[int, int, int]:
    """Joins the process group when there is more than one rank (NCCL: binds the local GPU
    first).  A short timeout makes ranks waiting for a lost peer end with an error."""
    world, rank, local = dist_env()
    if world > 1:
        import torch
        import torch.distributed as dist
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return world, rank, local


def rank_seed(seed: int, rank: int) -> int:
    """The event stream of a rank: disjoint from every other rank's."""
    return seed + 1_000_003 * rank


def max_over_ranks(value: float, device: str = "cuda") -> float:
    """The largest value over the ranks (the job's time is its slowest rank's)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_rate(world: int, units_per_rank: int, steps: int, ms: float) -> float:
    """Whole-job units per second: every rank's units over the slowest rank's time."""
    return world * units_per_rank * steps / (ms / 1e3)


def barrier():
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        dist.barrier()


def finish():
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        dist.destroy_process_group()
