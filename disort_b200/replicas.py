"""Multi-GPU runs as replicas: one process per GPU, no data-path collective.

Every (column, band) instance of a spectral loop is independent of every other
(the reference's loop body touches only its own config copy and result,
python_bindings.cpp:108-127, 170-190), so N GPUs run N replicas of a workload,
each on its own instances.  The only cross-rank steps are a barrier on both
sides of a timed region and the maximum of the device-timed durations: the
job's time is its slowest rank's, and its throughput counts the instances of
every rank.
"""
from __future__ import annotations

import datetime
import os


def rank_env() -> tuple[int, int, int]:
    """(rank, local_rank, world_size) of this process from the launcher's environment."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("LOCAL_RANK", "0")),
            int(os.environ.get("WORLD_SIZE", "1")))


def init(backend: str = "nccl", timeout_s: float = 120.0) -> None:
    """Join the process group when there is more than one rank (short timeout, so
    that ranks waiting on a rank that died end with an error)."""
    import torch.distributed as dist
    if rank_env()[2] > 1 and not dist.is_initialized():
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))


def finish() -> None:
    import torch.distributed as dist
    if dist.is_initialized():
        dist.destroy_process_group()


def barrier() -> None:
    import torch.distributed as dist
    if dist.is_initialized() and dist.get_world_size() > 1:
        dist.barrier()


def replica_seed(base: int, rank: int) -> int:
    """Seed of a rank's synthetic instances: distinct per rank, rank 0 = the
    single-GPU workload."""
    return base + rank


def max_over_ranks(ms: float, device=None) -> float:
    """Largest value over all ranks (the job's duration), as a float."""
    import torch
    import torch.distributed as dist
    if not (dist.is_initialized() and dist.get_world_size() > 1):
        return float(ms)
    t = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(units_per_rank: int, steps: int, world: int, ms_max: float) -> float:
    """Whole-job throughput: the units every rank processed over the slowest rank's time."""
    return units_per_rank * steps * world / (ms_max / 1000.0)
