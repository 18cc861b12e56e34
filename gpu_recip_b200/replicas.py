"""Replica bookkeeping for multi-GPU runs.

One smooth-PME evaluation does not shard across GPUs (its 3-D FFT would need all-to-all
transposes, which the reference never finished either), so N GPUs run N independent replicas:
each rank evaluates its own systems with no data-path collective.  The only collectives are for
measurement: a barrier around the timed region and a MAX over ranks of the measured time.
"""
import os
from datetime import timedelta
from typing import List, Sequence, Tuple


def rank_world() -> Tuple[int, int, int]:
    """(rank, world_size, local_rank) from the torchrun environment (1 process: 0, 1, 0)."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def replica_seed(base: int, rank: int) -> int:
    """Seed of the synthetic input of one replica: distinct per rank, reproducible."""
    return int(base) + 7919 * int(rank)


def partition(n: int, world: int, rank: int) -> range:
    """Contiguous share of n independent units (systems) owned by one rank; shares differ by at
    most one unit and cover 0..n-1 exactly once."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank must be in [0, world)")
    q, r = divmod(int(n), int(world))
    lo = rank * q + min(rank, r)
    return range(lo, lo + q + (1 if rank < r else 0))


def init(backend: str, timeout_s: float = 120.0):
    """Initialise the process group when running under torchrun (world > 1)."""
    import torch.distributed as dist
    _, world, _ = rank_world()
    if world > 1 and not dist.is_initialized():
        dist.init_process_group(backend, timeout=timedelta(seconds=timeout_s))
    return world > 1


def barrier():
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        dist.barrier()


def max_over_ranks(value: float, device=None) -> float:
    """The largest value over all ranks (the value itself on one process)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value: float, device=None) -> float:
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def aggregate_rate(units_per_rank: Sequence[float], seconds: float) -> float:
    """Whole-job throughput: all ranks' units over the slowest rank's time."""
    if seconds <= 0:
        raise ValueError("seconds must be positive")
    return float(sum(units_per_rank)) / float(seconds)


def shutdown():
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        dist.destroy_process_group()
