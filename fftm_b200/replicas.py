"""Host logic of the multi-GPU forms (one process per GPU).

A single transform does not shard here: the reference's single-GPU ffts path has no
exchange step, so N GPUs run N independent replicas of the same solve and the
whole-job rate is the units all ranks processed over the slowest rank's device time.
A batch of independent uneven transforms shards by transform: each rank takes its
greedy longest-processing-time share (:func:`fftm_b200.batch.partition_lpt`) and runs
it with no collective on the data path.  The only collectives are the barrier around
the timed region and the max-over-ranks reduction of the time.
"""
from __future__ import annotations

import datetime
import os


def env_rank():
    """(rank, world_size, local_rank) from the torchrun environment (defaults 0, 1, 0)."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init_group(backend: str, device=None, timeout_s: float = 120.0):
    """Initialises the default process group when WORLD_SIZE > 1 and returns the
    torch.distributed module, else None.  A short timeout turns a rank that never
    arrives into an error on the others instead of a hang."""
    _, world, _ = env_rank()
    if world <= 1:
        return None
    import torch.distributed as dist
    kw = {"timeout": datetime.timedelta(seconds=timeout_s)}
    if device is not None and backend == "nccl":
        kw["device_id"] = device
    dist.init_process_group(backend, **kw)
    return dist


def max_over_ranks(dist, value: float, device=None) -> float:
    """The maximum of a per-rank value (e.g. the timed milliseconds) over all ranks."""
    if dist is None:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(units_per_rank_step: float, steps: int, world: int, max_ms: float) -> float:
    """Units per second of the whole job: every rank's units over the slowest rank's time."""
    return units_per_rank_step * steps * world / (max_ms * 1e-3)


def shard(shapes, rank: int, world: int):
    """Indices of the batch transforms that rank `rank` of `world` runs."""
    from .batch import partition_lpt
    if world <= 1:
        return list(range(len(shapes)))
    return partition_lpt(shapes, world)[rank]
