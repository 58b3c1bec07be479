"""Replica-parallel frames on several GPUs of one node.

The frame does not shard: every pixel path reads the whole scene, and the
screen-space passes (ReSTIR spatial reuse, a-trous, TAA) couple pixels up to
~75 px apart.  N GPUs therefore run N independent replicas of the job, one
process per GPU (torchrun), each rendering its own stretch of the camera path.
Nothing crosses GPUs on the data path; after the timed region one all-reduce
takes the slowest rank's times, and the job's throughput is the units all
ranks processed divided by that time.
"""
from __future__ import annotations

# each replica starts this many frames further along the camera path, so the
# replicas do not render identical frames
FRAME_STRIDE = 7


def replica_first_frame(rank: int) -> int:
    return rank * FRAME_STRIDE


def max_over_ranks(values, world: int, device=None):
    """Element-wise maximum of a list of floats over all ranks (one all-reduce;
    every rank must call it at the same point)."""
    import torch
    t = torch.tensor(list(values), dtype=torch.float64, device=device)
    if world > 1:
        import torch.distributed as dist
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.tolist()


def job_throughput(units_per_rank: float, world: int, seconds: float) -> float:
    """Units of the whole job (all ranks) per second, timed by the slowest rank."""
    if seconds <= 0:
        raise ValueError("non-positive time")
    return units_per_rank * world / seconds
