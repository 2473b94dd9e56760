"""Replicas: the multi-GPU form of the query path.

Points are independent and no step of the path exchanges data, so N GPUs run
N replicas, one process per GPU (torchrun), each with its own index and its
own points (weak scaling), or with one shard of a common point array (strong
scaling).  The only collectives are for measurement: the slowest rank's time
and a barrier around the timed region.  No collective touches the data path.
"""
import os


def world():
    """(rank, world size, local rank) from the torchrun environment."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def shard(n, rank, size):
    """[start, end) of rank's contiguous share of n points (sizes differ by at most one)."""
    base, extra = divmod(n, size)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def max_over_ranks(value, device=None):
    """The largest value over all ranks (a time: the job ends with its slowest rank)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier():
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.barrier()
