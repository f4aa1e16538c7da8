"""One process per GPU for independent replicas (and the one real exchange).

The PM path does not shard: every rank runs its own simulation (its own
noise seed) and the job's throughput is the sum over ranks, timed as the
maximum over ranks.  The only data exchange is the all-reduce that averages
the learned correction's parameter gradient across ranks training on
different seed pairs (about 10^4 numbers per optimiser step).  Launch with
``torchrun`` (RANK / WORLD_SIZE / LOCAL_RANK / MASTER_ADDR / MASTER_PORT);
NCCL on GPUs, gloo on CPU.
"""
from __future__ import annotations

import datetime
import os

import torch


def setup(backend=None, timeout_s=600):
    """(rank, world, local_rank); initialises the process group when world > 1."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1 and not torch.distributed.is_initialized():
        import torch.distributed as dist
        if backend is None:
            backend = "nccl" if torch.cuda.is_available() else "gloo"
        kw = {}
        if backend == "nccl":
            torch.cuda.set_device(local)
            kw["device_id"] = torch.device("cuda", local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s), **kw)
    return rank, world, local


def _device():
    import torch.distributed as dist
    return torch.device("cuda", torch.cuda.current_device()) if dist.get_backend() == "nccl" else torch.device("cpu")


def barrier(world):
    if world > 1:
        torch.distributed.barrier()


def max_over_ranks(x, world):
    """Maximum of a float over ranks (the job's time is its slowest rank's)."""
    if world == 1:
        return float(x)
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=_device())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x, world):
    if world == 1:
        return float(x)
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=_device())
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def average_gradient(grad, world):
    """In-place mean of a gradient tensor over ranks (data-parallel training
    of the learned correction); the tensor must live on the backend's device."""
    if world > 1:
        import torch.distributed as dist
        dist.all_reduce(grad, op=dist.ReduceOp.SUM)
        grad /= world
    return grad


def replica_seed(base, rank):
    """Seed of rank's independent replica."""
    return int(base) + int(rank)


def teardown(world):
    if world > 1 and torch.distributed.is_initialized():
        torch.distributed.destroy_process_group()
