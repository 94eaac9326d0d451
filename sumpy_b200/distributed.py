"""Host-side plumbing for running on several GPUs of one node.

sumpy's distributed FMM (sumpy/distributed.py) partitions one tree across
MPI ranks through boxtree. This build does not partition a tree: a single
problem runs on one GPU and several GPUs run independent problems
(replicas, or a batch of independent point sets split across ranks). What
is shared between ranks is only host bookkeeping, which lives here:
process-group set-up from the torchrun environment, the max-over-ranks
reduction of step times, and the assignment of independent problems to
ranks (longest first, to the least loaded rank).
"""
from __future__ import annotations

import datetime
import os

import torch
import torch.distributed as dist


def env_ranks():
    """(rank, world_size, local_rank) from the torchrun environment."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend="nccl", timeout_s=300):
    """Initialise the default process group when WORLD_SIZE > 1; return
    (rank, world_size, local_rank)."""
    rank, world, local = env_ranks()
    if world > 1 and not dist.is_initialized():
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return rank, world, local


def max_over_ranks(value, device=None):
    """Maximum of a float over all ranks (identity on one rank)."""
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64,
                     device=device if device is not None else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def shard_problems(costs, world):
    """Assign independent problems to ranks: largest cost first, each to the
    currently least loaded rank. Returns a list of index lists, one per rank."""
    order = sorted(range(len(costs)), key=lambda i: -costs[i])
    load = [0.0] * world
    out = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        out[r].append(i)
        load[r] += costs[i]
    return [sorted(x) for x in out]
