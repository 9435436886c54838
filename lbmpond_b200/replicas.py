"""Multi-process plumbing for runs on several GPUs (one process per GPU).

The PonD step has no exchange between independent problems, so N GPUs run N
replicas (one box each) or split a batch of independent 1D problems; the only
collectives are the barrier around a timed region and the maximum of the
ranks' times.  torch.distributed is the transport: NCCL on GPUs, gloo on CPU
(tests).
"""
from __future__ import annotations

import datetime
import os

import numpy as np


def setup(backend: str = "nccl", timeout_s: float = 600.0):
    """Join the process group the launcher describes (RANK, WORLD_SIZE,
    LOCAL_RANK, MASTER_ADDR/PORT); returns (rank, local_rank, world, dist or
    None for a single process)."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world == 1:
        return rank, local, world, None
    import torch
    import torch.distributed as dist
    kw = {"timeout": datetime.timedelta(seconds=timeout_s)}
    if backend == "nccl":
        torch.cuda.set_device(local)
        kw["device_id"] = torch.device("cuda", local)
    dist.init_process_group(backend, **kw)
    return rank, local, world, dist


def _device(dist):
    import torch
    return torch.device("cuda", torch.cuda.current_device()) if dist.get_backend() == "nccl" else torch.device("cpu")


def max_over_ranks(dist, value: float) -> float:
    """The largest value any rank holds (every rank gets it)."""
    if dist is None:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=_device(dist))
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(dist, value: float) -> float:
    if dist is None:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=_device(dist))
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def barrier(dist):
    if dist is not None:
        dist.barrier()


def partition_problems(lengths, world: int):
    """Split independent problems over `world` ranks with balanced node
    counts: longest first, each to the rank with the fewest nodes so far
    (ties to the lower rank).  Returns one sorted index array per rank;
    every problem appears exactly once."""
    lengths = np.asarray(lengths, dtype=np.int64)
    load = np.zeros(world, dtype=np.int64)
    owner = np.empty(lengths.size, dtype=np.int64)
    for p in np.argsort(-lengths, kind="stable"):
        r = int(np.argmin(load))
        owner[p] = r
        load[r] += lengths[p]
    return [np.flatnonzero(owner == r) for r in range(world)]
