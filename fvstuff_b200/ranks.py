"""One process per GPU.  The path does not shard a grid (no spatial
decomposition): N GPUs run N replicas of a grid, or split a batch's
instances between them.  There is no data-path collective; the only
collectives are the max over ranks of a measured time and sums of counters,
taken at the end of a run.

Works with the NCCL backend on GPUs and with gloo on CPU (the tests run two
gloo ranks); rendezvous through MASTER_ADDR / MASTER_PORT as torchrun sets
them.
"""
from __future__ import annotations

import datetime
import heapq
import os
from typing import Sequence


def env() -> tuple[int, int, int]:
    """(rank, world size, local rank) from the torchrun environment."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend: str | None = None, timeout_s: float = 120.0):
    """Join the process group when WORLD_SIZE > 1; returns torch.distributed
    or None for a single process.  A short timeout makes a rank that never
    arrives at a collective an error instead of a hang."""
    _, world, _ = env()
    if world <= 1:
        return None
    import torch
    import torch.distributed as dist
    if backend is None:
        backend = "nccl" if torch.cuda.is_available() else "gloo"
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return dist


def _reduce(x: float, dist, op) -> float:
    if dist is None:
        return float(x)
    import torch
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=op)
    return float(t.item())


def max_over_ranks(x: float, dist=None) -> float:
    return _reduce(x, dist, dist.ReduceOp.MAX if dist else None)


def sum_over_ranks(x: float, dist=None) -> float:
    return _reduce(x, dist, dist.ReduceOp.SUM if dist else None)


def gather(obj, dist=None) -> list:
    """Every rank's `obj`, in rank order (a single process: [obj])."""
    if dist is None:
        return [obj]
    out = [None] * dist.get_world_size()
    dist.all_gather_object(out, obj)
    return out


def shard_by_work(costs: Sequence[float], rank: int, world: int) -> list[int]:
    """Indices of the items rank `rank` takes: longest-processing-time-first
    assignment (each item, largest cost first, to the least-loaded rank; ties
    to the lower rank), so every rank computes the same partition and the
    largest load exceeds the mean by at most the largest single cost."""
    if world <= 1:
        return list(range(len(costs)))
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    heap = [(0.0, r) for r in range(world)]
    mine = []
    for i in order:
        load, r = heapq.heappop(heap)
        if r == rank:
            mine.append(i)
        heapq.heappush(heap, (load + costs[i], r))
    return sorted(mine)


def finish(dist) -> None:
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
