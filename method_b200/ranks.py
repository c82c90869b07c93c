"""One process per GPU: rank discovery, barrier, max-over-ranks device timing
and the partition of an ensemble's members over ranks.

The single-domain time step has no exchange step on one GPU, so several GPUs
run independent replicas; an ensemble's members are independent, so they are
split over the ranks by cell count (greedy longest-processing-time first) and
each rank advances its own share with no collective on the data path.  The
only collectives are the barrier around timed regions and the max-over-ranks
reduction of the measured times.
"""
from __future__ import annotations

import datetime
import heapq
import os


def rank_env():
    """(rank, world_size, local_rank) from the torchrun environment."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


class Ranks:
    """Process group of a multi-rank run (a no-op for one process)."""

    def __init__(self, backend: str = "nccl", timeout_s: float = 120.0):
        import torch
        self.torch = torch
        self.rank, self.world, self.local = rank_env()
        self.backend = backend
        self.dist = None
        if backend == "nccl":
            torch.cuda.set_device(self.local)
        if self.world > 1:
            import torch.distributed as dist
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
            self.dist = dist

    def barrier(self):
        if self.dist:
            self.dist.barrier()
        if self.backend == "nccl":
            self.torch.cuda.synchronize()

    def max(self, x: float) -> float:
        """The maximum of x over all ranks (every rank gets it)."""
        if not self.dist:
            return float(x)
        dev = "cuda" if self.backend == "nccl" else "cpu"
        t = self.torch.tensor([float(x)], device=dev, dtype=self.torch.float64)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def sum(self, x: float) -> float:
        if not self.dist:
            return float(x)
        dev = "cuda" if self.backend == "nccl" else "cpu"
        t = self.torch.tensor([float(x)], device=dev, dtype=self.torch.float64)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM)
        return float(t.item())

    def close(self):
        if self.dist:
            self.dist.barrier()
            self.dist.destroy_process_group()
            self.dist = None


def lpt_partition(costs, n_parts):
    """Greedy longest-processing-time-first split of items with the given
    costs into n_parts lists of item indices (each list ascending).  Ties go
    to the lower part index, so every rank computes the same split."""
    if n_parts < 1:
        raise ValueError("n_parts must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    heap = [(0, p) for p in range(n_parts)]
    parts = [[] for _ in range(n_parts)]
    for i in order:
        load, p = heapq.heappop(heap)
        parts[p].append(i)
        heapq.heappush(heap, (load + costs[i], p))
    return [sorted(p) for p in parts]
