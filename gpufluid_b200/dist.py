"""Multi-GPU coordination: one process per GPU, replicas and scene shards.

The single-scene substep does not shard within this build: N GPUs run N
independent replicas, timed on the device, and the job's time is the maximum
over ranks.  A batch of independent scenes shards by scene: ``shard_scenes``
splits the scenes over the ranks by particle count (longest-processing-time
greedy bin packing), each rank steps its shard with no exchange, and the
per-scene metrics are gathered once at the end.  The process group is
``torch.distributed`` (NCCL between GPUs, gloo on CPU), with a short timeout
so that ranks waiting for a lost peer end with an error.
"""
from __future__ import annotations

import datetime
import heapq
import os
from typing import List, Sequence


class Ranks:
    """Rank, world size and the few collectives the replicas need.  With a
    world of one no process group is created and every collective is local."""

    def __init__(self, backend: str = "nccl", device=None, timeout_s: float = 120.0):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local_rank = int(os.environ.get("LOCAL_RANK", "0"))
        self.backend = backend
        self.device = device
        self._dist = None
        if self.world > 1:
            import torch.distributed as dist
            kw = {"timeout": datetime.timedelta(seconds=timeout_s)}
            if backend == "nccl" and device is not None:
                import torch
                kw["device_id"] = torch.device(device)
            dist.init_process_group(backend, **kw)
            self._dist = dist

    def barrier(self):
        if self._dist is not None:
            self._dist.barrier()

    def _tensor(self, values):
        import torch
        dev = self.device if self.backend == "nccl" else "cpu"
        return torch.tensor(values, dtype=torch.float64, device=dev)

    def max(self, x: float) -> float:
        """Maximum of x over the ranks (the job's time of a timed region)."""
        if self._dist is None:
            return float(x)
        t = self._tensor([x])
        self._dist.all_reduce(t, op=self._dist.ReduceOp.MAX)
        return float(t.item())

    def sum(self, x: float) -> float:
        if self._dist is None:
            return float(x)
        t = self._tensor([x])
        self._dist.all_reduce(t, op=self._dist.ReduceOp.SUM)
        return float(t.item())

    def gather(self, values: Sequence[float]) -> List[List[float]]:
        """Every rank's list of values (lists of equal length), on every rank."""
        if self._dist is None:
            return [list(map(float, values))]
        t = self._tensor(list(values))
        out = [self._tensor([0.0] * len(values)) for _ in range(self.world)]
        self._dist.all_gather(out, t)
        return [[float(v) for v in o.cpu().tolist()] for o in out]

    def close(self):
        if self._dist is not None:
            self._dist.destroy_process_group()
            self._dist = None


def shard_scenes(particle_counts: Sequence[int], world: int) -> List[List[int]]:
    """Split scene indices over `world` ranks, largest scenes first, each to
    the rank with the fewest particles so far (ties to the lowest rank);
    every rank's list is in ascending scene order."""
    if world < 1:
        raise ValueError("world must be >= 1")
    heap = [(0, r) for r in range(world)]
    shards: List[List[int]] = [[] for _ in range(world)]
    order = sorted(range(len(particle_counts)), key=lambda i: (-int(particle_counts[i]), i))
    for i in order:
        load, r = heapq.heappop(heap)
        shards[r].append(i)
        heapq.heappush(heap, (load + int(particle_counts[i]), r))
    return [sorted(s) for s in shards]
