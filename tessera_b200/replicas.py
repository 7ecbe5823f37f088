"""Multi-GPU layer: replicas and scene parallelism, no data-path collective.

A single MPM scene does not shard without a halo exchange (a grid-block
momentum sum after P2G and particle migration after G2P), which none of the
workloads needs; scenes are independent, so multi-GPU work is placed by scene:
one process per GPU, each advancing its own scenes (or its own replica of the
benchmark scene) in its own batch.  The only cross-rank traffic is bookkeeping:
the max over ranks of a device time and the sum of the work done, through
torch.distributed (NCCL on GPUs, gloo on CPU for the tests).

Placement is deterministic and needs no communication: every rank computes
the same assignment from the same list of scene footprints (longest
processing time first onto the least-loaded rank).
"""

from __future__ import annotations

import heapq


def place_by_footprint(sizes, world: int) -> list[int]:
    """Owner rank of each item: largest first onto the least-loaded rank
    (ties to the lower rank).  Identical on every rank."""
    if world < 1:
        raise ValueError("world must be at least 1")
    order = sorted(range(len(sizes)), key=lambda i: (-float(sizes[i]), i))
    heap = [(0.0, r) for r in range(world)]
    owner = [0] * len(sizes)
    for i in order:
        load, r = heapq.heappop(heap)
        owner[i] = r
        heapq.heappush(heap, (load + float(sizes[i]), r))
    return owner


def my_items(sizes, world: int, rank: int) -> list[int]:
    """Indices of the items this rank owns, in their original order."""
    owner = place_by_footprint(sizes, world)
    return [i for i, r in enumerate(owner) if r == rank]


class Reducer:
    """Max / sum of host floats over the ranks of the default process group
    (a pass-through with one rank).  `device` is where the backend wants its
    tensors: "cuda" for NCCL, "cpu" for gloo."""

    def __init__(self, world: int, device: str = "cuda"):
        self.world = int(world)
        self.device = device

    def _reduce(self, value: float, op_name: str) -> float:
        if self.world == 1:
            return float(value)
        import torch
        import torch.distributed as dist

        t = torch.tensor([float(value)], dtype=torch.float64, device=self.device)
        dist.all_reduce(t, op=getattr(dist.ReduceOp, op_name))
        return float(t.item())

    def max(self, value: float) -> float:
        return self._reduce(value, "MAX")

    def sum(self, value: float) -> float:
        return self._reduce(value, "SUM")

    def barrier(self) -> None:
        if self.world > 1:
            import torch.distributed as dist

            dist.barrier()
