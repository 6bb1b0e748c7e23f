"""Multi-GPU sharding of the encode/decode path: one process per GPU.

Every 4x4 block is independent, so the path needs no exchange step: textures
are partitioned across ranks and each rank encodes its share on its own GPU.
The partition is deterministic and balances estimated cost (largest first,
each texture to the currently lightest rank), so every rank computes the same
assignment without communicating. ``torch.distributed`` (NCCL on GPUs, gloo
on CPU) is used only for the barrier and the max-over-ranks time.
"""

from __future__ import annotations

import heapq
from typing import Callable, Sequence, TypeVar

T = TypeVar("T")


def shard(items: Sequence[T], world: int, rank: int, cost: Callable[[T], float]) -> list[int]:
    """Indices of ``items`` assigned to ``rank`` (greedy LPT on ``cost``)."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError("rank out of range")
    order = sorted(range(len(items)), key=lambda i: (-cost(items[i]), i))
    heap = [(0.0, r) for r in range(world)]
    mine = []
    for i in order:
        load, r = heapq.heappop(heap)
        if r == rank:
            mine.append(i)
        heapq.heappush(heap, (load + cost(items[i]), r))
    return sorted(mine)


def max_over_ranks(x: float) -> float:
    """Max of a per-rank scalar (e.g. a timing) over the process group; the
    identity without one."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return x
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def block_cost(width: int, height: int, fmt: str = "bc1", level: int = 5) -> float:
    """Relative encode cost of a texture (blocks x per-block cost of its class)."""
    nb = ((width + 3) // 4) * ((height + 3) // 4)
    if fmt in ("bc4", "bc5"):
        return nb * 0.2
    return nb * (13.0 if level >= 13 else 2.8 if level >= 9 else 1.0)
