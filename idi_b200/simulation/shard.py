"""Sharding images across ranks (one process per GPU).

Images are independent, so multi-GPU runs need no data-path collective:
each rank simulates its own images.  The helpers here assign images to
ranks -- contiguous ranges, or balanced by emitter count for uneven batches
(longest-processing-time greedy) -- and reduce a timing to its maximum over
ranks, which is the only collective a benchmark needs.
"""

from __future__ import annotations

import heapq
from typing import List, Sequence, Tuple


def shard_range(n: int, rank: int, world: int) -> Tuple[int, int]:
    """Contiguous [start, stop) of n items for `rank`; sizes differ by at most one."""
    if world < 1 or not 0 <= rank < world or n < 0:
        raise ValueError("bad shard arguments")
    base, extra = divmod(n, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def shard_by_cost(counts: Sequence[int], world: int) -> List[List[int]]:
    """Images per rank, balancing the sum of emitter counts (greedy, largest first).

    Deterministic: ties are broken by image index and rank."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(counts)), key=lambda i: (-int(counts[i]), i))
    heap = [(0, r) for r in range(world)]
    out: List[List[int]] = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + int(counts[i]), r))
    for lst in out:
        lst.sort()
    return out


def max_over_ranks(value: float) -> float:
    """Maximum of a float over the default process group (identity without one)."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    dev = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend() == "nccl" else torch.device("cpu")
    t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
