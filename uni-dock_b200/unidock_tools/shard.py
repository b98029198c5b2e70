"""Ligand sharding across GPUs (one process per GPU, no data-path collective).

(ligand, chain) work items are independent, so a screen splits by ligand:
each rank searches its own share against its own copy of the grid maps and
writes its own outputs.  Shares are balanced by a per-ligand cost (atoms x
pairs x BFGS steps is a good proxy), largest first onto the least-loaded rank,
which is deterministic, so every rank computes the same partition without
communicating.
"""
from __future__ import annotations

import heapq


def shard(n_items: int, rank: int, world: int, cost=None) -> list[int]:
    """Indices (ascending) of the items rank `rank` of `world` processes.
    Without costs: round robin.  With costs: longest-processing-time-first."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank must be in [0, world)")
    if cost is None:
        return list(range(rank, n_items, world))
    if len(cost) != n_items:
        raise ValueError("one cost per item")
    order = sorted(range(n_items), key=lambda i: (-float(cost[i]), i))
    heap = [(0.0, r) for r in range(world)]
    owner = [0] * n_items
    for i in order:
        load, r = heapq.heappop(heap)
        owner[i] = r
        heapq.heappush(heap, (load + float(cost[i]), r))
    return [i for i in range(n_items) if owner[i] == rank]


def ligand_cost(ligand) -> float:
    """Search cost proxy of an engine.Ligand: BFGS steps x (atoms + pairs)."""
    return float(ligand.local_steps * (ligand.n_atoms + ligand.n_pairs))
