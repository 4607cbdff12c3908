"""Multi-GPU sharding of independent work (one process per GPU).

Tiles (with their halos) and DEM requests are independent units, so the path
needs no data exchange between GPUs: each rank takes a share of the units,
interpolates it on its own device, and only timing and (optionally) result
assembly cross ranks.  The reference runs one process over all work packages
in turn (binRun, terranni.cpp:394-426); this module is what replaces that loop
when several GPUs share the work.

- ``partition_by_cost``: longest-processing-time assignment of units to ranks
  by an estimated cost (cells + points of a tile), deterministic, so every
  rank computes the same partition without communicating;
- ``route_least_loaded``: the rank a new request goes to, for serving;
- ``max_over_ranks`` / ``gather_to_root``: the only collectives, for the
  timing rule (slowest rank) and for assembling results on rank 0.
"""
from __future__ import annotations

import heapq

import numpy as np


def tile_cost(side_cols, side_rows, points):
    """Estimated work of a tile: cells plus points (both passes are linear in
    them; lakes add span work that scales with the cells)."""
    return int(side_cols) * int(side_rows) + int(points)


def partition_by_cost(costs, world):
    """Assigns unit k to a rank: units in decreasing cost, each to the rank
    with the least assigned cost so far (ties: lowest rank).  Returns one
    sorted index list per rank."""
    if world < 1:
        raise ValueError("world must be >= 1")
    costs = np.asarray(costs, dtype=np.int64)
    order = sorted(range(len(costs)), key=lambda k: (-int(costs[k]), k))
    heap = [(0, r) for r in range(world)]
    parts = [[] for _ in range(world)]
    for k in order:
        load, r = heapq.heappop(heap)
        parts[r].append(k)
        heapq.heappush(heap, (load + int(costs[k]), r))
    return [sorted(p) for p in parts]


def route_least_loaded(loads, cost):
    """Rank for a new unit of `cost` given the ranks' outstanding loads
    (list, updated in place); ties go to the lowest rank."""
    r = min(range(len(loads)), key=lambda k: (loads[k], k))
    loads[r] += int(cost)
    return r


def max_over_ranks(x, device=None):
    """Largest value of x over all ranks (x itself without a process group)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device or "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_to_root(obj):
    """Every rank's object on rank 0 (list by rank), None elsewhere."""
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return [obj]
    out = [None] * dist.get_world_size() if dist.get_rank() == 0 else None
    dist.gather_object(obj, out, dst=0)
    return out
