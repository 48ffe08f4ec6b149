"""Sharding a sweep of independent problems over ranks (one GPU each).

Problems of a sweep share nothing, so a multi-GPU sweep needs no data-path
collective: each rank takes a subset and runs it as its own batch.  The
subsets come from a greedy longest-processing-time bin packing on each
problem's cost (cells x steps): problems in decreasing cost order, each to
the currently lightest rank (ties to the lowest rank).  Every rank computes
the same partition from the same costs, so no exchange of the assignment is
needed either; results are gathered on the host afterwards.
"""
from __future__ import annotations

import heapq


def partition(costs, world: int) -> list[list[int]]:
    """Indices of `costs` per rank (each list in increasing index order)."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda q: (-costs[q], q))
    heap = [(0, r) for r in range(world)]
    heapq.heapify(heap)
    out = [[] for _ in range(world)]
    for q in order:
        load, r = heapq.heappop(heap)
        out[r].append(q)
        heapq.heappush(heap, (load + costs[q], r))
    return [sorted(x) for x in out]


def imbalance(costs, parts) -> float:
    """Largest rank load over the mean load (1.0 = perfect balance)."""
    loads = [sum(costs[q] for q in p) for p in parts]
    mean = sum(loads) / max(len(loads), 1)
    return max(loads) / mean if mean else 1.0


def variant_costs(seeds, steps: int, spread: bool = False) -> list[int]:
    """cells x steps of each inverted-F variant (workloads.ifa_variant with
    `spread`), from its grid alone."""
    from .scenario import DEFAULTS, build_grid
    from .workloads import ifa_variant
    out = []
    for s in seeds:
        scn = ifa_variant(int(s), steps=steps, spread=spread)
        cell = dict(DEFAULTS["cell"], **(scn.get("cell") or {}))
        g = build_grid(cell["dx"], cell["dy"], cell["dz"], scn["boundary"], scn.get("bricks") or [],
                       scn.get("spheres") or [], scn.get("courantFactor", DEFAULTS["courantFactor"]), steps)
        out.append(g.nx * g.ny * g.nz * steps)
    return out
