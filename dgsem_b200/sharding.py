"""Placement of independent meshes of a batch on the ranks of a job (one
process per GPU): the batched mode's natural sharding unit is the mesh, and
meshes never exchange data, so the only decision is which rank advances
which mesh.  The cost of a mesh is its stage work, elements x n^d nodes x
(d (n - 1) + 2 d) flux evaluations per node (two-point fluxes along each
line through the node plus the face fluxes); meshes are placed by the
longest-processing-time rule (largest first, onto the least-loaded rank),
which keeps the most loaded rank within 4/3 of the optimum.  The placement
is a pure function of the mesh list, so every rank computes the same one
without communication.
"""
from __future__ import annotations

import heapq
from typing import Sequence


def mesh_cost(cells: Sequence[int], polydeg: int) -> float:
    """Relative stage cost of one mesh of `cells` elements at degree `polydeg`."""
    d = len(cells)
    n = polydeg + 1
    elems = 1
    for c in cells:
        elems *= int(c)
    return float(elems * n ** d * (d * (n - 1) + 2 * d))


def assign_meshes(costs: Sequence[float], world_size: int) -> list[list[int]]:
    """Indices of the meshes each rank advances (each list ascending); every
    mesh is on exactly one rank."""
    if world_size < 1:
        raise ValueError("world_size must be at least 1")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    heap = [(0.0, r) for r in range(world_size)]
    out: list[list[int]] = [[] for _ in range(world_size)]
    for i in order:
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + float(costs[i]), r))
    return [sorted(v) for v in out]


def local_meshes(specs, rank: int, world_size: int):
    """The (index, spec) pairs of `specs` ((cells, polydeg, ...) tuples) that
    rank `rank` of `world_size` advances."""
    costs = [mesh_cost(s[0], s[1]) for s in specs]
    return [(i, specs[i]) for i in assign_meshes(costs, world_size)[rank]]
