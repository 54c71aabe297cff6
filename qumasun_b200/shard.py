"""Sharding of independent solves across ranks (one process per GPU).

k-points and cells never communicate during an eigensolve, so a multi-GPU run
partitions them: units are assigned to ranks by greedy longest-processing-time
(largest estimated cost first, each to the currently least-loaded rank), every
rank solves its own units on its own GPU with no collective on the data path,
and only the small results (eigenvalues, iteration counts, timings) travel to
rank 0 through the process group's object gather.

The cost model per unit is N_grid * n_states * (16 bytes of stencil traffic +
projector bytes) + n_states^2 * N_grid (Gram and rotation), the shape that
dominates one LOBPCG iteration.
"""
from __future__ import annotations

import heapq


def unit_cost(n_grid, n_states, n_atoms=0, sphere_points_per_atom=13_700, complex_states=False):
    """Relative cost of one LOBPCG solve on a cell."""
    c = 2 if complex_states else 1
    stencil = n_grid * n_states * 16 * c
    proj = n_atoms * sphere_points_per_atom * n_states * 8 * 4 * c
    gemm = (3 * n_states) ** 2 * n_grid * c * c
    return float(stencil + proj + gemm)


def lpt_assign(costs, n_ranks):
    """Greedy longest-processing-time assignment: returns one list of unit indices per
    rank (each list in the order the rank should run them) and the per-rank loads.
    Ties are broken by unit index and rank index, so every rank computes the same
    assignment from the same costs."""
    if n_ranks <= 0:
        raise ValueError("n_ranks must be positive")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    heap = [(0.0, r) for r in range(n_ranks)]
    heapq.heapify(heap)
    parts = [[] for _ in range(n_ranks)]
    loads = [0.0] * n_ranks
    for i in order:
        load, r = heapq.heappop(heap)
        parts[r].append(i)
        loads[r] = load + costs[i]
        heapq.heappush(heap, (loads[r], r))
    return parts, loads


def run_sharded(costs, solve, group=None):
    """Solve units `0..len(costs)-1` across the ranks of `group` (torch.distributed;
    None = one process): rank r runs solve(i) for its LPT share and rank 0 receives
    {i: result} for all units (other ranks receive None). `solve` must not call any
    collective; the only collective is the gather of the results."""
    import torch.distributed as dist
    if group is None and not (dist.is_available() and dist.is_initialized()):
        return {i: solve(i) for i in lpt_assign(costs, 1)[0][0]}
    ws = dist.get_world_size(group)
    rank = dist.get_rank(group)
    parts, _ = lpt_assign(costs, ws)
    mine = {i: solve(i) for i in parts[rank]}
    gathered = [None] * ws if rank == 0 else None
    dist.gather_object(mine, gathered, dst=0, group=group)
    if rank != 0:
        return None
    out = {}
    for part in gathered:
        out.update(part)
    return out
