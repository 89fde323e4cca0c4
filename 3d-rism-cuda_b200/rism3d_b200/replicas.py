"""Multi-GPU plumbing for independent solves (one process per GPU,
torch.distributed for the few host-level exchanges; no collective touches
the solve itself).

A single 3D-RISM solve is not sharded: one 256^3 solve fits one GPU and is
transform-bound.  N GPUs run N independent solves (replicas) or split a
batch of small solutes by estimated cost; the only exchanges are a barrier
around timed regions, the max of the per-rank times, and the sum of the
per-rank unit counts."""
from __future__ import annotations

import heapq


def partition_by_cost(costs, world):
    """Longest-processing-time greedy split of units with the given costs
    over `world` ranks: returns one sorted index list per rank; every unit
    appears exactly once and the largest rank load is within one unit's cost
    of the mean."""
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    heap = [(0.0, r) for r in range(world)]
    heapq.heapify(heap)
    parts = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        parts[r].append(i)
        heapq.heappush(heap, (load + costs[i], r))
    return [sorted(p) for p in parts]


def solve_cost(grid_points, natoms):
    """Relative cost of one solute: the iteration streams the grid (the
    atoms only enter the one-off potential and energy integrals)."""
    return float(grid_points) + 64.0 * natoms


def _dev(dist_device):
    import torch
    return torch.device(dist_device) if dist_device else torch.device("cpu")


def max_over_ranks(x, dist_device=None):
    """Max of a per-rank scalar (timings: the slowest rank sets the time)."""
    import torch
    import torch.distributed as D
    if not (D.is_available() and D.is_initialized()):
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=_dev(dist_device))
    D.all_reduce(t, op=D.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x, dist_device=None):
    """Sum of a per-rank count (units processed by the whole job)."""
    import torch
    import torch.distributed as D
    if not (D.is_available() and D.is_initialized()):
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=_dev(dist_device))
    D.all_reduce(t, op=D.ReduceOp.SUM)
    return float(t.item())


def job_rate(units_this_rank, seconds_this_rank, dist_device=None):
    """Whole-job throughput: all ranks' units over the slowest rank's time."""
    units = sum_over_ranks(units_this_rank, dist_device)
    secs = max_over_ranks(seconds_this_rank, dist_device)
    return units / secs if secs > 0 else 0.0
