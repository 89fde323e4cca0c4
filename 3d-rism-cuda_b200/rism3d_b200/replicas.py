"""Multi-GPU plumbing for independent solves (one process per GPU,
torch.distributed for the few host-level exchanges; no collective touches
the solve itself).

A single 3D-RISM solve is not sharded: one 256^3 solve fits one GPU and is
transform-bound.  N GPUs run N independent solves (replicas) or split a
batch of small solutes by estimated cost; the only exchanges are a barrier
around timed regions, the max of the per-rank times, and the sum of the
per-rank unit counts, and one gather of the per-solute result scalars of a
split batch back into input order."""
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


# Per-solute result scalars carried back from a split batch, in this order.
RESULT_KEYS = ("sfe_sc", "sfe_sc_hnc", "sfe_gf", "pmv", "pressure", "correction", "se",
               "se_lj", "se_es", "rms", "iterations", "iterations_fp32", "status")
_INT_KEYS = {"iterations", "iterations_fp32", "status"}


def gather_results(results, indices, n_total, dist_device=None):
    """Gather every rank's per-solute results into input order.

    ``results[i]`` is the result dict of solute ``indices[i]`` (this rank's
    part of a batch split by ``partition_by_cost``).  One all-gather of a
    fixed-width float64 table (index + the scalars of RESULT_KEYS), padded
    to the largest part, brings every rank's rows to every rank; the return
    value is a list of ``n_total`` dicts (one per solute of the whole batch,
    in input order) on every rank.  Raises if a solute is missing or
    claimed twice.  Without an initialised process group the local results
    are simply reordered."""
    import torch
    import torch.distributed as D
    if len(results) != len(indices):
        raise ValueError("one result per index")
    width = 1 + len(RESULT_KEYS)
    dev = _dev(dist_device)
    rows = torch.full((len(results), width), float("nan"), dtype=torch.float64)
    for r, (i, res) in enumerate(zip(indices, results)):
        rows[r, 0] = float(i)
        for k, key in enumerate(RESULT_KEYS):
            rows[r, 1 + k] = float(res[key])
    if D.is_available() and D.is_initialized():
        world = D.get_world_size()
        cnt = torch.tensor([len(results)], dtype=torch.int64, device=dev)
        cnts = [torch.zeros_like(cnt) for _ in range(world)]
        D.all_gather(cnts, cnt)
        cap = max(1, max(int(c.item()) for c in cnts))
        pad = torch.full((cap, width), -1.0, dtype=torch.float64)
        pad[: len(results)] = rows
        pad = pad.to(dev)
        parts = [torch.empty_like(pad) for _ in range(world)]
        D.all_gather(parts, pad)
        table = torch.cat([p[: int(c.item())].cpu() for p, c in zip(parts, cnts)])
    else:
        table = rows
    out = [None] * n_total
    for row in table.tolist():
        i = int(row[0])
        if not 0 <= i < n_total or out[i] is not None:
            raise ValueError("solute %d gathered twice or out of range" % i)
        out[i] = {key: (int(v) if key in _INT_KEYS else v)
                  for key, v in zip(RESULT_KEYS, row[1:])}
    missing = [i for i, r in enumerate(out) if r is None]
    if missing:
        raise ValueError("solutes missing from the gather: %s" % missing[:8])
    return out
