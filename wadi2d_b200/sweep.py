"""Storm sweeps over several GPUs: one process per GPU, the runs shared out by their estimated cost, each rank
stepping its share as one batch, and the per-run results gathered on rank 0 at the end. Runs are independent, so
there is no exchange while they step (weak scaling); the only collective is the final gather.

The reference runs a study's storms one after another on one device (wadi2d/arf.py:346-372); its results table
(design_table, wadi2d/arf.py:240-266) reads each run's peaks. ``gather_results`` gives rank 0 the same per-run
records in the study's order.
"""

from __future__ import annotations

import heapq

import numpy as np


def run_cost(cells: float, simulated_s: float, dx: float) -> float:
    """Estimated cell-steps of a run: cells x simulated time / dx (the step is proportional to the cell size)."""
    return float(cells) * float(simulated_s) / float(dx)


def partition(costs, world: int) -> list[list[int]]:
    """Longest-processing-time split of runs over ``world`` ranks: runs by falling cost, each to the least loaded rank
    (ties to the lower rank). Deterministic; each rank's list is in the study's order."""
    if world < 1:
        raise ValueError("world must be at least 1")
    costs = np.asarray(costs, np.float64)
    order = sorted(range(costs.size), key=lambda r: (-costs[r], r))
    heap = [(0.0, rank) for rank in range(world)]
    out: list[list[int]] = [[] for _ in range(world)]
    for r in order:
        load, rank = heapq.heappop(heap)
        out[rank].append(r)
        heapq.heappush(heap, (load + float(costs[r]), rank))
    return [sorted(x) for x in out]


def imbalance(costs, parts: list[list[int]]) -> float:
    """Largest rank load over the mean load (1.0 = even)."""
    costs = np.asarray(costs, np.float64)
    loads = np.array([costs[p].sum() for p in parts])
    return float(loads.max() / max(loads.mean(), 1e-300))


def gather_results(local: dict, world: int, rank: int, group=None) -> dict | None:
    """Each rank's {run index: record} to rank 0, merged in run order; other ranks get None. One collective
    (gather_object), taken by every rank in the same order."""
    if world == 1:
        return dict(sorted(local.items()))
    import torch.distributed as dist

    box = [None] * world if rank == 0 else None
    dist.gather_object(local, box, dst=0, group=group)
    if rank != 0:
        return None
    merged: dict = {}
    for part in box:
        for k, v in part.items():
            if k in merged:
                raise ValueError(f"run {k} came back from two ranks")
            merged[k] = v
    return dict(sorted(merged.items()))
