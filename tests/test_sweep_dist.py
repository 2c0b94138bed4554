"""Sweeps over several ranks, on CPU: the cost split of the runs, and the gather of per-run records to rank 0 over
two gloo ranks (the same collective the GPU sweep takes over NCCL)."""

from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from wadi2d_b200 import workloads
from wadi2d_b200.sweep import gather_results, imbalance, partition, run_cost


def test_partition_covers_every_run_once_and_balances():
    rng = np.random.default_rng(0)
    costs = rng.lognormal(0.0, 1.5, 64)
    for world in (1, 2, 3, 8):
        parts = partition(costs, world)
        flat = sorted(r for p in parts for r in p)
        assert flat == list(range(64))
        assert all(p == sorted(p) for p in parts)
        # LPT: the largest load is within the largest single run of the mean
        loads = [costs[p].sum() for p in parts]
        assert max(loads) <= np.mean(loads) + costs.max() + 1e-9
    assert imbalance(costs, partition(costs, 2)) < 1.05
    assert partition(costs, 4) == partition(costs, 4)


def test_partition_of_the_ensemble_by_estimated_cell_steps():
    specs = workloads.ensemble(64)
    costs = [run_cost(s.side**2, (s.duration_min + 30.0) * 60.0, s.dx) for s in specs]
    parts = partition(costs, 8)
    assert imbalance(costs, parts) < 1.25
    assert sum(len(p) for p in parts) == 64


def test_partition_rejects_no_ranks():
    with pytest.raises(ValueError):
        partition([1.0], 0)


def test_gather_on_one_rank_is_the_local_records():
    assert gather_results({3: "c", 1: "a"}, 1, 0) == {1: "a", 3: "c"}


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, costs, out) -> None:
    import datetime

    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        mine = partition(costs, world)[rank]
        local = {r: {"peak_q": float(r) * 1.5, "rank": rank} for r in mine}
        merged = gather_results(local, world, rank)
        if rank == 0:
            out.put(merged)
        else:
            assert merged is None
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_gather_every_run_in_order():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    costs = list(np.random.default_rng(5).lognormal(0.0, 1.0, 21))
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, costs, q)) for r in range(2)]
    for p in procs:
        p.start()
    merged = q.get(timeout=120)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert list(merged) == list(range(21))
    parts = partition(costs, 2)
    for r, rec in merged.items():
        assert rec["peak_q"] == r * 1.5
        assert r in parts[rec["rank"]]
