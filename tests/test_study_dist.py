"""The depth-area study split over two gloo ranks on CPU (the collective a GPU study takes over NCCL): each rank
solves its share of the storm areas, rank 0 gathers every run and reads the same design table and composites as one
process solving them all. The solver is a stand-in with the real one's arguments and results."""

from __future__ import annotations

import os
import socket
from types import SimpleNamespace

import numpy as np
import torch.multiprocessing as mp

from wadi2d_b200 import study as S
from wadi2d_b200.forcing import ArfTable, UniformStorm

NL, SHAPE = 3, (6, 7)
STORM = UniformStorm(60.0, 90.0, arf=ArfTable(np.array([0.1, 1.0, 10.0, 100.0]), np.array([1.0, 0.9, 0.8, 0.6])))
AREAS = [0.2, 0.7, 2.5, 9.0, 30.0]
LINE_AREAS = [0.3, None, 12.0]
CELL_AREA = np.exp(np.linspace(np.log(0.05), np.log(80.0), SHAPE[0] * SHAPE[1])).reshape(SHAPE)
CAT = SimpleNamespace(lines=[None] * NL)


def fake_solve(cat, storms, t_end, window, every, num, batched):
    """Deterministic per storm: peaks and envelopes from the storm's depth, so a run gives the same record wherever
    it is solved."""
    n = len(storms)
    peaks = np.array([[s.total_depth * (k + 1) for k in range(NL)] for s in storms])
    times = np.array([[1000.0 + s.total_depth + k for k in range(NL)] for s in storms])
    steps = np.array([int(100 * s.total_depth) for s in storms])
    envs = [{f: np.full(SHAPE, s.total_depth * (1 + j)) for j, f in enumerate(("depth", "speed", "hazard"))}
            for s in storms]  # fmt: skip
    return peaks, times, steps, envs, 0.5 + 0.1 * n


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out) -> None:
    import datetime

    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        res = S.run_study_sharded(CAT, STORM, AREAS, ["a", "b", "c"], LINE_AREAS, CELL_AREA, 3600.0,
                                  solve=fake_solve)  # fmt: skip
        if rank == 0:
            out.put((res.table, {k: v for k, v in res.composite.items()}, res.steps.tolist(), res.seconds))
        else:
            assert res is None
    finally:
        dist.destroy_process_group()


def test_one_process_reads_what_the_ranks_solved():
    res = S.run_study_sharded(CAT, STORM, AREAS, ["a", "b", "c"], LINE_AREAS, CELL_AREA, 3600.0, world=1, rank=0,
                              solve=fake_solve)  # fmt: skip
    peaks, times, steps, envs, _ = fake_solve(CAT, S.storms_at(STORM, AREAS), 0, 0, 0, None, True)
    assert res.table == S.design_table(["a", "b", "c"], LINE_AREAS, AREAS, peaks, times)
    assert np.array_equal(res.composite["hazard"], S.composite_map([e["hazard"] for e in envs], AREAS, CELL_AREA))
    assert res.steps.tolist() == steps.tolist()


def test_two_gloo_ranks_give_the_one_process_study():
    one = S.run_study_sharded(CAT, STORM, AREAS, ["a", "b", "c"], LINE_AREAS, CELL_AREA, 3600.0, world=1, rank=0,
                              solve=fake_solve)  # fmt: skip
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    table, composite, steps, seconds = q.get(timeout=120)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert table == one.table
    for name in S.COMPOSITE_MAPS:
        assert np.array_equal(composite[name], one.composite[name]), name
    assert steps == one.steps.tolist()
    assert seconds == max(0.5 + 0.1 * 3, 0.5 + 0.1 * 2)  # the slowest rank's: three runs on rank 0, two on rank 1
