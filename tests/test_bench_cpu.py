"""The CPU sample of bench.py, which is all the reference arm times and the GPU arm's ``cpu_baseline`` leg: the middle
32 x 32-tile block of the grid, its tables from the oracle's table builder on the block's own pixels, the oracle's
step on host threads. No GPU needed."""

from __future__ import annotations

import types

import numpy as np

import bench
from wadi2d_b200.grid import TileGrid


def test_the_block_is_the_middle_32_x_32_tiles():
    grid = TileGrid.from_mask(np.ones((4096, 4096), bool), 0.0, 0.0, 30.0)
    j0, i0, side = bench.cpu_block(grid)
    assert side == 32 * bench.CPU_BLOCK_TILES == 1024
    assert (j0, i0) == (48 * 32, 48 * 32)  # 129 tile rows: 48 before the block, 49 after
    assert j0 % 32 == 0 and j0 + side <= grid.shape[0]


def test_cpu_sample_steps_the_oracle_on_the_block():
    n, k = 1100, 4
    grid = TileGrid.from_mask(np.ones((n, n), bool), 0.0, 0.0, 30.0)
    j0, i0, side = bench.cpu_block(grid)
    rng = np.random.default_rng(5)
    bed = 100.0 + 0.02 * np.cumsum(rng.normal(0.0, 1.0, (grid.shape[0] * k + 2, grid.shape[1] * k + 2)), axis=1)
    c = types.SimpleNamespace(dx=30.0, k=k, manning=0.035)
    c.block_z = bed[j0 * k : (j0 + side) * k + 2, i0 * k : (i0 + side) * k + 2]
    rate = np.full(grid.shape, 40.0 / 3.6e6)
    value, done, seconds, cells = bench.cpu_sample(bench.block_inputs(c, grid, rate), 0.0, 2, steps=2, warmup=1)
    assert side == 1024 and cells == (side - 2) ** 2  # the padded grid's outer ring is inactive
    assert done == 2 and seconds > 0.0
    assert value == cells * done / seconds
