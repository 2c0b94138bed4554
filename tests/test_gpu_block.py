"""Configuration 3 on the B200 against the oracle: the middle 32 x 32-tile block of the 4096 x 4096 seeded catchment
that bench.py times (padded as the reference pads a grid: 1,044,484 active cells inside an inactive outer ring), its
tables from the oracle's table builder on the block's own pixels, 0.05 m of water under the storm's peak rain, 200
steps of each's host-driven loop at the reference's dt rule (``bench.block_parity``, which the default bench line also
reports). The exact build must be the oracle bit for bit, the fast build within the step's accuracy bounds."""

from __future__ import annotations

import os

import numpy as np
import pytest

import bench

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def block():
    import torch

    from wadi2d_b200 import workloads
    from wadi2d_b200.grid import TileGrid

    c = workloads.catchment(n=4096, device=torch.device("cuda", 0))
    grid = TileGrid.from_mask(np.ones((4096, 4096), bool), 0.0, 0.0, c.dx)
    bench.cut_block(c, grid)
    del c.z
    torch.cuda.empty_cache()
    return bench.block_inputs(c, grid, bench.peak_rate(c))


def test_exact_build_is_the_oracle_bit_for_bit_on_configuration3(block):
    r = bench.block_parity(block, "exact", 200, os.cpu_count() or 1)
    assert r["steps"] == 200
    assert r["dt_identical"], r
    assert r["bit_identical"], r
    assert r["within_bounds"], r


def test_fast_build_within_the_bounds_on_configuration3(block):
    r = bench.block_parity(block, "fast", 200, os.cpu_count() or 1)
    assert r["steps"] == 200
    assert r["wet_set_identical"], r
    assert r["depth_within"], r
    assert r["discharge_within"], r
    assert r["dt_max_rel_diff"] < 1e-5, r
