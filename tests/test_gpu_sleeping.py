"""Sleeping tiles on the B200 (the reference's W90, tests/solver/test_sleeping.py:111-117): a tile that neither holds
water nor can be reached by any before the next check is not stepped, and the run is the run that steps every tile
to the last bit: every state array, the step count and the time step. A valley of 64 x 256 cells, a source at its head
and a free outfall at its foot; the flood wakes the valley as it goes. Through the host-driven loop and the device
loop."""

from __future__ import annotations

import numpy as np
import pytest

from wadi2d_b200.backend import BoundaryCells
from wadi2d_b200.config import Numerics, Tables
from wadi2d_b200.grid import TileGrid
from wadi2d_b200.model import Model
from wadi2d_b200.state import state_index
from wadi2d_b200.tables import ArrayBed, build_tables

pytestmark = pytest.mark.gpu

DX = 10.0
FIELDS = ("h", "d", "u", "v", "mx", "my", "qx", "qy", "res", "om")


def _valley(adaptive: bool):
    """A valley falling 0.2 % along x with 5 % side slopes, 64 x 256 cells of 10 m, Manning 0.035; a 6 m3/s source on
    a 3 x 3 block at the head of its axis and a free outfall across its foot."""
    ny, nx = 64, 256
    tg = TileGrid.from_mask(np.ones((ny, nx), bool), 0.0, 0.0, DX)
    pny, pnx = tg.shape
    j, i = np.mgrid[0:pny, 0:pnx]
    axis = 1 + ny // 2
    z = 0.002 * DX * (pnx - i) + 0.05 * DX * np.abs(j - axis)
    tables = build_tables(tg, ArrayBed(z.astype(np.float64), DX), Tables(), 0.035)
    m = Model(tables, Numerics())
    m.stepper.adaptive_active = adaptive
    rows = np.arange(1, 1 + ny)
    cols = np.full(ny, nx)
    cells = state_index(tg, rows, cols).astype(np.int32)
    k = cells.size
    m.set_boundary(BoundaryCells(cells, cells.copy(), np.ones(k, np.int32), np.zeros(k, np.float32),
                                 np.zeros(k, np.float32)))  # fmt: skip
    m.set_depth(np.zeros(tg.shape))
    rate = np.zeros(tg.shape)
    rate[axis - 1 : axis + 2, 2:5] = 6.0 / (9.0 * DX * DX)
    m.set_source(rate)
    return m


@pytest.mark.parametrize("loop", ["host", "device"])
def test_sleeping_tiles_give_the_all_tiles_run(loop):
    a, b = _valley(True), _valley(False)
    awake = []
    for t in (60.0, 600.0, 1800.0, 3600.0):
        for m in (a, b):
            if loop == "host":
                m.advance(t)
            else:
                m.run(t)
        awake.append(int(a.backend.nact))
        assert a.stepper.nsteps == b.stepper.nsteps, t
        assert a.stepper.dt == b.stepper.dt, t
        for f in FIELDS:
            assert np.array_equal(a.backend.get_field(f), b.backend.get_field(f)), (t, f)
    every = a.grid.ntiles - 1  # the padded grid's allocated tiles
    assert int(b.backend.nact) == every  # the reference steps every tile
    assert awake[0] < every // 2  # at first most of the valley sleeps
    assert awake[-1] > awake[0]  # the flood wakes it as it goes
