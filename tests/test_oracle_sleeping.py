"""Sleeping tiles on the oracle, with the reference's scenarios (tests/solver/test_sleeping.py:19-107, the squares-only
cases; the valley of tests/strips/valley.py without its strip). A tile that neither holds water nor can be reached
by any before the next check is not stepped. The run equals the one that steps every tile, to the last bit: every
state array, the step count, the time and the time step. No GPU needed.

The valley falls 1 % along x and rises 2 % either side of its axis. It has 20 m cells, 2 x 2 pixels a cell, and
Manning n = 0.035, so water put in at the head runs down a narrow course and the hills stay dry."""

from __future__ import annotations

import numpy as np
import pytest

from oracle import oracle as O

DX, K, SLOPE, SIDE, MANNING = 20.0, 2, 0.01, 0.02, 0.035
FIELDS = ("h", "d", "u", "v", "mx", "my", "qx", "qy", "res")


class Valley:
    """``tiles_y`` x ``tiles_x`` tiles of dry valley on the oracle; ``sleeping`` off steps every tile every step."""

    def __init__(self, tiles_y: int, tiles_x: int, sleeping: bool) -> None:
        mask = np.ones((tiles_y * 32 - 2, tiles_x * 32 - 2), bool)
        self.grid = O.Grid.from_mask(mask, 0.0, 0.0, DX)
        ny, nx = self.grid.shape
        self.axis = ny // 2
        p = DX / K
        xx, yy = np.meshgrid((np.arange(nx * K) + 0.5) * p, (np.arange(ny * K) + 0.5) * p)
        bed = 200.0 - SLOPE * xx + SIDE * np.abs(yy - (self.axis + 0.5) * DX)
        tables = O.build_tables(self.grid, bed.astype(np.float32).astype(np.float64), p, MANNING)
        self.model = O.Model(self.grid, tables)
        self.model.adaptive_active = sleeping
        self.model.set_depth(np.zeros(self.grid.shape))

    def head(self, discharge: float, column: int = 8) -> np.ndarray:
        """A source rate grid, m/s, putting ``discharge`` into the two squares beside the axis's band at
        ``column``."""
        rate = np.zeros(self.grid.shape)
        rate[[self.axis - 2, self.axis + 2], column] = discharge / (2 * DX * DX)
        return rate

    def open_end(self) -> None:
        """A free outflow on the last active column."""
        g = self.grid
        col = int(np.nonzero(g.mask.any(axis=0))[0][-1])
        cells = np.array([self.model.cell_state_index(int(j), col) for j in np.nonzero(g.mask[:, col])[0]], np.int32)
        zero, f = np.zeros(cells.size, np.int32), np.zeros(cells.size, np.float32)
        self.model.set_boundary(O.Boundary(cells, zero, np.ones(cells.size, np.int32), f, f.copy()))

    def awake(self) -> int:
        return int(self.model.backend.nact)

    def set_depth(self, h: np.ndarray) -> None:
        self.model.set_depth(h * self.grid.mask)

    def set_source(self, rate: np.ndarray) -> None:
        self.model.set_source(rate * self.grid.mask)


def pair(tiles_y: int, tiles_x: int) -> tuple[Valley, Valley]:
    return Valley(tiles_y, tiles_x, True), Valley(tiles_y, tiles_x, False)


def both(a: Valley, b: Valley, act) -> None:
    act(a)
    act(b)


def run_same(a: Valley, b: Valley, times, floor: int | None = None) -> list[int]:
    """Advance both through ``times``, equal to the bit at each; the sleeping run's awake tiles at each time."""
    awake = []
    for t in times:
        a.model.advance(t)
        b.model.advance(t)
        assert (a.model.nsteps, a.model.t, a.model.dt) == (b.model.nsteps, b.model.t, b.model.dt), t
        for name in FIELDS:
            fa, fb = a.model.field(name), b.model.field(name)
            assert np.array_equal(fa, fb), f"t = {t:g} s: {name} differs in {int(np.sum(fa != fb))} cells"
        awake.append(a.awake())
    assert b.awake() == b.grid.ntiles - 1  # stepping every tile never sleeps
    if floor is not None:
        assert min(awake) <= floor, awake
    return awake


def test_still_water_in_one_corner_leaves_the_rest_asleep():
    a, b = pair(3, 4)

    def lake(v: Valley) -> None:
        h = np.zeros(v.grid.shape)
        h[v.axis - 6 : v.axis + 7, 100:125] = 0.6  # a pond across the axis in the last tile column
        v.set_depth(h)

    both(a, b, lake)
    assert a.awake() < b.awake() == 12
    assert max(run_same(a, b, [30.0, 120.0, 400.0])) < 12
    assert a.model.volume() == pytest.approx(0.6 * 13 * 25 * DX * DX, rel=1e-6)


def test_a_front_that_crosses_tile_borders_in_every_direction():
    a, b = pair(5, 5)

    def columns(v: Valley) -> None:
        h = np.zeros(v.grid.shape)
        h[8:24, 70:90] = 2.0  # north hillside: runs south across two rows of tiles
        h[136:152, 70:90] = 2.0  # south hillside: north across two
        h[72:88, 70:90] = 3.0  # on the axis: backs up west and runs east
        v.set_depth(h)

    both(a, b, columns)
    first = a.awake()
    assert first == 15  # the three wet tiles and their neighbours, of 25
    awake = run_same(a, b, [20.0, 60.0, 150.0, 400.0, 900.0])
    wet = a.model.field("h") > 0.0
    assert wet[32:64, :].any() and wet[96:128, :].any() and wet[:, :64].any() and wet[:, 96:].any()
    assert awake[-1] > first


def test_rain_that_starts_later_on_a_sleeping_tile():
    a, b = pair(2, 8)
    both(a, b, lambda v: v.set_source(v.head(30.0)))
    run_same(a, b, [200.0])
    assert a.awake() < 16

    def rain(v: Valley) -> None:
        rate = v.head(30.0)
        rate[5:25, 200:230] = 60.0 / 3.6e6  # 60 mm/h on a dry hillside six tiles down the valley
        v.set_source(rate)

    far = a.model.cell_state_index(10, 210) // O.STRIDE2
    assert far not in set(a.model.backend.active_tiles.tolist())
    both(a, b, rain)
    assert far in set(a.model.backend.active_tiles.tolist())
    run_same(a, b, [260.0, 500.0, 900.0])
    assert a.model.field("h")[5:25, 200:230].min() > 0.0


def test_an_inflow_at_the_head_and_an_open_end():
    a, b = pair(2, 8)
    both(a, b, Valley.open_end)
    both(a, b, lambda v: v.set_source(v.head(40.0)))
    awake = run_same(a, b, [60.0, 300.0, 900.0, 1800.0, 3600.0], floor=8)
    assert awake[0] < awake[-1] == 16  # the flood reaches the end and wakes the valley as it goes
    assert a.model.field("h")[a.axis, -20:].max() > 0.0


def test_a_tile_that_dries_sleeps_again_and_wakes_again():
    a, b = pair(2, 8)

    def source(v: Valley, mm_h: float, everywhere: bool = False) -> None:
        rate = np.full(v.grid.shape, mm_h / 3.6e6) if everywhere else np.zeros(v.grid.shape)
        rate[8:20, 200:215] = mm_h / 3.6e6
        v.set_source(rate)

    both(a, b, lambda v: source(v, 40.0))
    assert a.awake() == 6  # the rained tile and its neighbours
    run_same(a, b, [120.0])
    assert a.model.volume() > 0.0
    both(a, b, lambda v: source(v, -4000.0, everywhere=True))  # a loss that takes every drop, wherever it ran
    run_same(a, b, [600.0])
    assert a.model.volume() == 0.0
    both(a, b, lambda v: source(v, 0.0))
    assert a.awake() == 16  # a change of source drops no tile: only a check does
    run_same(a, b, [700.0, 1200.0])
    assert a.awake() == 0  # dry at two checks in a row: every tile left the list
    both(a, b, lambda v: source(v, 40.0))
    assert a.awake() == 6  # and the rained tile and its neighbours wake at once
    run_same(a, b, [1300.0, 1800.0])
    assert a.model.volume() > 0.0
