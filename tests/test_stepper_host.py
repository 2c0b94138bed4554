"""The host loop's control (``stepper.Stepper``: the step rule, the refresh and activity schedule, sleeping tiles,
the failures) on the CPU, driven through a stand-in backend that scripts the wave speed and the wet tiles and logs
every call. With WADI2D_REFERENCE naming the reference's source tree, the reference's own Stepper
(wadi2d/solver/stepper.py:24-133) is driven through the same script and must make the same calls."""

from __future__ import annotations

import importlib
import math
import os
import sys

import numpy as np
import pytest

from wadi2d_b200.config import Numerics
from wadi2d_b200.grid import TileGrid
from wadi2d_b200.stepper import NumericalFailure, Stepper

REF = os.environ.get("WADI2D_REFERENCE")
NUM = dict(cfl=0.45, dt_max=5.0, dt_min=1e-3, dt_every=4, wave_floor=3.0, active_every=3)


class ScriptedBackend:
    """The members the stepper uses. ``waves``: the wave maximum each refresh reads, in order; ``wet(n)``: the wet
    tiles after n steps."""

    def __init__(self, ntiles: int, waves, wet):
        self.ntiles, self.waves, self.wet = ntiles, list(waves), wet
        self.nsteps = 0
        self.active_tiles = np.zeros(0, np.int32)
        self.nact = 0
        self.log: list[tuple] = []

    def step(self, dt, refresh, activate):
        self.log.append(("step", dt, bool(refresh), bool(activate)))
        self.nsteps += 1

    def max_wave(self):
        return self.waves.pop(0)

    def wet_flags(self):
        return self.wet(self.nsteps).astype(np.int32)

    def set_active(self, tiles):
        self.active_tiles = np.asarray(tiles, np.int32)
        self.nact = int(self.active_tiles.size)
        self.log.append(("active", tuple(int(t) for t in self.active_tiles)))

    def refresh_plan(self, tiles):
        self.log.append(("plan", tuple(int(t) for t in tiles)))

    def refresh_halos(self):
        self.log.append(("halos",))


def _grid():
    return TileGrid.from_mask(np.ones((94, 126), bool), 0.0, 0.0, 30.0)  # 3 x 4 tiles of 32 cells


def _wet_script(ntiles):
    """Water in tile 1 to start; tile 6 wets from step 4 to step 9; everything dries after step 14."""

    def wet(n):
        w = np.zeros(ntiles, bool)
        if n < 14:
            w[1] = True
        if 4 <= n < 9:
            w[6] = True
        return w

    return wet


def _drive(stepper_cls, num, t_end=60.0, waves=None):
    grid = _grid()
    waves = [2.0, 6.0, 12.0, 4.0, 1.0, 2.5, 8.0, 3.5, 9.0, 5.0, 7.0] * 4 if waves is None else waves
    b = ScriptedBackend(grid.ntiles, waves, _wet_script(grid.ntiles))
    s = stepper_cls(b, grid, num)
    s.rebuild_active()
    t = s.advance(t_end)
    return s, b, t


def test_step_rule_schedule_and_exact_end():
    num = Numerics(**NUM)
    s, b, t = _drive(Stepper, num)
    steps = [e for e in b.log if e[0] == "step"]
    assert t == s.t and abs(t - 60.0) < 1e-9
    assert sum(e[1] for e in steps) == pytest.approx(60.0, abs=1e-9)
    # the first step is refreshed and uses cfl dx / wave_floor; refresh every dt_every steps; a check every
    # active_every steps
    assert steps[0][1] == pytest.approx(min(0.45 * 30.0 / 3.0, 5.0))
    for n, (_, _, refresh, activate) in enumerate(steps):
        assert refresh == (n % 4 == 0)
        assert activate == (n % 3 == 0)
    # between refreshes dt holds; after one it is cfl dx / max(w, floor), capped at dt_max, and the last step ends
    # on t_end
    waves = [2.0, 6.0, 12.0, 4.0, 1.0, 2.5, 8.0, 3.5, 9.0, 5.0, 7.0]
    dt, k = min(0.45 * 30.0 / 3.0, 5.0), 0
    for n, e in enumerate(steps[:-1]):
        assert e[1] == pytest.approx(dt)
        if n % 4 == 0:
            dt = min(0.45 * 30.0 / max(waves[k % len(waves)], 3.0), 5.0)
            k += 1


def test_a_dry_tile_sleeps_after_two_checks_and_a_woken_tile_is_refreshed():
    num = Numerics(**NUM)
    grid = _grid()
    s, b, _ = _drive(Stepper, num)
    actives = [set(e[1]) for e in b.log if e[0] == "active"]
    nb1 = {int(t) for t in grid.nbr[1] if t} | {1}
    nb6 = {int(t) for t in grid.nbr[6] if t} | {6}
    assert actives[0] == nb1  # the fresh list: tile 1 and its neighbours
    assert any(nb6 <= a for a in actives)  # tile 6 and its neighbours joined while it was wet
    woken = [e for e in b.log if e[0] == "plan"]
    assert woken and all(set(e[1]) <= nb6 - nb1 for e in woken)
    assert all(b.log[b.log.index(e) + 1] == ("halos",) for e in woken)
    assert actives[-1] == set()  # all dry: every tile has left, two checks after it was last wanted


@pytest.mark.parametrize("wave,message", [(math.nan, "non-finite wave speed"), (1e9, "below the minimum")])
def test_a_non_finite_wave_or_a_collapsed_step_stops_the_run(wave, message):
    with pytest.raises(NumericalFailure, match=message):
        _drive(Stepper, Numerics(**NUM), waves=[2.0, wave, 2.0, 2.0])


@pytest.mark.skipif(not REF, reason="WADI2D_REFERENCE (the reference source tree) is not set")
def test_the_references_stepper_makes_the_same_calls(monkeypatch):
    monkeypatch.syspath_prepend(REF)
    for name in [n for n in sys.modules if n == "wadi2d" or n.startswith("wadi2d.")]:
        monkeypatch.delitem(sys.modules, name)
    try:
        theirs = importlib.import_module("wadi2d.solver.stepper")
        RefNumerics = importlib.import_module("wadi2d.config.schema").Numerics
        for waves in (None, [2.0, 40.0, 0.5, 25.0] * 20):
            mine, b1, t1 = _drive(Stepper, Numerics(**NUM), waves=waves)
            ref, b2, t2 = _drive(theirs.Stepper, RefNumerics(**NUM), waves=waves)
            assert b1.log == b2.log
            assert (t1, mine.nsteps, mine.dt) == (t2, ref.nsteps, ref.dt)
            np.testing.assert_array_equal(mine.idle, ref.idle)
        with pytest.raises(theirs.NumericalFailure, match="non-finite"):
            _drive(theirs.Stepper, RefNumerics(**NUM), waves=[2.0, math.nan])
    finally:
        for name in [n for n in sys.modules if n == "wadi2d" or n.startswith("wadi2d.")]:
            del sys.modules[name]
