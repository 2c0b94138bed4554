"""Failures the reference's review found by running its code (tests/solver/test_review_regressions.py:26-140), run on
the B200 through this package's host-driven loop (``Model.advance``, the reference's loop) with the same cases and
limits: rain on deep water stored in full (float32 alone would round it away), the step following a sudden drop,
the first step on dry ground, water left to drain when a source stops, an empty grid, a NaN stopping the run, and a
narrow pond on a face line staying calm."""

from __future__ import annotations

import numpy as np
import pytest

from wadi2d_b200.config import Numerics, Tables
from wadi2d_b200.grid import TileGrid
from wadi2d_b200.model import Model
from wadi2d_b200.stepper import NumericalFailure
from wadi2d_b200.tables import ArrayBed, build_tables

pytestmark = pytest.mark.gpu


def _model(bed, dx: float, nside: int, num=None, k: int = 1, n: float = 0.03):
    tg = TileGrid.from_mask(np.ones((nside, nside), bool), 0.0, 0.0, dx)
    return Model(build_tables(tg, ArrayBed(bed(tg, k), dx / k), Tables(), n), num or Numerics()), tg


def _flat(tg, k):
    return np.zeros((tg.shape[0] * k + 2, tg.shape[1] * k + 2))


@pytest.mark.parametrize("depth, mm_h", [(20.0, 10.0), (20.0, 30.0), (2.0, 3.0)])
def test_rain_on_deep_water_is_stored_in_full(depth, mm_h):
    """The compensated float32 residual keeps rain that float32 alone would round away on deep water."""
    m, tg = _model(_flat, 10.0, 30)
    h0 = np.where(tg.mask, depth, 0.0)
    m.set_depth(h0)
    rate = np.where(tg.mask, mm_h / 3.6e6, 0.0)
    m.set_source(rate)
    m.advance(3600.0)
    stored = float((m.field("h").astype(np.float64) - h0).sum())
    assert stored == pytest.approx(float(rate.sum()) * 3600.0, rel=0.01)


def test_step_follows_a_sudden_drop():
    """A pool over a 30 m cliff: with the step refreshed every 8 steps the Courant number stays below 1."""

    def cliff(tg, k):
        z = np.zeros((tg.shape[0] * k + 2, tg.shape[1] * k + 2))
        z[:, tg.shape[1] // 2 :] = -30.0
        return z

    dx = 10.0
    m, tg = _model(cliff, dx, 62, Numerics(dt_every=8))
    h = np.zeros(tg.shape)
    h[:, : tg.shape[1] // 2] = 3.0
    m.set_depth(np.where(tg.mask, h, 0.0))
    worst = 0.0

    def watch(s):
        nonlocal worst
        if s.nsteps % 8 == 0:
            worst = max(worst, float(np.abs(s.backend.get_field("u")).max()) * s.dt / dx)

    m.advance(40.0, watch)
    assert worst < 1.0


def test_first_step_on_dry_ground_is_not_the_longest():
    m, _ = _model(_flat, 20.0, 30)
    assert m.stepper.dt <= m.num.cfl * 20.0 / m.num.wave_floor + 1e-9


def test_water_is_not_stranded_when_a_source_stops():
    """Rain starts and ends between two wet-flag checks on a dry slope; the water must still drain."""

    def slope(tg, k):
        return np.tile(0.01 * 20.0 * (tg.shape[1] - np.arange(tg.shape[1] + 2)), (tg.shape[0] + 2, 1))

    m, tg = _model(slope, 20.0, 120)
    m.set_source(np.where(tg.mask, 0.1, 0.0))  # 0.1 m in one second
    m.advance(1.0)
    m.set_source(np.zeros(tg.shape))
    before = m.field("h").copy()
    m.advance(600.0)
    assert np.abs(m.field("h") - before).max() > 0.0


def test_an_empty_grid_does_not_crash():
    m, _ = _model(_flat, 20.0, 30)
    m.advance(10.0)
    assert m.stepper.t == pytest.approx(10.0)


def test_nan_stops_the_run():
    m, tg = _model(_flat, 10.0, 30)
    m.set_depth(np.where(tg.mask, 1.0, 0.0))
    u = m.backend.get_field("u")
    u[m.cell_state_index(10, 10)] = float("nan")
    m.backend.set_field("u", u)
    m.stepper.refresh_due = True
    with pytest.raises(NumericalFailure):
        m.advance(5.0)


def test_narrow_pond_on_a_face_line_stays_calm():
    """A one-pixel trench along a face with a small level difference across it must not grow."""
    k, dx, nside = 10, 20.0, 30

    def trench(tg, kk):
        z = np.zeros((tg.shape[0] * kk + 2, tg.shape[1] * kk + 2))
        c = 15 * kk
        z[:, c - 1 : c + 1] = -2.0
        return z

    m, tg = _model(trench, dx, nside, Numerics(dt_every=1), k=k)
    h0 = np.zeros(tg.shape)
    h0[:, 14] = 0.05
    h0[:, 15] = 0.03
    m.set_depth(np.where(tg.mask, h0, 0.0))
    zmin = np.asarray(m.tables.zmin)
    peak = 0.0

    def watch(_):
        nonlocal peak
        d = m.field("d") + zmin
        peak = max(peak, float(np.abs(d[10, 14] - d[10, 15])))

    for t in range(1, 21):
        m.advance(float(t * 3), watch if t % 5 == 0 else None)
    assert peak < 0.5
