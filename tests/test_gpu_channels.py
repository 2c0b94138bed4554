"""Steady uniform flow in straight channels on the B200, with the reference's setups and limits.

- A channel three cells wide laid at 45 degrees across the grid, with vertical walls
  (tests/solver/test_dry_faces.py:17-58). With dry and closed neighbour faces mirrored (the default), the mean level
  along its middle stays within 3 % of Manning's normal depth. Advected as real zero velocities they deepen it by
  5 to 12 %.
- A 60 m channel at a 1 % slope carrying 300 m3/s, with 2 m banks, on 20 m cells (tests/solver/test_face_level.py:
  34-97, the tile kernel). The level a cell holds over the bed at its own centre stays within 1.5 % of the normal
  depth.

Each channel starts at its normal level. A source block feeds the discharge at the upstream end, and a block of
fixed-level cells holds the normal level at the downstream end. The model is run through the reference's host loop
(``Model.advance``)."""

from __future__ import annotations

import numpy as np
import pytest
from scipy.optimize import brentq

from wadi2d_b200.backend import BoundaryCells
from wadi2d_b200.config import Numerics, Tables
from wadi2d_b200.grid import TileGrid
from wadi2d_b200.model import Model
from wadi2d_b200.state import level_of
from wadi2d_b200.tables import ArrayBed, build_tables, hbar_at_level

pytestmark = pytest.mark.gpu


def _hold_level(model: Model, tg: TileGrid, where: np.ndarray, depth: np.ndarray, hbar: np.ndarray) -> None:
    """Fixed-level boundary cells (kind 0) at ``where``: level ``depth`` over the cell's lowest bed, mean depth
    ``hbar``."""
    jj, ii = np.nonzero(where)
    cells = np.array([model.cell_state_index(int(j), int(i)) for j, i in zip(jj, ii, strict=True)], np.int32)
    zero = np.zeros(cells.size, np.int32)
    model.set_boundary(BoundaryCells(cells, zero, zero.copy(), depth.astype(np.float32), hbar.astype(np.float32)))


def _diagonal_channel_error(mirror: bool) -> float:
    """Per cent by which the mean level along the middle of the 45-degree channel exceeds Manning's normal depth."""
    dx, k, slope, n, width, q, side, offset = 20.0, 20, 0.002, 0.03, 60.0, 60.0, 128, 5.0
    tg = TileGrid.from_mask(np.ones((side, side), bool), 0.0, 0.0, dx)
    ny, nx = tg.shape
    p = dx / k
    half = 0.5 * np.sqrt(2.0)  # cos and sin of 45 degrees

    def along_across(x, y):
        return x * half + y * half, -x * half + y * half - offset

    # pixels: one-pixel rim (bed offset 1, 1), coordinates from the padded grid's centre
    px = (np.arange(nx * k + 2) - 0.5) * p - 0.5 * nx * dx
    py = (np.arange(ny * k + 2) - 0.5) * p - 0.5 * ny * dx
    s_p, t_p = along_across(*np.meshgrid(px, py))
    bed = -slope * s_p + np.where(np.abs(t_p) >= width / 2, 5.0, 0.0)
    yn = brentq(lambda y: width * y * (width * y / (width + 2 * y)) ** (2 / 3) * slope**0.5 / n - q, 0.01, 20.0)
    tables = build_tables(tg, ArrayBed(bed, p, 1, 1), Tables(), n)
    model = Model(tables, Numerics(mirror_dry_faces=mirror))

    cx = (np.arange(nx) + 0.5) * dx - 0.5 * nx * dx
    cy = (np.arange(ny) + 0.5) * dx - 0.5 * ny * dx
    s_c, t_c = along_across(*np.meshgrid(cx, cy))
    level = -slope * s_c + yn
    zmin = np.asarray(tables.zmin)
    h0 = hbar_at_level(level, zmin, tg.from_tiles(tables.hc), tg.from_tiles(tables.dtab))
    h0 = np.where(np.abs(t_c) < width / 2 + 2 * dx, h0, 0.0)
    model.set_depth(h0)
    reach = 0.45 * side * dx
    feed = (s_c > -reach) & (s_c < -reach + 120.0) & (np.abs(t_c) < width / 2 + dx)
    model.set_source(np.where(feed, q / (feed.sum() * dx * dx), 0.0))
    out = (s_c > reach - 120.0) & (s_c < reach) & (np.abs(t_c) < width + 3 * dx)
    _hold_level(model, tg, out, np.maximum(level - zmin, 0.0)[out], h0[out])
    model.advance(4000.0)
    middle = (np.abs(s_c) < 0.15 * side * dx) & (np.abs(t_c) < 0.71 * dx)
    return float(np.mean((zmin + model.field("d") + slope * s_c)[middle]) / yn - 1.0) * 100.0


@pytest.mark.parametrize(("mirror", "low", "high"), [(False, 5.0, 12.0), (True, -3.0, 3.0)])
def test_the_45_degree_channel(mirror: bool, low: float, high: float) -> None:
    err = _diagonal_channel_error(mirror)
    assert low < err < high, f"mirror={mirror}: {err:.2f} % over the normal depth"


def test_steady_uniform_flow_holds_the_normal_depth_at_20_m() -> None:
    side, dx, k = 96, 20.0, 10
    slope, n, wall, width, bank, q = 0.01, 0.03, 5.0, 60.0, 2.0, 300.0
    # the Lotter sum across the section, as the sub-grid conveyance holds it (no wall friction)
    yn = brentq(lambda y: (width * y ** (5 / 3) + 2 * bank * (3 / 8) * y ** (8 / 3)) * slope**0.5 / n - q, 0.01, 20)
    tg = TileGrid.from_mask(np.ones((side, side), bool), 0.0, 0.0, dx)
    ny, nx = tg.shape
    p = dx / k
    xm, ym = 0.5 * side * dx, -0.5 * side * dx
    X, Y = np.meshgrid(tg.x0 + (np.arange(nx * k) + 0.5) * p, tg.y0 - (np.arange(ny * k) + 0.5) * p)
    s_p, t_p = X - xm, Y - ym
    bed = (100.0 - slope * s_p + np.clip((np.abs(t_p) - width / 2) / bank, 0.0, wall)).astype(np.float32)
    tables = build_tables(tg, ArrayBed(bed.astype(np.float64), p), Tables(), n)
    model = Model(tables, Numerics())

    jj, ii = np.mgrid[0:ny, 0:nx]
    cx, cy = tg.xy_of(jj, ii)
    s_c, t_c = cx - xm, cy - ym
    zmin = np.asarray(tables.zmin)
    hc, dtab = tg.from_tiles(tables.hc), tg.from_tiles(tables.dtab)
    level = 100.0 - slope * s_c + yn
    hb = hbar_at_level(level, zmin, hc, dtab)
    hb = np.where((np.abs(t_c) < width / 2 + bank * yn + 2 * dx) & tg.mask, hb, 0.0)
    model.set_depth(hb)
    reach = 0.45 * side * dx
    feed = (s_c > -reach) & (s_c < -reach + 6 * dx) & (np.abs(t_c) < width / 2 + dx) & tg.mask
    model.set_source(np.where(feed, q / (feed.sum() * dx * dx), 0.0))
    out = (s_c > reach - 6 * dx) & (s_c < reach) & (np.abs(t_c) < width + 3 * dx) & tg.mask
    _hold_level(model, tg, out, level_of(hb[out], hc[out], dtab[out]), hb[out])
    model.advance(3000.0)
    middle = (np.abs(s_c) < 0.15 * side * dx) & (np.abs(t_c) < 0.71 * dx) & tg.mask
    ratio = float(np.mean((zmin + model.field("d").astype(np.float64) + slope * s_c - 100.0)[middle])) / yn
    assert abs(ratio - 1.0) < 0.015, f"depth {ratio:.4f} of the normal depth"
