"""Analytic cases of the reference's own suite (tests/solver/test_subgrid.py:49-92), run on the B200 through this
package (GPU-built tables, the device-resident loop): rain on a plane reaches the kinematic-wave equilibrium within
3 %, and a thin crest passes critical flow within 1 %."""

from __future__ import annotations

import numpy as np
import pytest

from wadi2d_b200.backend import BoundaryCells
from wadi2d_b200.config import CRITICAL_WEIR_COEFF, Numerics, Tables
from wadi2d_b200.grid import TileGrid
from wadi2d_b200.model import Model
from wadi2d_b200.tables import ArrayBed, build_tables

pytestmark = pytest.mark.gpu
RAIN_MM_H = 50.0


def _pixels(tg: TileGrid, k: int):
    ny, nx = tg.shape
    p = tg.dx / k
    return np.meshgrid(tg.x0 + (np.arange(nx * k) + 0.5) * p, tg.y0 - (np.arange(ny * k) + 0.5) * p)


@pytest.mark.parametrize("slope", [0.01, 0.05, 0.2])
def test_sheet_flow_on_a_plane_matches_the_kinematic_wave(slope):
    n, length, dx, k = 0.05, 2000.0, 20.0, 20
    nx, ny = int(length / dx), 3
    tg = TileGrid.from_mask(np.ones((ny, nx), bool), 0.0, 0.0, dx)
    xs, _ = _pixels(tg, k)
    tables = build_tables(tg, ArrayBed((length - xs) * slope, dx / k), Tables(), n)
    m = Model(tables, Numerics(dt_max=2.0))
    rain = np.zeros(tg.shape)
    i = RAIN_MM_H / 3.6e6
    rain[1 : 1 + ny, 1:nx] = i
    m.set_source(rain)
    cells = [m.cell_state_index(j + 1, nx) for j in range(ny)]
    m.set_boundary(BoundaryCells(np.array(cells, np.int32), np.zeros(ny, np.int32), np.ones(ny, np.int32),
                                 np.zeros(ny, np.float32), np.zeros(ny, np.float32)))  # fmt: skip
    tc = (n * length / (slope**0.5 * i ** (2.0 / 3.0))) ** 0.6
    m.run(2.5 * tc)
    q_end = i * length
    h_end = (q_end * n / slope**0.5) ** 0.6
    hmean = float(m.field("h")[1 + ny // 2, 1:nx].mean())
    assert hmean == pytest.approx(0.625 * h_end, rel=0.03)
    outflow = float(m.field("qx")[1 + ny // 2, nx]) / dx
    assert outflow == pytest.approx(q_end, rel=0.03)


def test_thin_crest_passes_critical_flow():
    nx, ny, k, dx, crest, head = 120, 4, 4, 5.0, 3.0, 1.0
    tg = TileGrid.from_mask(np.ones((ny, nx), bool), 0.0, 0.0, dx)
    xs, _ = _pixels(tg, k)
    i_crest = 61
    z = np.zeros(xs.shape)
    z[(xs >= i_crest * dx) & (xs < i_crest * dx + dx / k)] = crest
    tables = build_tables(tg, ArrayBed(z, dx / k), Tables(), 0.012)
    m = Model(tables, Numerics(cfl=0.4, dt_every=1))
    h0 = np.zeros(tg.shape)
    h0[:, :i_crest] = crest + head
    m.set_depth(h0)
    n_b = ny * 3
    cells = [m.cell_state_index(j + 1, c) for j in range(ny) for c in (1, 2, 3)]
    m.set_boundary(BoundaryCells(np.array(cells, np.int32), np.zeros(n_b, np.int32), np.zeros(n_b, np.int32),
                                 np.full(n_b, crest + head, np.float32), np.full(n_b, crest + head, np.float32)))  # fmt: skip
    m.run(300.0)
    q = float(m.field("qx")[2, i_crest]) / dx
    hup = float(m.field("h")[2, i_crest - 3]) - crest
    assert q == pytest.approx(CRITICAL_WEIR_COEFF * hup**1.5, rel=0.01)
