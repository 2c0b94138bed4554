"""The step limiter on the B200 (wadi2d/solver/limiter.py:113-191; the reference's own tests are
tests/solver/test_limiter.py:39-115): the device probe gives every face of a tile the wave speed and new velocity
that a real step computes, bit for bit; the report names the face whose wave the step rule read; and reading it
leaves the water bit-identical."""

from __future__ import annotations

import numpy as np
import pytest

from oracle import oracle as O
from wadi2d_b200 import workloads
from wadi2d_b200.backend import BoundaryCells
from wadi2d_b200.config import Numerics
from wadi2d_b200.grid import TileGrid
from wadi2d_b200.layout import HALO, TILE, local_index
from wadi2d_b200.limiter import step_limiter, tile_waves
from wadi2d_b200.model import Model
from wadi2d_b200.state import state_index
from wadi2d_b200.tables import GridTables

pytestmark = pytest.mark.gpu


def _model(n=64, t_end=900.0):
    w = workloads.v_channel_plane(n=n, dx=10.0, k=5, seed=0)
    og = O.Grid.from_mask(np.ones((n, n), bool), 0.0, 0.0, w.dx)
    tab = O.build_tables(og, w.z, w.dx / w.k, w.manning)
    g = TileGrid.from_mask(np.ones((n, n), bool), 0.0, 0.0, w.dx)
    m = Model(GridTables.from_dict(g, tab), Numerics(cfl=w.cfl))
    rows, cols = w.outfall
    cells = np.array([state_index(g, int(j), int(i)) for j, i in zip(rows, cols, strict=True)], np.int32)
    nb = cells.size
    m.set_boundary(BoundaryCells(cells, np.zeros(nb, np.int32), np.ones(nb, np.int32), np.zeros(nb, np.float32),
                                 np.zeros(nb, np.float32)))  # fmt: skip
    rate = np.zeros(g.shape)
    rate[1 : 1 + w.ny, 1 : w.nx] = 4.0 * w.rain_mm_h / 3.6e6
    m.set_source(rate)
    m.run(t_end)
    return m, g


def _own(t: int) -> np.ndarray:
    jj, ii = np.divmod(np.arange(TILE * TILE), TILE)
    return local_index(t, jj + HALO, ii + HALO).astype(np.int64)


def test_probe_gives_the_waves_and_velocities_of_a_real_step():
    m, g = _model()
    b = m.backend
    dt = float(np.float32(m.stepper.dt))
    for t in range(1, g.ntiles):
        wx, wy, ux, vy = tile_waves(b, t, dt)
        if t == 1:
            probes = {}
        probes[t] = (max(float(wx.max()), float(wy.max())), ux.reshape(-1).copy(), vy.reshape(-1).copy())
    before = {f: m.field(f) for f in ("h", "d", "u", "v", "qx", "qy")}
    b.step(dt, True, False)  # one refresh step of the face pass from the probed state
    wave = b.wave
    assert max(p[0] for p in probes.values()) > 0.0
    for t, (wmax, ux, vy) in probes.items():
        assert np.float32(wave[t]) == np.float32(wmax), t
        assert np.array_equal(b.u[_own(t)], ux), t
        assert np.array_equal(b.v[_own(t)], vy), t
    # the probes wrote nothing: a second model stepped without them agrees bit for bit
    m2, _ = _model()
    for f, a in before.items():
        assert np.array_equal(m2.field(f), a), f


def test_limiter_names_the_leading_face_and_leaves_the_water_as_it_is():
    m, g = _model()
    m2, _ = _model()
    for _ in range(4):
        rep = step_limiter(m)
        assert rep is not None and rep["source"] == "tiles"
        t = rep["tile"]
        wave = np.asarray(m.backend.wave, np.float64)
        assert t == int(np.argmax(wave[1:])) + 1
        wx, wy, _, _ = tile_waves(m.backend, t, m.stepper.dt)
        assert rep["wave"] == round(float(max(wx.max(), wy.max())), 3)
        assert rep["axis"] in ("x", "y")
        assert 0 <= rep["j"] < g.shape[0] and 0 <= rep["i"] < g.shape[1]
        assert rep["speed"] <= rep["wave"] + 1e-6
        assert rep["dt_without_tile"] >= rep["dt_tile"] - 1e-9
        m.run(m.stepper.t + 120.0)
        m2.run(m2.stepper.t + 120.0)
    assert m.stepper.nsteps == m2.stepper.nsteps
    for f in ("h", "d", "u", "v", "qx", "qy", "res"):
        assert np.array_equal(m.field(f), m2.field(f)), f


def test_limiter_on_a_dry_grid_is_none():
    w = workloads.v_channel_plane(n=40, dx=10.0, k=5, seed=0)
    og = O.Grid.from_mask(np.ones((40, 40), bool), 0.0, 0.0, w.dx)
    tab = O.build_tables(og, w.z, w.dx / w.k, w.manning)
    g = TileGrid.from_mask(np.ones((40, 40), bool), 0.0, 0.0, w.dx)
    m = Model(GridTables.from_dict(g, tab), Numerics())
    m.run(30.0)
    assert step_limiter(m) is None
