"""Still water on the B200. Two beds:

- terraces: every cell flat at its own level, levels on a 1/8 m grid 1,500 m above the datum, half of them above the
  water. Every level, depth and face invert is exactly representable, so a face between two wet cells sees the same
  level on both sides to the bit; the water must stay exactly still: u, v, mx, my, qx, qy exactly 0 and h, d unchanged
  bit for bit over 1,000 steps, in both builds.
- the reference's rough lake (wadi2d/validation/cases/lake_at_rest.py:142-151: a seeded Gaussian random bed of 0.5 m
  amplitude and a correlation length of 5 cells, water at the mean bed, here lifted 1,500 m), its depths set from the
  level through the tables (``hbar_at_level``, FP64, as the reference does). The levels above each cell's lowest pixel
  and the face inverts are rounded separately to float32, so the reference's own step moves this water at the
  round-off level: on the oracle, after 1,000 steps, face velocities reach 6.3e-5 m/s, unit discharges 8.5e-5 m2/s
  and depths change by 1.8e-6 m. The exact build must give the oracle's state bit for bit after 1,000 steps; both
  builds must keep the depth change within 1e-5 m, velocities and unit discharges within 1e-3 (the reference's own
  test of this case allows 1e-2 m/s, tests/solver/test_analytic.py:52-66) and the volume to 1e-6."""

from __future__ import annotations

import math

import numpy as np
import pytest

from oracle import oracle as O
from wadi2d_b200 import tables as T
from wadi2d_b200.config import Numerics
from wadi2d_b200.grid import TileGrid
from wadi2d_b200.model import Model

pytestmark = pytest.mark.gpu

STEPS = 1000
FIELDS = ("h", "d", "u", "v", "mx", "my", "qx", "qy", "res", "om")


class _Stop(Exception):
    pass


def _steps(model, n):
    def cb(st):
        if st.nsteps >= n:
            raise _Stop

    try:
        model.advance(1e12, cb)
    except _Stop:
        pass


def _rough(amplitude, corr, seed, n_modes=256):
    rng = np.random.default_rng(seed)
    kx, ky = rng.normal(0.0, 1.0 / corr, size=(2, n_modes))
    phase = rng.uniform(0.0, 2.0 * math.pi, size=n_modes)

    def bed(x, y):
        total = np.zeros_like(x, dtype=np.float64)
        for a, b, c in zip(kx, ky, phase, strict=True):
            total += np.cos(a * x + b * y + c)
        return amplitude * math.sqrt(2.0 / n_modes) * total

    return bed


def _lake(bed_pixels, n, dx, k, level, arith):
    """The oracle's tables of the bed (n x n cells, padded), a product model on them (``arith`` build) and an oracle
    model, both at the level through the tables."""
    og = O.Grid.from_mask(np.ones((n, n), bool), 0.0, 0.0, dx)
    tab = O.build_tables(og, bed_pixels, dx / k, 0.03, local_radius=True)
    grid = TileGrid(og.x0, og.y0, og.dx, og.mask)
    tables = T.GridTables.from_dict(grid, tab)
    h = T.hbar_at_level(level, tables.zmin, grid.from_tiles(tables.hc), grid.from_tiles(tables.dtab))
    assert np.array_equal(h, O.hbar_at_level(level, tab["zmin"], og.from_tiles(tab["hc"]), og.from_tiles(tab["dtab"])))
    h = np.where(grid.mask, h, 0.0)
    m = Model(tables, Numerics(dt_every=1, arithmetic=arith))
    m.set_depth(h)
    ref = O.Model(og, tab, O.Numerics(dt_every=1))
    ref.set_depth(h)
    return m, ref


@pytest.mark.parametrize("arith", ["exact", "fast"])
@pytest.mark.parametrize("loop", ["host", "device"])
def test_water_on_terraces_stays_exactly_still(arith, loop):
    n, dx, k = 64, 1.0, 4
    pad = 32 * int(np.ceil((n + 2) / 32))
    rng = np.random.default_rng(1)
    cellz = 1500.0 + 0.125 * rng.integers(0, 9, size=(pad, pad))
    z = np.repeat(np.repeat(cellz, k, 0), k, 1)
    m, _ = _lake(z, n, dx, k, 1500.5, arith)
    h0, d0 = m.field("h").copy(), m.field("d").copy()
    wet = int((h0 > 0).sum())
    assert 0.3 * n * n < wet < 0.8 * n * n
    if loop == "host":
        _steps(m, STEPS)
    else:
        m.run(1e12, max_steps=STEPS)
    assert m.stepper.nsteps == STEPS
    for name in ("u", "v", "mx", "my", "qx", "qy"):
        assert not np.any(m.field(name)), name
    assert np.array_equal(m.field("h"), h0)
    assert np.array_equal(m.field("d"), d0)


@pytest.mark.parametrize("arith", ["exact", "fast"])
def test_rough_lake_at_rest_keeps_the_reference_round_off(arith):
    n, dx, k, lift = 64, 0.1, 4, 1500.0
    pad = 32 * int(np.ceil((n + 2) / 32))
    p = dx / k
    xs, ys = np.meshgrid((np.arange(pad * k) - k + 0.5) * p, (np.arange(pad * k) - k + 0.5) * p)
    z = _rough(0.5, 5.0 * dx, 0)(xs, ys) + lift
    m, ref = _lake(z, n, dx, k, lift, arith)
    h0 = m.field("h").astype(np.float64)
    v0 = m.volume()
    _steps(m, STEPS)
    assert m.stepper.nsteps == STEPS
    if arith == "exact":
        _steps(ref, STEPS)
        for name in FIELDS:
            assert np.array_equal(m.field(name), ref.field(name)), name
    h = m.field("h").astype(np.float64)
    assert np.abs(h - h0).max() <= 1e-5
    for name in ("u", "v"):
        assert np.abs(m.field(name)).max() <= 1e-3, name
    for name in ("qx", "qy"):
        assert np.abs(m.field(name) / dx).max() <= 1e-3, name
    assert abs(m.volume() / v0 - 1.0) <= 1e-6
