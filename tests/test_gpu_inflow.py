"""Lumped inflows on the device (``run.DeviceInflow``, w2b_inflow_window) against their host form
(``forcing.Forcing.rate`` with injections, the levels read back from the device as wadi2d/forcing.py:631-644 does):
the same float32 source rates bit for bit, the same window volumes, and configuration 2 stepped through either gives
the same run bit for bit."""

from __future__ import annotations

import numpy as np
import pytest

from oracle import oracle as O
from wadi2d_b200 import forcing as F
from wadi2d_b200 import workloads
from wadi2d_b200.backend import BoundaryCells
from wadi2d_b200.config import Numerics
from wadi2d_b200.grid import TileGrid
from wadi2d_b200.maxima import Tally
from wadi2d_b200.model import Model
from wadi2d_b200.run import DeviceInflow, DeviceRain, run_windows
from wadi2d_b200.state import state_index
from wadi2d_b200.tables import GridTables, hbar_at_level

pytestmark = pytest.mark.gpu


def _plane(n=96):
    w = workloads.v_channel_plane(n=n, dx=10.0, k=5, seed=0)
    og = O.Grid.from_mask(np.ones((n, n), bool), 0.0, 0.0, w.dx)
    tab = O.build_tables(og, w.z, w.dx / w.k, w.manning, local_radius=True)
    g = TileGrid(og.x0, og.y0, og.dx, og.mask)
    return g, GridTables.from_dict(g, tab), w


@pytest.mark.parametrize("case", ["wet", "dry", "rain"])
def test_device_inflow_rates_equal_the_host_form(case):
    """One window: an injection of 1,500 cells (np.sum's pairwise order past 128 terms) and one of 6; levels random
    (case wet), all below the floor (dry: all to the lowest cell), or under rain on half the cells (rain)."""
    g, tables, w = _plane()
    m = Model(tables, Numerics())
    rng = np.random.default_rng(4)
    h = np.where(g.mask, rng.uniform(0.0, 0.3, g.shape), 0.0)
    if case == "dry":
        h = np.minimum(h, 0.01)
    m.set_depth(h)
    jj, ii = np.nonzero(g.mask)
    interior = state_index(g, jj, ii).astype(np.int64)
    pos = {int(k): p for p, k in enumerate(interior)}
    block = np.zeros_like(g.mask)
    block[:60, :40] = g.mask[:60, :40]
    big = state_index(g, *np.nonzero(block))[:1500].astype(np.int64)
    assert big.size == 1500
    small = state_index(g, np.array([70, 70, 70, 71, 71, 71]), np.array([10, 11, 12, 10, 11, 12])).astype(np.int64)
    injections = []
    for name, idx, low in (("big", big, 17), ("small", small, 4)):
        injections.append(F.Injection(name, np.array([pos[int(k)] for k in idx]), idx, low,
                                      np.array([0.0, 600.0, 1800.0]), np.array([0.0, 120.0, 0.0]), 0.1))  # fmt: skip
    storm = F.UniformStorm(50.0, 60.0) if case == "rain" else None
    rained = np.zeros(interior.size, bool)
    rained[: interior.size // 2] = True
    host = F.Forcing(interior, g.dx**2, storm=storm, rained=rained if storm else None, injections=injections,
                     depth_reader=lambda inj: m.read_cells("d", inj.index))  # fmt: skip
    t0, t1 = 300.0, 330.0
    rate, _, vol = host.rate(t0, t1)
    if storm is not None:
        DeviceRain(m, storm, interior[rained]).window(t0, t1)
    dev = DeviceInflow(m, injections, g.dx**2, rained=interior[rained] if storm else None)
    flowing = dev.window(t0, t1)
    src = np.asarray(m.backend.src[interior])
    if storm is None:
        assert np.array_equal(src, rate)
    else:  # the rain pass wrote the rained cells; the inflow cells must match wherever they are
        cells = np.concatenate([inj.cells for inj in injections])
        assert np.array_equal(src[cells], rate[cells])
        assert np.array_equal(src[rained], rate[rained])
    got = dev.volume.cpu().numpy()
    assert [float(x) for x in got[:2]] == [inj.window for inj in injections]
    assert float(got[2]) == vol and vol > 0.0
    assert flowing.size > 0
    if case == "dry":
        for inj in injections:
            nz = np.nonzero(src[inj.cells] != 0.0)[0]
            assert nz.tolist() == [inj.lowest]


def _config2(device_inflow: bool):
    n, k, t_end = 96, 4, 1800.0
    c = workloads.crest_valley(n=n, k=k, breaklines=10, t_end=t_end)
    og = O.Grid.from_mask(np.ones((n, n), bool), 0.0, 0.0, c.dx)
    cr = c.crest
    tab = O.build_tables(og, c.z, c.dx / c.k, c.manning, crest=O.Crest(cr.xz, cr.xlen, cr.xc, cr.yz, cr.ylen, cr.yc))
    g = TileGrid.from_mask(np.ones((n, n), bool), 0.0, 0.0, c.dx)
    m = Model(GridTables.from_dict(g, tab), Numerics())
    rows, cols = c.outfall
    cells = state_index(g, rows, cols).astype(np.int32)
    nb = cells.size
    m.set_boundary(BoundaryCells(cells, cells.copy(), np.ones(nb, np.int32), np.zeros(nb, np.float32),
                                 np.zeros(nb, np.float32)))  # fmt: skip
    rr, rc, level = c.reservoir
    h0 = np.zeros(g.shape)
    h0[rr, rc] = hbar_at_level(np.full(rr.size, level), tab["zmin"][rr, rc], g.from_tiles(tab["hc"])[rr, rc],
                               g.from_tiles(tab["dtab"])[rr, rc])  # fmt: skip
    m.set_depth(h0)
    taken = np.zeros(g.shape, bool)
    taken[rows, cols] = True
    inner = g.mask & ~taken
    jj, ii = np.nonzero(inner)
    interior = state_index(g, jj, ii).astype(np.int64)
    (xf, xs), (yf, ys) = F.open_faces(g, inner, taken)
    tally = Tally(m, xf, xs, yf, ys)
    pos = {int(kk): p for p, kk in enumerate(interior)}
    injections = []
    for q, (ir, icol, low, times, flows) in enumerate(c.inflows):
        idx = state_index(g, ir, icol).astype(np.int64)
        injections.append(F.Injection(f"in{q}", np.array([pos[int(kk)] for kk in idx]), idx, low, times, flows, 0.1))
    if device_inflow:
        out = run_windows(m, t_end, inflow=DeviceInflow(m, injections, c.dx**2), tally=tally)
    else:
        forcing = F.Forcing(interior, c.dx**2, injections=injections,
                            depth_reader=lambda inj: m.read_cells("d", inj.index))  # fmt: skip
        out = run_windows(m, t_end, host_forcing=forcing, tally=tally)
    return m, out


def test_configuration2_with_device_inflows_is_the_host_form_bit_for_bit():
    mh, oh = _config2(False)
    md, od = _config2(True)
    assert md.stepper.nsteps == mh.stepper.nsteps
    assert od.balance.inflow == oh.balance.inflow and od.balance.inflow > 0.0
    assert od.balance.outflow == oh.balance.outflow
    for name in ("h", "d", "u", "v", "mx", "my", "qx", "qy", "res"):
        assert np.array_equal(md.field(name), mh.field(name)), name
