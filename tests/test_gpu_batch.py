"""Batches on the B200: three runs of uneven size, cell size, storm and end time stepped together in one device loop
(w2b_advance_runs) give each run exactly what it gives alone (Model.run through the window driver): the same steps,
bit-identical fields and envelopes, and the same books."""

from __future__ import annotations

import numpy as np
import pytest

from wadi2d_b200 import forcing as F
from wadi2d_b200 import workloads
from wadi2d_b200.backend import BoundaryCells
from wadi2d_b200.batch import Batch
from wadi2d_b200.config import Numerics, Tables
from wadi2d_b200.grid import TileGrid
from wadi2d_b200.maxima import Maxima, Tally
from wadi2d_b200.model import Model
from wadi2d_b200.run import DeviceRain, run_windows
from wadi2d_b200.state import state_index
from wadi2d_b200.tables import ArrayBed, build_tables

pytestmark = pytest.mark.gpu
FIELDS = ("h", "d", "qx", "qy", "u", "v", "res")
RUNS = [  # side, dx, seed, relief, storm depth mm, duration min, recession min, pond depth m
    (40, 10.0, 1, 20.0, 40.0, 20.0, 15.0, 0.0),
    (90, 25.0, 2, 60.0, 60.0, 40.0, 10.0, 0.6),
    (64, 15.0, 3, 30.0, 30.0, 30.0, 25.0, 0.0),
]


def _inputs(n, dx, seed, relief, pond):
    c = workloads.catchment(n=n, dx=dx, k=4, seed=seed, relief=relief, device="cuda")
    grid = TileGrid.from_mask(np.ones((n, n), bool), 0.0, 0.0, dx)
    tables = build_tables(grid, ArrayBed(c.z, dx / 4), Tables(), c.manning, device="cuda")
    rows, cols = c.boundary_cells()
    cells = state_index(grid, rows, cols).astype(np.int32)
    nb = cells.size
    bc = BoundaryCells(cells, cells.copy(), np.ones(nb, np.int32), np.zeros(nb, np.float32), np.zeros(nb, np.float32))
    taken = np.zeros(grid.shape, bool)
    taken[rows, cols] = True
    inner = grid.mask & ~taken
    jj, ii = np.nonzero(inner)
    interior = state_index(grid, jj, ii).astype(np.int64)
    (xf, xs), (yf, ys) = F.open_faces(grid, inner, taken)
    h0 = np.zeros(grid.shape)
    if pond > 0.0:  # a pond in the north-west quarter, to start from a wet state
        h0[1 : 1 + n // 4, 1 : 1 + n // 4] = pond
    return grid, tables, bc, interior, (xf, xs, yf, ys), h0


def _alone(spec, inputs, num):
    n, dx, seed, relief, depth, dur, rec, pond = spec
    grid, tables, bc, interior, tally_spec, h0 = inputs
    m = Model(tables, num)
    m.set_boundary(bc)
    m.set_depth(h0)
    tally = Tally(m, *tally_spec)
    maxima = Maxima(m, 0.1, 0.05, every=4)
    rain = DeviceRain(m, F.UniformStorm(depth, dur), interior)
    out = run_windows(m, (dur + rec) * 60.0, rain=rain, window=30.0, maxima=maxima, tally=tally)
    res = {f: m.field(f) for f in FIELDS}
    res["env"] = maxima.fields()
    res["nsteps"] = m.stepper.nsteps
    res["t"] = m.stepper.t
    res["rain"] = out.balance.rain
    res["outflow"] = out.balance.outflow
    return res


def test_runs_in_a_batch_step_exactly_as_alone():
    num = Numerics()
    inputs = [_inputs(s[0], s[1], s[2], s[3], s[7]) for s in RUNS]
    alone = [_alone(s, i, num) for s, i in zip(RUNS, inputs, strict=True)]
    B = Batch([i[0] for i in inputs], [i[1] for i in inputs], num)
    B.set_boundary([i[2] for i in inputs])
    B.set_depth([i[5] for i in inputs])
    B.set_tally([i[4] for i in inputs])
    B.reset_envelope()
    t_end = np.array([(s[5] + s[6]) * 60.0 for s in RUNS])
    storms = [F.UniformStorm(s[4], s[5]) for s in RUNS]
    cells = [B.native_of(r, i[3]) for r, i in enumerate(inputs)]
    books = B.run_windows(t_end, storms, window=30.0, max_every=4, cells=cells)
    assert len({int(a["nsteps"]) for a in alone}) == len(RUNS)  # the runs do take different step counts
    for r, a in enumerate(alone):
        assert B.nsteps[r] == a["nsteps"], r
        assert B.t[r] == a["t"], r
        for f in FIELDS:
            assert np.array_equal(B.field(r, f), a[f]), (r, f)
        env = B.envelope(r)
        for k, v in a["env"].items():
            assert np.array_equal(env[k], v), (r, k)
        assert books[r].rain == pytest.approx(a["rain"], rel=1e-12)
        assert books[r].outflow == pytest.approx(a["outflow"], rel=1e-12, abs=1e-9)
        assert a["outflow"] > 0.0
        assert float(a["env"]["depth"].max()) > 0.0


def test_batch_storage_reads_each_runs_half():
    num = Numerics()
    inputs = [_inputs(s[0], s[1], s[2], s[3], 0.3) for s in RUNS[:2]]
    B = Batch([i[0] for i in inputs], [i[1] for i in inputs], num)
    B.set_boundary([i[2] for i in inputs])
    B.set_depth([i[5] for i in inputs])
    # three steps of run 0 alone leave the two runs on different halves
    B.advance(np.array([1e9, 0.0]), max_steps=3)
    assert list(B.halves()) == [1, 0]
    assert list(B.nsteps) == [3, 0]
    from wadi2d_b200.run import DeviceStorage

    for r, i in enumerate(inputs):
        g = i[0]
        st = DeviceStorage(B, B.cells(r))()
        jj, ii = np.nonzero(g.mask)
        h = B.field(r, "h")[jj, ii].astype(np.float64) + B.field(r, "res")[jj, ii].astype(np.float64)
        want = float(np.sum(h)) * float(np.float32(g.dx)) ** 2
        assert st == pytest.approx(want, rel=1e-12), r
        assert st > 0.0
