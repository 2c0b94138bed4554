"""Checkpoint and resume on the B200 (wadi2d/io/checkpoint.py:23-86): the saved state, envelope, clock and tally come
back exactly in a freshly built model, and the resumed run continues as the uninterrupted one does, bit for bit (every
tile stepped, the refresh cadence of the uninterrupted run). The results file takes the model's maxima and maps."""

from __future__ import annotations

import numpy as np
import pytest

from oracle import oracle as O
from wadi2d_b200 import workloads
from wadi2d_b200.backend import BoundaryCells
from wadi2d_b200.config import Numerics
from wadi2d_b200.forcing import Balance
from wadi2d_b200.grid import TileGrid
from wadi2d_b200.maxima import Maxima, Tally
from wadi2d_b200.model import Model
from wadi2d_b200.runfolder import SAVED_ARRAYS, Results, checkpoint_job, load_checkpoint, read_results, save_checkpoint
from wadi2d_b200.state import state_index
from wadi2d_b200.tables import GridTables

pytestmark = pytest.mark.gpu
N = 64


def _build(tab, g, w):
    m = Model(GridTables.from_dict(g, tab), Numerics(cfl=w.cfl))
    m.stepper.adaptive_active = False
    rows, cols = w.outfall
    cells = np.array([state_index(g, int(j), int(i)) for j, i in zip(rows, cols, strict=True)], np.int32)
    nb = cells.size
    m.set_boundary(BoundaryCells(cells, np.zeros(nb, np.int32), np.ones(nb, np.int32), np.zeros(nb, np.float32),
                                 np.zeros(nb, np.float32)))  # fmt: skip
    rate = np.zeros(g.shape)
    rate[1 : 1 + w.ny, 1 : w.nx] = 3.0 * w.rain_mm_h / 3.6e6
    m.set_source(rate)
    maxima = Maxima(m, 0.1, 0.05, every=4)
    tally = Tally(m, cells.astype(np.int64), np.ones(nb), np.zeros(0, np.int64), np.zeros(0))
    return m, maxima, tally


def test_checkpoint_restores_exactly_and_the_run_continues_bit_for_bit(tmp_path):
    w = workloads.v_channel_plane(n=N, dx=10.0, k=5, seed=0)
    og = O.Grid.from_mask(np.ones((N, N), bool), 0.0, 0.0, w.dx)
    tab = O.build_tables(og, w.z, w.dx / w.k, w.manning)
    g = TileGrid.from_mask(np.ones((N, N), bool), 0.0, 0.0, w.dx)
    a, amax, atal = _build(tab, g, w)
    a.run(900.0, maxima=amax, tally=atal)
    saved = {n: a.backend.get_field(n) for n in SAVED_ARRAYS}
    raw = amax.raw()
    bal = Balance(rain=123.0)
    save_checkpoint(tmp_path / "checkpoint.h5", a, amax, atal, bal, "job-1", times=[0.0, 600.0],
                    series=[{"depth_m": [0.0, 0.5]}], next_series=660.0, next_map=1200.0)  # fmt: skip
    assert checkpoint_job(tmp_path / "checkpoint.h5") == "job-1"
    b, bmax, btal = _build(tab, g, w)
    got = load_checkpoint(tmp_path / "checkpoint.h5", b, bmax, btal, Balance)
    for n in SAVED_ARRAYS:
        own_a = a.field(n)
        assert np.array_equal(b.field(n), own_a), n
        assert np.array_equal(b.backend.get_field(n), saved[n]), n
    for k, v in bmax.raw().items():
        assert np.array_equal(v, raw[k]), k
    assert (b.stepper.t, b.stepper.dt, b.stepper.nsteps) == (a.stepper.t, a.stepper.dt, a.stepper.nsteps)
    assert btal.volume() == pytest.approx(atal.volume(), rel=1e-14)
    assert got["balance"].rain == 123.0 and got["balance"].outflow == pytest.approx(atal.volume(), rel=1e-14)
    assert got["times"] == [0.0, 600.0] and got["series"] == [{"depth_m": [0.0, 0.5]}]
    assert (got["next_series"], got["next_map"]) == (660.0, 1200.0)
    # the resumed run keeps the uninterrupted run's refresh cadence; every tile steps in both
    b.stepper.refresh_due = a.stepper.refresh_due
    a.run(1800.0, maxima=amax, tally=atal)
    b.run(1800.0, maxima=bmax, tally=btal)
    assert b.stepper.nsteps == a.stepper.nsteps
    for n in ("h", "d", "u", "v", "qx", "qy", "res", "om"):
        assert np.array_equal(b.field(n), a.field(n)), n
    fa, fb = amax.fields(), bmax.fields()
    for k in fa:
        assert np.array_equal(fa[k], fb[k]), k
    assert btal.volume() == pytest.approx(atal.volume(), rel=1e-12)
    assert atal.volume() > 0.0
    # the results file takes the envelope and a map
    r = Results(tmp_path / "results.h5", g, "", "{}")
    r.maxima(fa)
    r.snapshot(b.stepper.t, {"depth": b.field("d"), "mean_depth": b.field("h"), "speed": b.cell_speed()})
    r.close()
    f = read_results(tmp_path / "results.h5")
    assert np.array_equal(f.get("maxima/depth"), fa["depth"].astype(np.float32))
    assert np.array_equal(f.get("maps/t000001800/mean_depth"), b.field("h"))
