"""Runs on the B200: the device rain and storage against the host forms, and configuration 1 at full size
(256 x 256 cells, 2 h, CFL 0.9, 1 h of rain) against the oracle field by field, with the mass balance."""

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
from wadi2d_b200.run import DeviceRain, DeviceStorage
from wadi2d_b200.state import state_index
from wadi2d_b200.tables import GridTables

pytestmark = pytest.mark.gpu


def c1(n: int):
    w = workloads.v_channel_plane(n=n, dx=10.0, k=5, seed=0)
    og = O.Grid.from_mask(np.ones((n, n), bool), 0.0, 0.0, w.dx)
    tab = O.build_tables(og, w.z, w.dx / w.k, w.manning)
    g = TileGrid.from_mask(np.ones((n, n), bool), 0.0, 0.0, w.dx)
    return w, og, g, tab


@pytest.mark.parametrize("loss", ["none", "scs", "ic"])
def test_device_rain_equals_host_rate(loss):
    w, og, g, tab = c1(64)
    m = Model(GridTables.from_dict(g, tab), Numerics())
    jj, ii = np.nonzero(g.mask)
    cells = state_index(g, jj, ii).astype(np.int64)
    rng = np.random.default_rng(4)
    mult = rng.lognormal(0.0, 0.4, cells.size)
    storm = F.TriangularStorm(80.0, 180.0)
    cn = rng.choice([60.0, 75.0, 90.0], cells.size)
    lossobj = {"none": None, "scs": F.ScsCurveNumber(cn), "ic": F.InitialConstantLoss(10.0, 2.0)}[loss]
    host = F.Forcing(cells, w.dx**2, storm, depth_factor=mult, loss=lossobj,
                     class_of=np.arange(cells.size) if loss == "scs" else None)  # fmt: skip
    dev = DeviceRain(m, storm, cells, multiplier=mult, loss=lossobj, curve_number=cn if loss == "scs" else None)
    for t0, t1 in ((0.0, 30.0), (1200.0, 1230.0), (5390.0, 5420.0), (10780.0, 10810.0)):
        rate, rain, _ = host.rate(t0, t1)
        vol = dev.window(t0, t1)
        got = m.backend.src[cells]
        assert np.array_equal(got, rate), (loss, t0)
        assert vol == pytest.approx(rain, rel=1e-12, abs=1e-9)


def test_device_storage_equals_host_sum():
    w, og, g, tab = c1(64)
    m = Model(GridTables.from_dict(g, tab), Numerics())
    rng = np.random.default_rng(2)
    m.set_depth(np.where(g.mask, rng.random(g.shape) * 0.3, 0.0))
    jj, ii = np.nonzero(g.mask)
    cells = state_index(g, jj, ii).astype(np.int64)
    assert DeviceStorage(m, cells)() == pytest.approx(F.storage(m, cells), rel=1e-13)


def _drive(m, g, w, rain_rate, outfall, t_mid, t_end, device):
    """Rain for t_mid seconds, then none, to t_end; the outfall tally and books either on the device or the host."""
    rate = np.zeros(g.shape)
    rate[1 : 1 + w.ny, 1 : w.nx] = rain_rate
    m.set_source(rate)
    if device:
        tally = Tally(m, outfall.astype(np.int64), np.ones(outfall.size), np.zeros(0, np.int64), np.zeros(0))
        m.run(t_mid, tally=tally)
        m.set_source(np.zeros(g.shape))
        m.run(t_end, tally=tally)
        return tally.volume()
    tally = O.Tally(m, outfall, np.ones(outfall.size), np.zeros(0, np.int64), np.zeros(0))
    last = [0.0]

    def on_step(st):
        tally.add(st.t - last[0])
        last[0] = st.t

    m.advance(t_mid, on_step)
    m.set_source(np.zeros(g.shape))
    m.advance(t_end, on_step)
    return tally.volume()


def test_configuration1_full_size_matches_the_oracle_and_balances():
    n = 256
    w, og, g, tab = c1(n)
    O.threads(0)
    rows, cols = w.outfall
    out_ref = np.array([state_index(g, int(j), int(i)) for j, i in zip(rows, cols, strict=True)], np.int32)
    nb = out_ref.size
    bc = (out_ref, np.zeros(nb, np.int32), np.ones(nb, np.int32), np.zeros(nb, np.float32), np.zeros(nb, np.float32))
    rain_rate = w.rain_mm_h / 3.6e6
    om = O.Model(og, tab, O.Numerics(cfl=w.cfl))
    om.set_boundary(O.Boundary(*bc))
    out_o = _drive(om, og, w, rain_rate, out_ref, w.rain_s, w.t_end, device=False)
    m = Model(GridTables.from_dict(g, tab), Numerics(cfl=w.cfl))
    m.set_boundary(BoundaryCells(*bc))
    out_g = _drive(m, g, w, rain_rate, out_ref, w.rain_s, w.t_end, device=True)
    assert m.stepper.nsteps == om.nsteps
    for name in ("h", "d", "qx", "qy", "u", "v"):
        a, b = m.field(name), O.from_state(og, om.backend.get_field(name))
        scale = max(float(np.abs(b).max()), 1e-6)
        tol = 1e-5 if name in ("h", "d") else 1e-4 * scale
        assert np.abs(a - b).max() <= tol, name
    assert np.array_equal(m.field("h") > 0, O.from_state(og, om.backend.get_field("h")) > 0)
    assert out_g == pytest.approx(out_o, rel=1e-9)
    # the books: rain in = outflow + storage change (interior cells), FP64
    taken = np.zeros(g.shape, bool)
    taken[rows, cols] = True
    jj, ii = np.nonzero(g.mask & ~taken)
    interior = state_index(g, jj, ii).astype(np.int64)
    area = w.dx**2
    rained = np.zeros(g.shape, bool)
    rained[1 : 1 + w.ny, 1 : w.nx] = True
    cells_rained = int((rained & g.mask & ~taken).sum())
    rain_volume = float(np.float32(rain_rate)) * cells_rained * area * w.rain_s
    bal = F.Balance(rain=rain_volume, outflow=out_g, storage=F.storage(m, interior))
    assert abs(bal.relative) < 1e-6, bal


def test_design_lines_take_the_peak_discharge_every_step():
    from wadi2d_b200.maxima import Lines, faces_across

    w, og, g, tab = c1(64)
    rows, cols = w.outfall
    out_ref = np.array([state_index(g, int(j), int(i)) for j, i in zip(rows, cols, strict=True)], np.int32)
    nb = out_ref.size
    bc = BoundaryCells(out_ref, np.zeros(nb, np.int32), np.ones(nb, np.int32), np.zeros(nb, np.float32),
                       np.zeros(nb, np.float32))  # fmt: skip
    rate = np.zeros(g.shape)
    rate[1 : 1 + w.ny, 1 : w.nx] = w.rain_mm_h / 3.6e6
    jj = np.arange(1, 1 + w.ny)
    lines = [faces_across(g, jj, np.full(jj.size, c), axis=1) for c in (20, 40, 60)]
    lines.append(faces_across(g, np.full(20, 33), np.arange(22, 42), axis=0, sign=-1.0))
    t_end = 1800.0

    dev = Model(GridTables.from_dict(g, tab), Numerics(cfl=w.cfl))
    dev.set_boundary(BoundaryCells(*[np.copy(x) for x in (bc.cell, bc.ref, bc.kind, bc.d0, bc.h0)]))
    dev.set_source(rate)
    ln = Lines(dev, lines)
    dev.run(t_end)
    q_dev, t_dev = ln.peaks()

    host = Model(GridTables.from_dict(g, tab), Numerics(cfl=w.cfl))
    host.set_boundary(bc)
    host.set_source(rate)
    peak = np.zeros(len(lines))
    when = np.zeros(len(lines))

    def on_step(st):
        for n, (xf, xs, yf, ys) in enumerate(lines):
            q = np.dot(host.read_cells("qx", xf), xs) + np.dot(host.read_cells("qy", yf), ys)
            if abs(q) > peak[n]:
                peak[n], when[n] = abs(q), st.t

    host.advance(t_end, on_step)
    assert dev.stepper.nsteps == host.stepper.nsteps
    assert np.all(q_dev > 0.0)
    np.testing.assert_allclose(q_dev, peak, rtol=1e-12)
    assert np.array_equal(t_dev, when)
    qn = ln.discharge()
    xf, xs, yf, ys = lines[1]
    assert qn[1] == pytest.approx(float(np.dot(dev.read_cells("qx", xf), xs)), rel=1e-12)


def test_fp64_level_in_the_near_dry_interval():
    """Numerics.level_fp64: the level of a cell in its table's first interval is formed in FP64 (the row coordinate
    and the interpolation), rounded once to float32; every other cell, and the depth, are as without it."""
    w, og, g, tab = c1(64)
    tables = GridTables.from_dict(g, tab)
    rng = np.random.default_rng(4)
    h0 = rng.uniform(0.0, 0.05, g.shape)  # shallow: many cells in their table's first interval

    def one_step(fp64: bool):
        m = Model(tables, Numerics(level_fp64=fp64))
        m.stepper.adaptive_active = False
        m.set_depth(h0)
        m.run(1e9, max_steps=1)
        return m.field("h"), m.field("d")

    h_off, d_off = one_step(False)
    h_on, d_on = one_step(True)
    assert np.array_equal(h_on, h_off)
    hc = g.from_tiles(tables.hc).astype(np.float32)
    dtab = g.from_tiles(tables.dtab).astype(np.float32)
    last = dtab.shape[-1] - 1
    h = h_on.astype(np.float32)
    inside = (hc > 0) & (h < hc)
    with np.errstate(divide="ignore", invalid="ignore"):
        s = np.sqrt(np.where(inside, h / np.where(hc > 0, hc, 1.0), 0.0).astype(np.float32)) * np.float32(last)
    first = inside & (s.astype(np.int64) == 0)
    assert first.sum() > 100
    assert np.array_equal(d_on[~first], d_off[~first])
    t0, t1 = dtab[..., 0].astype(np.float64), dtab[..., 1].astype(np.float64)
    sd = np.sqrt(h.astype(np.float64) / np.where(hc > 0, hc, 1.0).astype(np.float64)) * float(last)
    want = (t0 + sd * (t1 - t0)).astype(np.float32)
    assert np.array_equal(d_on[first], want[first])


def test_staged_source_windows_equal_the_synchronous_upload():
    """Each window's rates staged by SourceStager (uploaded on a side stream while the window before steps, then put
    in place by a device copy) give the run that a synchronous upload of the same rates gives, bit for bit; the rates
    differ from window to window, so a copy that landed late or early would show."""
    from wadi2d_b200 import _lib
    from wadi2d_b200.run import SourceStager

    w, og, g, tab = c1(64)
    a, b, c = (Model(GridTables.from_dict(g, tab), Numerics(arithmetic="fast")) for _ in range(3))
    for m in (a, b):
        m.stepper.adaptive_active = False
        m.set_depth(np.where(g.mask, 0.02, 0.0))
    rng = np.random.default_rng(9)
    natives = []
    for k in range(6):
        c.set_source(np.where(g.mask, rng.random(g.shape) * 2e-5 * (k + 1), 0.0))
        natives.append(c.backend.native("src").cpu().pin_memory())
    stager = SourceStager(b)
    stager.stage(natives[0])
    for k, rates in enumerate(natives):
        _lib.call("w2b_set_field", a.backend.handle, _lib.FIELD_ID["src"], rates.data_ptr(), _lib.LAYOUT_NATIVE, 1,
                  a.backend._stream())  # fmt: skip
        a.run(30.0 * (k + 1))
        stager.commit()
        if k + 1 < len(natives):
            stager.stage(natives[k + 1])
        b.run(30.0 * (k + 1))
    assert a.stepper.nsteps == b.stepper.nsteps > 6
    for name in ("h", "d", "u", "v", "qx", "qy", "mx", "my", "src"):
        assert np.array_equal(a.field(name), b.field(name)), name


def test_monitor_reads_in_one_round_trip_equal_the_reads_one_by_one():
    """MonitorReads (the design lines' discharge, the outfall volume and the FP64 storage behind one
    synchronisation) gives exactly what Lines.discharge, Tally.volume and DeviceStorage give, window after window."""
    from wadi2d_b200.maxima import Lines, faces_across
    from wadi2d_b200.run import MonitorReads

    w, og, g, tab = c1(64)
    m = Model(GridTables.from_dict(g, tab), Numerics(arithmetic="fast"))
    m.set_depth(np.where(g.mask, 0.02, 0.0))
    rate = np.zeros(g.shape)
    rate[1 : 1 + w.ny, 1 : w.nx] = w.rain_mm_h / 3.6e6
    m.set_source(rate)
    rows, cols = w.outfall
    outfall = np.array([m.cell_state_index(int(j), int(i)) for j, i in zip(rows, cols, strict=True)], np.int64)
    tally = Tally(m, outfall, np.ones(outfall.size), np.zeros(0, np.int64), np.zeros(0))
    line = Lines(m, [faces_across(g, np.full(20, 30), np.arange(20, 40), axis=0),
                     faces_across(g, np.full(10, 50), np.arange(5, 15), axis=0)])  # fmt: skip
    jj, ii = np.nonzero(g.mask)
    storage = DeviceStorage(m, state_index(g, jj, ii).astype(np.int64))
    monitor = MonitorReads(m, line, tally, storage)
    for k in range(1, 5):
        m.run(60.0 * k, tally=tally)
        q, outflow, stored = monitor()
        assert np.array_equal(q, line.discharge())
        assert outflow == tally.volume()
        assert stored == storage()
    assert stored > 0.0


def test_level_cache_holds_the_tables_pairs():
    """After a run, every cell that has a cached row holds the packed table's level pair at that row, bit for bit (the
    update pass gathers from the table only where a cell's row changed and caches what it read)."""
    w, og, g, tab = c1(64)
    m = Model(GridTables.from_dict(g, tab), Numerics(arithmetic="fast"))
    m.set_depth(np.where(g.mask, 0.05, 0.0))
    rate = np.zeros(g.shape)
    rate[1 : 1 + w.ny, 1 : w.nx] = w.rain_mm_h / 3.6e6
    m.set_source(rate)
    m.run(300.0)
    b = m.backend
    b.synchronize()
    nt, rows = g.ntiles, int(m.tables.dtab.shape[-1])
    row = b._t["lrow"].cpu().numpy().reshape(nt, 1024).astype(np.int64)
    pair = b._t["lpair"].cpu().numpy().reshape(nt, 1024, 2)
    table = b._t["dtab2"].cpu().numpy().reshape(nt, rows - 1, 1024, 2)
    t, c = np.nonzero(row != 255)
    assert t.size > 0.5 * (nt - 1) * 1024  # most wet cells have looked a row up
    assert np.all(row[t, c] < rows - 1)
    assert np.array_equal(pair[t, c].view(np.uint32), table[t, row[t, c], c].view(np.uint32))
