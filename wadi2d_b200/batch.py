"""Batches: many independent runs of uneven size advanced together in one device loop (the ensemble / ARF sweep the
reference runs one after another, wadi2d/arf.py:346-372).

Each run keeps its own padded grid (wadi2d/grid/tiles.py:52-64), tables, cell size, clock (t, dt, refresh cadence,
activity checks), sources, boundary cells, envelope and tally. The runs' tile grids are shelf-packed into one grid of
tiles; a run's padding ring (mask False: dry, closed faces) separates it from its neighbours, and tile neighbour links
between runs are cut, so no run wakes another's tiles. A run in a batch therefore steps exactly as it steps alone.
The step kernels read each tile's run (``tile_run``) for its dt, cell size, step flags and current half; every
unfinished run advances one of its own steps per loop step (w2b_advance_runs).
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from wadi2d_b200 import _lib
from wadi2d_b200.backend import B200Backend, BoundaryCells, NumericsRecord
from wadi2d_b200.config import Numerics
from wadi2d_b200.forcing import Balance, UniformStorm
from wadi2d_b200.grid import TileGrid
from wadi2d_b200.layout import GX, GY, STRIDE2, TILE, TILE2, native_of_ref
from wadi2d_b200.maxima import NAMES, NOT_ARRIVED
from wadi2d_b200.state import level_field, plan_field, state_index, to_state
from wadi2d_b200.stepper import NumericalFailure, Stepper
from wadi2d_b200.tablebuild import TILE_FIELDS, DeviceGridTables


CLOCK = np.dtype([("t", "f8"), ("dt", "f8"), ("nsteps", "i8"), ("refresh_due", "i4"), ("status", "i4"),
                  ("wave_max", "f4"), ("nact", "i4")])
"""W2BClock as a numpy record (the same fields, offsets and 40-byte size), so that a batch's clocks pass as one array."""


@dataclass
class Placement:
    oj: int  # tile offsets of the run's grid in the packed grid
    oi: int


def shelf_pack(shapes: list[tuple[int, int]], width: int | None = None) -> tuple[list[Placement], tuple[int, int]]:
    """Tile offsets of grids of (nty, ntx) tiles on shelves of ``width`` tiles (at least the widest grid), tallest
    first. Returns the placements in run order and the packed grid's (nty, ntx)."""
    widest = max(w for _, w in shapes)
    width = max(width or 0, widest)
    order = sorted(range(len(shapes)), key=lambda r: (-shapes[r][0], -shapes[r][1], r))
    out: dict[int, Placement] = {}
    y = x = shelf_h = 0
    for r in order:
        h, w = shapes[r]
        if x + w > width:
            y += shelf_h
            x = shelf_h = 0
        out[r] = Placement(y, x)
        x += w
        shelf_h = max(shelf_h, h)
    return [out[r] for r in range(len(shapes))], (y + shelf_h, width)


def _square_width(shapes: list[tuple[int, int]]) -> int:
    """A shelf width that makes the packed grid roughly square."""
    area = sum(h * w for h, w in shapes)
    return max(max(w for _, w in shapes), int(np.ceil(np.sqrt(area))))


@dataclass
class Packing:
    place: list[Placement]
    map: list[np.ndarray]  # run r's tile t is packed tile map[r][t] (0 -> 0)
    tile_run: np.ndarray  # run of each packed tile (the void tile: 0)
    grid: TileGrid  # the packed grid, neighbour links between runs cut


def pack(grids: list[TileGrid], width: int | None = None) -> Packing:
    """Shelf-pack the runs' tile grids into one grid of tiles (host only)."""
    for g in grids:
        m = g.mask
        if m[0].any() or m[-1].any() or m[:, 0].any() or m[:, -1].any():
            raise ValueError("a run's mask must leave its outer ring of cells False (TileGrid.from_mask does)")
    shapes = [(g.shape[0] // TILE, g.shape[1] // TILE) for g in grids]
    place, (nty, ntx) = shelf_pack(shapes, width or _square_width(shapes))
    mask = np.zeros((nty * TILE, ntx * TILE), bool)
    for g, pl in zip(grids, place, strict=True):
        ny, nx = g.shape
        mask[pl.oj * TILE : pl.oj * TILE + ny, pl.oi * TILE : pl.oi * TILE + nx] = g.mask
    grid = TileGrid(0.0, 0.0, float(grids[0].dx), mask)
    nt = grid.ntiles
    maps = []
    tile_run = np.zeros(nt, np.int32)
    for r, (g, pl) in enumerate(zip(grids, place, strict=True)):
        m = np.zeros(g.ntiles, np.int64)
        m[1:] = grid.tile_of[g.tiles[1:, 0] + pl.oj, g.tiles[1:, 1] + pl.oi]
        if np.any(m[1:] == 0) or len(np.unique(m[1:])) != g.ntiles - 1:
            raise AssertionError("packing lost a tile")
        maps.append(m)
        tile_run[m[1:]] = r
    if sum(g.ntiles - 1 for g in grids) != nt - 1:
        raise AssertionError("packed tiles and run tiles differ")
    # no wake-ups across runs: a neighbour of another run reads as the void tile
    cross = tile_run[grid.nbr] != tile_run[:, None]
    grid.nbr[cross] = 0
    grid.nbr[0] = 0
    return Packing(place, maps, tile_run, grid)


class Batch:
    """Runs ``grids[r]`` with tables ``tables[r]`` (GridTables or DeviceGridTables), one Numerics for all.

    The Model-like setters take one entry per run (None: leave the run as it is) in each run's own grid and indices;
    ``advance`` moves every run to its own end time in one device loop."""

    def __init__(self, grids: list[TileGrid], tables: list, num: Numerics | None = None, device=None,
                 width: int | None = None) -> None:  # fmt: skip
        import torch

        self.torch = torch
        if not torch.cuda.is_available():
            raise RuntimeError("Batch needs a CUDA device; this package has no CPU fallback")
        self.num = num or Numerics()
        if self.num.local_time_stepping:
            raise ValueError("local time stepping is not part of the uniform step")
        self.grids = list(grids)
        self.run_tables = list(tables)
        n = len(grids)
        if n < 1 or len(tables) != n:
            raise ValueError("one table set per grid")
        rows = tables[0].rows
        for tab in tables:
            if tab.rows != rows:
                raise ValueError("every run's tables need the same number of rows")
        packed = pack(grids, width)
        self.place, self.map, self.tile_run, grid = packed.place, packed.map, packed.tile_run, packed.grid
        tile_run = self.tile_run
        nt = grid.ntiles
        self.grid = grid
        dev = torch.device(device if device is not None else "cuda")
        # runs given the same table object (one catchment under many storms) share one copy of it: the static arrays
        # hold each distinct table set once, and every tile reads its set's tile (table_tile)
        distinct: list = []
        owner = []
        for tab in tables:
            u = next((k for k, v in enumerate(distinct) if v is tab), None)
            if u is None:
                u = len(distinct)
                distinct.append(tab)
            owner.append(u)
        shared = len(distinct) < n
        arrays = {}
        table_tile = None
        if shared:
            first = [owner.index(u) for u in range(len(distinct))]
            offset = np.cumsum([1] + [grids[r].ntiles - 1 for r in first])
            table_tile = np.zeros(nt, np.int32)
            for r in range(n):
                table_tile[self.map[r][1:]] = offset[owner[r]] + np.arange(grids[r].ntiles - 1)
            for f in TILE_FIELDS:
                srcs = [self._table_array(tab, f, dev) for tab in distinct]
                arrays[f] = torch.cat([srcs[0][:1]] + [x[1:] for x in srcs])
        else:
            for f in TILE_FIELDS:
                srcs = [self._table_array(tab, f, dev) for tab in tables]
                a = torch.empty((nt,) + tuple(srcs[0].shape[1:]), dtype=srcs[0].dtype, device=dev)
                a[0] = srcs[0][0]
                for r, src in enumerate(srcs):
                    a.index_copy_(0, torch.as_tensor(self.map[r][1:], device=dev), src[1:])
                arrays[f] = a
        self.tables = DeviceGridTables(grid, rows, arrays)
        self.table_tile = table_tile
        self.dx = np.array([g.dx for g in grids], np.float32)
        record = NumericsRecord.from_config(self.num, float(grids[0].dx))
        self.backend = B200Backend(self.tables, record, device=dev, tile_run=tile_run, nruns=n, grid=grid,
                                   table_tile=table_tile)  # fmt: skip
        for f in ("dtab", "ftabx", "ftaby"):  # packed into level-major pairs and quads by the backend
            del arrays[f]
        _lib.call("w2b_set_run_dx", self.backend.handle, self.dx.ctypes.data, n)
        # activity bookkeeping of all runs at once: the cut neighbour links keep the runs apart
        self.stepper = Stepper(self.backend, grid, self.num)
        self.t = np.zeros(n)
        self.dt = np.array([self.num.cfl * float(g.dx) / self.num.wave_floor for g in grids])
        self.nsteps = np.zeros(n, np.int64)
        self.refresh_due = np.ones(n, np.int32)
        self.status = np.zeros(n, np.int32)
        self.boundary_tiles = np.zeros(0, np.int64)
        self._source_tiles = np.zeros(nt, bool)
        # the device holds the activity state between advances: the host's copies are pulled before a host rebuild,
        # and its keep flags and idle counters pushed only when the host changed them
        self._device_newer = False
        self._push_keep = self._push_idle = True
        self._tally = None
        self._tally_slices: list[slice] = [slice(0, 0)] * n

    @staticmethod
    def _table_array(tab, f: str, dev):
        import torch

        on_dev = getattr(tab, "device_arrays", None) or {}
        if f in on_dev:
            return on_dev[f].to(dev)
        return torch.as_tensor(np.ascontiguousarray(getattr(tab, f)), device=dev)

    @property
    def nruns(self) -> int:
        return len(self.grids)

    # ------------------------------------------------------------------ indices

    def state_index(self, r: int, ref_index) -> np.ndarray:
        """Packed reference state indices of run r's reference state indices."""
        k = np.asarray(ref_index, np.int64)
        return self.map[r][k // STRIDE2] * STRIDE2 + k % STRIDE2

    def cells(self, r: int) -> np.ndarray:
        """Packed reference state indices of run r's mask cells, in row-major order of its grid."""
        return self.state_index(r, self.cells_ref(r))

    def native_cells(self, r: int) -> np.ndarray:
        """NATIVE indices of run r's mask cells, in row-major order of its grid."""
        return self.native_of(r, self.cells_ref(r))

    def native_of(self, r: int, ref_index) -> np.ndarray:
        """NATIVE indices (packed) of run r's own reference state indices."""
        return native_of_ref(self.grid.tiles, self.state_index(r, ref_index), self.grid.shape[1])

    def cells_ref(self, r: int) -> np.ndarray:
        """Run r's own reference state indices of its mask cells."""
        g = self.grids[r]
        jj, ii = np.nonzero(g.mask)
        return state_index(g, jj, ii)

    def tiles_of_native(self, native) -> np.ndarray:
        """The packed tiles holding NATIVE indices."""
        k = np.asarray(native, np.int64)
        px = self.backend.px
        j = k // px - GY
        i = k % px - GX
        return np.unique(self.grid.tile_of[j // TILE, i // TILE]).astype(np.int64)

    def _paste(self, per_run: list, fill: float = 0.0) -> np.ndarray:
        """Per-run (ny, nx) grids into one packed grid (None: zeros)."""
        out = np.full(self.grid.shape, fill)
        for g, pl, a in zip(self.grids, self.place, per_run, strict=True):
            if a is None:
                continue
            ny, nx = g.shape
            out[pl.oj * TILE : pl.oj * TILE + ny, pl.oi * TILE : pl.oi * TILE + nx] = np.where(g.mask, a, fill)
        return out

    def halves(self) -> np.ndarray:
        """Each run's current half of the ping-pong pairs (h, u, v, mx, my)."""
        out = np.zeros(self.nruns, np.int32)
        _lib.call("w2b_run_halves", self.backend.handle, out.ctypes.data, self.backend._stream())
        return out

    def _same_halves(self, what: str) -> None:
        if np.any(self.halves() != self.halves()[0]):
            raise RuntimeError(f"{what}: the runs' ping-pong halves differ; set the state before advancing")

    # ------------------------------------------------------------------ the reference model's setters, per run

    def _pull(self) -> None:
        """The device's active list and idle counters into the host's copies, before a host rebuild."""
        if not self._device_newer:
            return
        b = self.backend
        b.active_tiles = b._t["active"][: b.nact].cpu().numpy().astype(np.int32)
        self.stepper.idle[:] = b._t["idle"].cpu().numpy()
        self._device_newer = False

    def set_depth(self, hbars: list) -> None:
        """Mean depth grids (one per run; None: dry), levels through each run's tables in FP64, zero velocities."""
        self._same_halves("set_depth")
        h, d, om = [], [], []
        for g, tab, hb in zip(self.grids, self.run_tables, hbars, strict=True):
            hr = np.where(g.mask, 0.0 if hb is None else hb, 0.0)
            h.append(hr)
            d.append(level_field(tab, hr))
            om.append(plan_field(tab, hr))
        b, grid = self.backend, self.grid
        ph = self._paste(h)
        b.set_field("h", to_state(grid, ph))
        b.set_field("d", to_state(grid, self._paste(d)))
        b.set_field("om", to_state(grid, self._paste(om)))
        ny, nx = grid.shape
        blocks = (ph > 0.0).reshape(ny // TILE, TILE, nx // TILE, TILE).any(axis=(1, 3))
        wet = np.zeros(grid.ntiles, np.int32)
        wet[1:] = blocks[grid.tiles[1:, 0], grid.tiles[1:, 1]]
        b.wet[:] = wet
        self._pull()
        self.stepper.rebuild_active()
        self._push_idle = True

    def set_source(self, rates: list) -> None:
        """Net source rate grids, m/s (one per run; None: no source). Tiles with a source stay active."""
        grid = self.grid
        pr = self._paste(rates)
        self.backend.set_field("src", to_state(grid, pr))
        ny, nx = grid.shape
        blocks = (pr != 0.0).reshape(ny // TILE, TILE, nx // TILE, TILE).any(axis=(1, 3))
        self._source_tiles[:] = False
        self._source_tiles[1:] = blocks[grid.tiles[1:, 0], grid.tiles[1:, 1]]
        self._keep()
        self.refresh_due[:] = 1

    def set_source_tiles(self, tiles: np.ndarray) -> None:
        """Packed tiles kept active for a source written on the device (rain windows)."""
        self._source_tiles[:] = False
        self._source_tiles[np.asarray(tiles, np.int64)] = True
        self._keep()
        self.refresh_due[:] = 1

    def _keep(self) -> None:
        self._pull()
        self._push_keep = True
        st = self.stepper
        st.keep_active[:] = self._source_tiles
        st.keep_active[self.boundary_tiles] = True
        st.keep_active[0] = False
        st.rebuild_active(retain=True)

    def set_boundary(self, per_run: list) -> None:
        """Boundary cells of each run (BoundaryCells in the run's own state indices; None: none)."""
        parts = [b if b is not None else BoundaryCells.empty() for b in per_run]
        cell = np.concatenate([self.state_index(r, b.cell) for r, b in enumerate(parts)]).astype(np.int32)
        ref = np.concatenate([self.state_index(r, b.ref) if len(b.cell) else np.zeros(0, np.int64)
                              for r, b in enumerate(parts)]).astype(np.int32)  # fmt: skip
        bc = BoundaryCells(cell, ref, np.concatenate([np.asarray(b.kind) for b in parts]).astype(np.int32),
                           np.concatenate([np.asarray(b.d0) for b in parts]).astype(np.float32),
                           np.concatenate([np.asarray(b.h0) for b in parts]).astype(np.float32))  # fmt: skip
        self.backend.set_boundary(bc)
        self.boundary_tiles = np.unique(cell.astype(np.int64) // STRIDE2)
        self._keep()

    def set_tally(self, per_run: list) -> None:
        """Tallied faces of each run: (xfaces, xsign, yfaces, ysign) in the run's own state indices, or None."""
        faces, axis, sign, self._tally_slices = [], [], [], []
        at = 0
        for r, spec in enumerate(per_run):
            xf, xs, yf, ys = spec if spec is not None else ((), (), (), ())
            f = np.concatenate((self.state_index(r, np.asarray(xf, np.int64)),
                                self.state_index(r, np.asarray(yf, np.int64))))  # fmt: skip
            faces.append(f)
            axis.append(np.concatenate((np.zeros(len(xf)), np.ones(len(yf)))))
            sign.append(np.concatenate((np.asarray(xs, np.float64), np.asarray(ys, np.float64))))
            self._tally_slices.append(slice(at, at + f.size))
            at += f.size
        self._tally = self.backend.set_tally(np.concatenate(faces), np.concatenate(axis).astype(np.int32),
                                             np.concatenate(sign).astype(np.float32))  # fmt: skip

    def set_lines(self, per_run: list) -> None:
        """Design lines of each run: a list of (xfaces, xsign, yfaces, ysign) in the run's own state indices (or
        None). ``line_peaks`` gives each run's peaks in the same order."""
        from wadi2d_b200.maxima import Lines

        flat, self._line_slices = [], []
        for r, lines in enumerate(per_run):
            at = len(flat)
            for xf, xs, yf, ys in lines or ():
                flat.append((self.state_index(r, np.asarray(xf, np.int64)), xs,
                             self.state_index(r, np.asarray(yf, np.int64)), ys))  # fmt: skip
            self._line_slices.append(slice(at, len(flat)))
        self.lines = Lines(self, flat)

    def line_peaks(self, r: int) -> tuple[np.ndarray, np.ndarray]:
        """Run r's design-line peaks |Q| (m3/s) and their times (s)."""
        q, t = self.lines.peaks()
        s = self._line_slices[r]
        return q[s], t[s]

    # ------------------------------------------------------------------ the loop

    def advance(self, t_end, max_every: int = 0, arrive: float = 0.1, deep: float = 0.05,
                max_steps: int | None = None, raise_on_failure: bool = True) -> np.ndarray:  # fmt: skip
        """Every run to its t_end (one value, or one per run) in one device loop; the envelope every ``max_every`` of
        each run's steps and the tally every step. Returns each run's status (0, or its failure code)."""
        n = self.nruns
        te = np.ascontiguousarray(np.broadcast_to(np.asarray(t_end, np.float64), (n,)))
        b, st, num = self.backend, self.stepper, self.num
        torch = self.torch
        if self._push_keep:
            b._t["keep"].copy_(torch.as_tensor(st.keep_active.astype(np.int32), device=b.device))
            self._push_keep = False
        if self._push_idle:
            b._t["idle"].copy_(torch.as_tensor(st.idle, device=b.device))
            self._push_idle = False
        st._dev_keep = st._dev_idle = None  # this loop keeps its own account of what the device holds
        cfg = _lib.Stepper(num.cfl, num.wave_floor, num.dt_max, num.dt_min, num.dt_every, num.active_every,
                           int(st.adaptive_active), int(max_every), arrive, deep)  # fmt: skip
        clocks = np.zeros(n, CLOCK)
        clocks["t"], clocks["dt"], clocks["nsteps"] = self.t, self.dt, self.nsteps
        clocks["refresh_due"], clocks["nact"] = self.refresh_due, b.nact
        limit = (1 << 62) if max_steps is None else int(max_steps)
        status = int(_lib.lib().w2b_advance_runs(b.handle, ctypes.byref(cfg), te.ctypes.data, limit,
                                                 clocks.ctypes.data, b._stream()))  # fmt: skip
        self.t[:], self.dt[:], self.nsteps[:] = clocks["t"], clocks["dt"], clocks["nsteps"]
        self.status[:] = clocks["status"]
        self.refresh_due[:] = 0
        b.nact = int(clocks["nact"][0])
        self._device_newer = True
        if status not in (_lib.OK, _lib.ENONFINITE, _lib.EDTMIN):
            raise _lib.W2BError(status, "w2b_advance_runs")
        if raise_on_failure and np.any(self.status != 0):
            bad = int(np.nonzero(self.status)[0][0])
            raise NumericalFailure(f"run {bad} failed with status {int(self.status[bad])} at t = {self.t[bad]:.3f} s")
        return self.status.copy()

    def run_windows(self, t_end, storms: list, window: float = 30.0, max_every: int = 0, arrive: float = 0.1,
                    deep: float = 0.05, cells: list | None = None) -> list[Balance]:  # fmt: skip
        """Every run to its t_end under its own uniform storm (any object with ``cumulative_depth(minutes)``), window
        by window as the run driver does for one run (wadi2d/run.py:1712-1740): per window each run's rate over its
        ``cells`` (NATIVE indices; all its mask cells by default) is written on the device (w2b_source_runs), its
        tiles stay active while its rain falls, and the batch advances every run to its own window end. Returns each
        run's books (rain from the float32 rates in FP64; outflow from the tally)."""
        torch = self.torch
        b = self.backend
        n = self.nruns
        te = np.ascontiguousarray(np.broadcast_to(np.asarray(t_end, np.float64), (n,)))
        if cells is None:
            cells = [self.native_cells(r) for r in range(n)]
        counts = np.array([np.asarray(c).size for c in cells], np.float64)
        cat = torch.as_tensor(np.concatenate([np.asarray(c, np.int64) for c in cells]).astype(np.int32), device=b.device)
        run_tiles = [self.tiles_of_native(c) for c in cells]
        rates_dev = torch.zeros(n, dtype=torch.float32, device=b.device)
        area = self.dx.astype(np.float64) ** 2
        books = [Balance() for _ in range(n)]
        uniform = all(isinstance(x, UniformStorm) for x in storms)
        if uniform:  # every storm linear in time: the cumulative depths of all runs at once, element for element
            total = np.array([x.total_depth for x in storms], np.float64)
            dur = np.array([x.duration_minutes for x in storms], np.float64)
        kind = type(storms[0])
        many = getattr(kind, "cumulative_many", None) if all(type(x) is kind for x in storms) else None
        stacked = kind.stack(storms) if many is not None else None
        falling_last = None
        while True:
            live = self.t < te - 1e-9
            if not live.any():
                break
            t0 = self.t.copy()
            t1 = np.where(live, np.minimum(t0 + window, te), t0)
            rates = np.zeros(n, np.float32)
            if uniform:
                f0 = total * np.clip((t0 / 60.0) / dur, 0.0, 1.0)
                f1 = total * np.clip((t1 / 60.0) / dur, 0.0, 1.0)
            elif many is not None:  # storms of one kind that rate many at once, as each would alone
                f0 = many(stacked, t0 / 60.0)
                f1 = many(stacked, t1 / 60.0)
            else:
                f0, f1 = np.zeros(n), np.zeros(n)
                for r in np.nonzero(live)[0]:
                    f0[r] = float(np.asarray(storms[r].cumulative_depth(np.array([t0[r] / 60.0])))[0])
                    f1[r] = float(np.asarray(storms[r].cumulative_depth(np.array([t1[r] / 60.0])))[0])
            span = np.where(live, t1 - t0, 1.0)
            rates[live] = ((f1 - f0) / (1000.0 * span))[live].astype(np.float32)
            falling = live & (f1 > f0)
            for r in np.nonzero(live)[0]:
                books[r].rain += float(rates[r]) * counts[r] * area[r] * (t1[r] - t0[r])
            rates_dev.copy_(torch.as_tensor(rates))
            _lib.call("w2b_source_runs", b.handle, int(cat.numel()), cat.data_ptr(), rates_dev.data_ptr(),
                      b._stream())  # fmt: skip
            if self.stepper.adaptive_active and (falling_last is None
                                                 or not np.array_equal(falling & live, falling_last)):
                keep = [run_tiles[r] for r in np.nonzero(falling & live)[0]]
                tiles = np.concatenate(keep) if keep else np.zeros(0, np.int64)
                st = self.stepper
                if np.all(st.keep_active[tiles]):
                    # no tile joins the kept set: the host's rebuild (retain) would leave the active list as it is,
                    # since every device rebuild already took the wet and kept tiles with their neighbours; only the
                    # kept flags change (they go to the device with the next advance, when they do change)
                    if falling_last is None or not np.array_equal(falling & live, falling_last):
                        self._source_tiles[:] = False
                        self._source_tiles[tiles] = True
                        st.keep_active[:] = self._source_tiles
                        st.keep_active[self.boundary_tiles] = True
                        st.keep_active[0] = False
                        self._push_keep = True
                else:
                    self.set_source_tiles(tiles)
                falling_last = falling & live
            self.refresh_due[live] = 1
            self.advance(t1, max_every=max_every, arrive=arrive, deep=deep)
        out = self.tally_volumes()
        for r in range(n):
            books[r].outflow = float(out[r])
        return books

    # ------------------------------------------------------------------ reading back

    def field(self, r: int, name: str) -> np.ndarray:
        """Run r's field on its own (ny, nx) grid; ping-pong fields read the run's current half."""
        b = self.backend
        b.synchronize()
        if name in ("h", "u", "v", "mx", "my"):
            if name in ("u", "v", "mx", "my"):
                b.sync_momentum()
            t = b._t[name][int(self.halves()[r])]
        elif name in ("d", "qx", "qy", "qx1", "qy1", "res", "src", "om", "zcx", "zcy"):
            t = b._t[name]
        else:
            raise KeyError(name)
        g, pl = self.grids[r], self.place[r]
        ny, nx = g.shape
        px = b.px
        rows = np.arange(ny) + pl.oj * TILE + 4
        cols = np.arange(nx) + pl.oi * TILE + 32
        k = (rows[:, None] * px + cols[None, :]).reshape(-1)
        out = t[self.torch.as_tensor(k, device=b.device)].cpu().numpy().reshape(ny, nx)
        out[~g.mask] = 0.0
        return out

    def volume(self, r: int) -> float:
        return float(self.field(r, "h").sum(dtype=np.float64) * float(self.grids[r].dx) ** 2)

    def reset_envelope(self) -> None:
        for a, nme in zip(self.backend.envelope(), NAMES, strict=True):
            a.fill_(NOT_ARRIVED if nme == "arrival" else 0.0)

    def envelope(self, r: int) -> dict[str, np.ndarray]:
        """Run r's envelope fields on its own (ny, nx) grid, as Maxima.fields gives them for a run alone."""
        g = self.grids[r]
        out = {}
        for nme, a in zip(NAMES, self.backend.envelope(), strict=True):
            tiles = a.view(-1, TILE2)[self.torch.as_tensor(self.map[r], device=a.device)].cpu().numpy()
            out[nme] = g.from_tiles(tiles.reshape(-1, TILE, TILE))
        return out

    def tally_volumes(self) -> np.ndarray:
        """Each run's tallied volume, m3."""
        tot = self._tally.cpu().numpy() if self._tally is not None else np.zeros(0)
        return np.array([float(tot[s].sum()) for s in self._tally_slices])
