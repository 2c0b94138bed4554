"""The adapter of tests/golden/cases.py onto this package's CUDA path. Tables come from ``table_source``: the oracle
(test infrastructure, pinned to the reference) by default, so a step comparison sees the reference's own tables;
``"gpu"`` builds them with the package's GPU builder instead. ``arith`` picks the step's build: ``"exact"`` (the
reference's float32 bits) or ``"fast"``."""

from __future__ import annotations

from oracle import oracle as O
from wadi2d_b200 import tables as T
from wadi2d_b200.backend import BoundaryCells
from wadi2d_b200.config import Numerics, Tables
from wadi2d_b200.grid import TileGrid
from wadi2d_b200.maxima import Maxima, Tally
from wadi2d_b200.model import Model


class B200Api:
    def __init__(self, table_source: str = "oracle", device_loop: bool = False, arith: str = "exact") -> None:
        self.dts: list[float] = []
        self.table_source = table_source
        self.device_loop = device_loop
        self.arith = arith
        self.models: list[Model] = []

    def grid(self, mask, x0, y0, dx):
        return TileGrid.from_mask(mask, x0, y0, dx)

    def tables(self, grid, z, pixel, manning, local, crest, npix):
        if self.table_source == "gpu":
            cfg = Tables(face_conveyance="local_radius" if local else "strips")
            return T.build_tables(grid, T.ArrayBed(z, pixel), cfg, manning, crest=crest, npix=npix)
        og = O.Grid(grid.x0, grid.y0, grid.dx, grid.mask)
        d = O.build_tables(og, z, pixel, manning, crest=crest, local_radius=local, npix=npix)
        return T.GridTables.from_dict(grid, d)

    def model(self, grid, tables, numerics):
        m = Model(tables, Numerics(**numerics, arithmetic=self.arith))
        step = m.backend.step

        def logged(dt, want_wave, want_wet):
            self.dts.append(float(dt))
            step(dt, want_wave, want_wet)

        m.backend.step = logged
        if self.device_loop:
            m.advance = lambda t_end, on_step=None: m.run(t_end, maxima=self._maxima, tally=self._tally)
        self._maxima = self._tally = None
        self.models.append(m)
        return m

    def boundary(self, cell, ref, kind, d0, h0):
        return BoundaryCells(cell, ref, kind, d0, h0)

    def maxima(self, m, arrive, deep):
        self._maxima = Maxima(m, arrive, deep)
        return self._maxima

    def tally(self, m, xf, xs, yf, ys):
        self._tally = Tally(m, xf, xs, yf, ys)
        return self._tally

    def hbar_at_level(self, level, zmin, hc, dtab):
        return T.hbar_at_level(level, zmin, hc, dtab)

    def from_tiles(self, grid, tables, name):
        return grid.from_tiles(getattr(tables, name))

    def zmin(self, tables):
        return tables.zmin

    def crest(self, shape):
        return T.CrestFaces.empty(shape)
