"""The adapter of tests/golden/cases.py onto the oracle (test infrastructure)."""

from __future__ import annotations

import numpy as np

from oracle import oracle as O


class OracleApi:
    def __init__(self) -> None:
        self.dts: list[float] = []

    def grid(self, mask, x0, y0, dx):
        return O.Grid.from_mask(mask, x0, y0, dx)

    def tables(self, grid, z, pixel, manning, local, crest, npix):
        return O.build_tables(grid, z, pixel, manning, crest=crest, local_radius=local, npix=npix)

    def model(self, grid, tables, numerics):
        m = O.Model(grid, tables, O.Numerics(**numerics))
        self.dts = m.dts
        return m

    def boundary(self, cell, ref, kind, d0, h0):
        return O.Boundary(cell, ref, kind, d0, h0)

    def maxima(self, m, arrive, deep):
        return O.Maxima(m, arrive, deep)

    def tally(self, m, xf, xs, yf, ys):
        return O.Tally(m, xf, xs, yf, ys)

    def hbar_at_level(self, level, zmin, hc, dtab):
        return O.hbar_at_level(level, zmin, hc, dtab)

    def from_tiles(self, grid, tables, name):
        return grid.from_tiles(tables[name])

    def zmin(self, tables):
        return tables["zmin"]

    def crest(self, shape):
        return O.Crest.empty(shape)
