"""The adapter of tests/golden/cases.py onto the oracle (test infrastructure)."""

from __future__ import annotations

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
        self._maxima = O.Maxima(m, arrive, deep)
        return self._maxima

    def tally(self, m, xf, xs, yf, ys):
        self._tally = O.Tally(m, xf, xs, yf, ys)
        return self._tally

    def hbar_at_level(self, level, zmin, hc, dtab):
        return O.hbar_at_level(level, zmin, hc, dtab)

    def from_tiles(self, grid, tables, name):
        return grid.from_tiles(tables[name])

    def zmin(self, tables):
        return tables["zmin"]

    def crest(self, shape):
        return O.Crest.empty(shape)


class Fp64Api(OracleApi):
    """The FP64 run (oracle/fp64.py) through the same calls, stepped through a given dt sequence: ``advance`` replays
    ``dts`` (a float32 run's own steps) instead of applying the dt rule."""

    def __init__(self, dts) -> None:
        super().__init__()
        self._replay = [float(x) for x in dts]

    def model(self, grid, tables, numerics):
        from oracle import fp64

        m = fp64.Model64(grid, tables, O.Numerics(**numerics))
        replay = self._replay
        m.advance = lambda t_end, on_step=None: m.replay(replay, on_step)
        self.dts = m.dts
        return m

    def maxima(self, m, arrive, deep):
        from oracle import fp64

        self._maxima = fp64.Maxima64(m, arrive, deep)
        return self._maxima

    def tally(self, m, xf, xs, yf, ys):
        from oracle import fp64

        self._tally = fp64.Tally64(m, xf, xs, yf, ys)
        return self._tally
