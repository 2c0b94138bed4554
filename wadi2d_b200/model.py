"""Model: tables + backend + stepper, with the reference's methods (wadi2d/solver/model.py:32-188)."""

from __future__ import annotations

import numpy as np

from wadi2d_b200.backend import BoundaryCells, NumericsRecord, select_backend
from wadi2d_b200.config import Numerics
from wadi2d_b200.layout import HALO, STRIDE, STRIDE2, TILE, local_index
from wadi2d_b200.state import from_state, level_field, plan_field, to_state
from wadi2d_b200.stepper import Stepper
from wadi2d_b200.tables import GridTables


class Model:
    def __init__(self, tables: GridTables, num: Numerics | None = None, backend: str = "auto") -> None:
        self.tables = tables
        self.grid = tables.grid
        self.num = num or Numerics()
        if self.num.local_time_stepping:
            raise ValueError("local time stepping is not part of the uniform step")
        record = NumericsRecord.from_config(self.num, self.grid.dx)
        self.backend = select_backend(backend, tables, record)
        self.stepper = Stepper(self.backend, self.grid, self.num)
        self.boundary_tiles = np.zeros(0, np.int64)

    def set_depth(self, hbar: np.ndarray) -> None:
        """Mean depth grid, with levels through the table (FP64, as the reference) and zero velocities."""
        h = np.where(self.grid.mask, hbar, 0.0)
        d = level_field(self.tables, h)
        self.backend.set_field("h", to_state(self.grid, h))
        self.backend.set_field("d", to_state(self.grid, d))
        self.backend.set_field("om", to_state(self.grid, plan_field(self.tables, h)))
        self.backend.wet[:] = self._tile_wet(h)
        self.stepper.rebuild_active()

    def _tile_wet(self, h: np.ndarray) -> np.ndarray:
        g = self.grid
        ny, nx = g.shape
        blocks = (h > 0.0).reshape(ny // TILE, TILE, nx // TILE, TILE).any(axis=(1, 3))
        out = np.zeros(g.ntiles, np.int32)
        out[1:] = blocks[g.tiles[1:, 0], g.tiles[1:, 1]]
        return out

    def set_velocity(self, ucell: np.ndarray, vcell: np.ndarray) -> None:
        """Face velocities from cell-centred ones; momentum and discharge follow (wadi2d/solver/model.py:81-97)."""
        dx = self.grid.dx
        h = self.field("h")
        for axis, (uname, mname, qname), cell in ((1, ("u", "mx", "qx"), ucell), (0, ("v", "my", "qy"), vcell)):
            un = np.roll(cell, 1, axis=axis)
            hn = np.roll(h, 1, axis=axis)
            face = 0.5 * (cell + un)
            face = np.where((h > 0.0) & (hn > 0.0), face, 0.0)
            abar = 0.5 * (h + hn) * dx
            up = np.where(face > 0.0, hn, h) * dx
            self.backend.set_field(uname, to_state(self.grid, face))
            self.backend.set_field(mname, to_state(self.grid, abar * face))
            self.backend.set_field(qname, to_state(self.grid, up * face))

    def set_source(self, rate: np.ndarray) -> None:
        """Net source rate per cell, m/s, on a (ny, nx) grid; its tiles stay active."""
        g = self.grid
        self.backend.set_field("src", to_state(g, np.where(g.mask, rate, 0.0)))
        ny, nx = g.shape
        blocks = (np.asarray(rate) != 0.0).reshape(ny // TILE, TILE, nx // TILE, TILE).any(axis=(1, 3))
        keep = self.stepper.keep_active
        keep[:] = False
        keep[1:] = blocks[g.tiles[1:, 0], g.tiles[1:, 1]]
        keep[self.boundary_tiles] = True
        self.stepper.rebuild_active(retain=True)
        self.stepper.refresh_due = True

    def set_source_cells(self, cells: np.ndarray, rate: np.ndarray) -> None:
        """``rate`` per entry of ``cells`` (reference state indices of own cells)."""
        src = np.zeros(self.grid.ntiles * STRIDE2, np.float32)
        src[cells] = rate
        self.backend.set_field("src", src)
        keep = self.stepper.keep_active
        keep[:] = False
        keep[np.asarray(cells)[np.asarray(rate) != 0.0] // STRIDE2] = True
        keep[self.boundary_tiles] = True
        self.stepper.rebuild_active(retain=True)
        self.stepper.refresh_due = True

    def kicks_faces(self) -> bool:
        return True

    def set_momentum(self, kick) -> None:
        """A momentum source on faces (the reference's FaceKick) for the steps until the next call."""
        self.stepper.kick = None if kick is None else kick.on(self.backend)

    def device_index(self, index):
        return index

    def read_cells(self, name: str, index) -> np.ndarray:
        return getattr(self.backend, name)[index]

    def set_boundary(self, bc: BoundaryCells) -> None:
        self.backend.set_boundary(bc)
        self.boundary_tiles = np.unique(np.asarray(bc.cell) // STRIDE2)
        self.stepper.keep_active[self.boundary_tiles] = True
        self.stepper.pin(self.boundary_tiles)
        self.stepper.rebuild_active(retain=True)

    def advance(self, t_end: float, on_step=None) -> float:
        return self.stepper.advance(t_end, on_step)

    def run(self, t_end: float, maxima=None, tally=None, max_steps: int | None = None) -> float:
        """``advance`` resident on the device; ``maxima`` (this package's Maxima) is taken every ``maxima.every``
        steps and the boundary ``tally`` every step inside the loop."""
        if tally is not None and tally.backend is not self.backend:
            raise ValueError("the tally belongs to another model")
        every = 0 if maxima is None else int(maxima.every)
        arrive = 0.1 if maxima is None else maxima.arrive
        deep = 0.05 if maxima is None else maxima.deep
        return self.stepper.run(t_end, every, arrive, deep, max_steps)

    def field(self, name: str) -> np.ndarray:
        self.backend.synchronize()
        return from_state(self.grid, self.backend.get_field(name))

    def cell_speed(self) -> np.ndarray:
        u, v = self.field("u"), self.field("v")
        return np.hypot(0.5 * (u + np.roll(u, -1, axis=1)), 0.5 * (v + np.roll(v, -1, axis=0)))

    def discharge_x(self) -> np.ndarray:
        return self.field("qx")

    def discharge_y(self) -> np.ndarray:
        return self.field("qy")

    def volume(self) -> float:
        return float(self.field("h").sum(dtype=np.float64) * self.grid.dx**2)

    def cell_state_index(self, j: int, i: int) -> int:
        t, oj, oi = self.grid.locate(j, i)
        return int(local_index(t, oj + HALO, oi + HALO))


__all__ = ["HALO", "STRIDE", "BoundaryCells", "Model"]
