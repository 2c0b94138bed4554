"""Stepper: the time loop of wadi2d/solver/stepper.py:24-129, same fields and rules.

``advance`` is the reference's host loop, statement for statement (one ``backend.step`` per step, the host reading
the wave speed back on refresh steps and the wet flags on active-list steps). ``run`` is the same loop resident on
the device (``w2b_advance``): step rule, refresh cadence, sleeping tiles, the envelope every ``max_every`` steps and
the boundary tally every step, captured as CUDA graphs, with one host read per graph of 16 steps.
"""

from __future__ import annotations

from collections.abc import Callable
from dataclasses import dataclass

import numpy as np

from wadi2d_b200 import _lib
from wadi2d_b200.config import Numerics
from wadi2d_b200.grid import TileGrid
from wadi2d_b200.layout import STRIDE2

SLEEP_CHECKS = 2


class NumericalFailure(RuntimeError):
    """The time step collapsed or a NaN appeared."""


@dataclass
class Stepper:
    backend: object
    grid: TileGrid
    num: Numerics
    t: float = 0.0
    dt: float = 0.01
    nsteps: int = 0

    def __post_init__(self) -> None:
        self.adaptive_active = True
        self.keep_active = np.zeros(self.grid.ntiles, bool)
        self.pinned = np.zeros(self.grid.ntiles, bool)
        self.refresh_due = True
        self.dt = self.num.cfl * self.grid.dx / self.num.wave_floor
        self.kick = None
        self.wake_rules: list[Callable[[np.ndarray], np.ndarray]] = []
        self.idle = np.zeros(self.grid.ntiles, np.int32)
        # what the device's keep flags and idle counts hold, as far as this stepper knows (None: unknown); the device
        # loop uploads them only when the host's copies differ, so that a window's advance issues no host-to-device
        # copy of its own while the next window's source is uploaded (run.SourceStager)
        self._dev_keep: np.ndarray | None = None
        self._dev_idle: np.ndarray | None = None

    def pin(self, tiles: np.ndarray) -> None:
        """Tiles that must see every smallest step; the uniform step has no other kind."""

    def check_period(self) -> int:
        return int(self.num.active_every)

    def rebuild_active(self, retain: bool = False, check: bool = False) -> None:
        """wadi2d/solver/stepper.py:56-92."""
        ntiles = self.grid.ntiles
        if not self.adaptive_active:
            if int(self.backend.nact) != ntiles - 1:
                self.backend.set_active(np.arange(1, ntiles, dtype=np.int32))
            return
        wet = self.backend.wet_flags().astype(bool) | self.keep_active
        wet[0] = False
        act = wet.copy()
        act[self.grid.nbr[wet].ravel()] = True
        for rule in self.wake_rules:
            act |= rule(wet)
        current = np.zeros(ntiles, bool)
        current[self.backend.active_tiles] = True
        if retain:
            act |= current
        elif check:
            self.idle[act] = 0
            self.idle[~act] += 1
            act |= current & (self.idle < SLEEP_CHECKS)
        else:
            self.idle[:] = 0
        act[0] = False
        woken = act & ~current
        self.backend.set_active(np.nonzero(act)[0].astype(np.int32))
        if (retain or check) and woken.any():
            self._wake(np.nonzero(woken)[0].astype(np.int32))

    def _wake(self, tiles: np.ndarray) -> None:
        self.backend.refresh_plan(tiles)
        self.backend.refresh_halos()

    def advance(self, t_end: float, on_step: Callable[[Stepper], None] | None = None) -> float:
        """Run to ``t_end`` exactly, host-driven (wadi2d/solver/stepper.py:101-129)."""
        b = self.backend
        num = self.num
        dx = self.grid.dx
        while self.t < t_end - 1e-9:
            refresh = self.refresh_due or self.nsteps % num.dt_every == 0
            self.refresh_due = False
            activate = self.nsteps % num.active_every == 0
            dt = min(self.dt, t_end - self.t, num.dt_max)
            if self.kick is not None:
                self.kick.apply(b, dt)
            b.step(dt, refresh, activate)
            self.t += dt
            self.nsteps += 1
            if refresh:
                w = b.max_wave()
                if not np.isfinite(w):
                    raise NumericalFailure(f"non-finite wave speed at t = {self.t:.3f} s")
                self.dt = min(num.cfl * dx / max(w, num.wave_floor), num.dt_max)
                if self.dt < num.dt_min:
                    raise NumericalFailure(f"time step {self.dt:.2e} s below the minimum at t = {self.t:.3f} s")
            if activate and self.adaptive_active:
                self.rebuild_active(check=True)
            if on_step is not None:
                on_step(self)
        return self.t

    def run(self, t_end: float, max_every: int = 0, arrive: float = 0.1, deep: float = 0.05,
            max_steps: int | None = None) -> float:  # fmt: skip
        """``advance`` resident on the device: the envelope (if ``max_every``) and the backend's boundary tally are
        taken inside the loop. Returns t; raises NumericalFailure as ``advance`` does."""
        if self.kick is not None or self.wake_rules or getattr(self.backend, "hooks", None) is not None:
            raise RuntimeError("a face kick, wake rule or hook needs the host loop: use advance")
        b = self.backend
        torch = b.torch
        if not self.adaptive_active and int(b.nact) != self.grid.ntiles - 1:
            b.set_active(np.arange(1, self.grid.ntiles, dtype=np.int32))
        keep = self.keep_active.astype(np.int32)
        if self._dev_keep is None or not np.array_equal(keep, self._dev_keep):
            b._t["keep"].copy_(torch.as_tensor(keep, device=b.device))
            self._dev_keep = keep
        if self._dev_idle is None or not np.array_equal(self.idle, self._dev_idle):
            b._t["idle"].copy_(torch.as_tensor(self.idle, device=b.device))
        num = self.num
        cfg = _lib.Stepper(num.cfl, num.wave_floor, num.dt_max, num.dt_min, num.dt_every, num.active_every,
                           int(self.adaptive_active), int(max_every), arrive, deep)  # fmt: skip
        clock = _lib.Clock(self.t, self.dt, self.nsteps, int(self.refresh_due), 0, 0.0, int(b.nact))
        limit = (1 << 62) if max_steps is None else int(max_steps)
        status = b.advance_device(cfg, t_end, limit, clock)
        self.t, self.dt, self.nsteps = float(clock.t), float(clock.dt), int(clock.nsteps)
        self.refresh_due = False
        nact = int(clock.nact)
        b.active_tiles = b._t["active"][:nact].cpu().numpy().astype(np.int32)
        b.nact = nact
        self.idle[:] = b._t["idle"].cpu().numpy()
        self._dev_idle = self.idle.copy()
        if status == _lib.ENONFINITE:
            raise NumericalFailure(f"non-finite wave speed at t = {self.t:.3f} s")
        if status == _lib.EDTMIN:
            raise NumericalFailure(f"time step {self.dt:.2e} s below the minimum at t = {self.t:.3f} s")
        if status != _lib.OK:
            raise _lib.W2BError(status, "w2b_advance")
        return self.t


def state_size(grid: TileGrid) -> int:
    return grid.ntiles * STRIDE2
