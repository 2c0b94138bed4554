"""What a run accumulates on the device: the envelope and the FP64 boundary tally (wadi2d/engine/maxima.py:103-192),
on the B200 backend's own buffers. Same names and methods as the reference's Maxima and Tally."""

from __future__ import annotations

import numpy as np

from wadi2d_b200.layout import HALO, STRIDE, STRIDE2, TILE, TILE2
from wadi2d_b200.state import from_state

NAMES = ("depth", "mean_depth", "speed", "hazard", "arrival")
NOT_ARRIVED = -1.0


def _own_ref_index(ntiles: int) -> np.ndarray:
    """REF_TILE index of every own cell of tiles 1.., in tile-layout order."""
    jj, ii = np.divmod(np.arange(TILE2), TILE)
    t = np.arange(1, ntiles)[:, None]
    return (t * STRIDE2 + (jj[None, :] + HALO) * STRIDE + ii[None, :] + HALO).reshape(-1)


class Maxima:
    """Depth, mean depth, speed, hazard (speed x depth) and arrival envelopes, (ntiles, TILE, TILE) on the device."""

    def __init__(self, model, arrival_depth: float = 0.1, speed_depth: float = 0.05, every: int = 4) -> None:
        self.model = model
        self.backend = model.backend
        self.arrive = float(arrival_depth)
        self.deep = float(speed_depth)
        self.every = int(every)
        self.arrays = self.backend.envelope()
        for a, n in zip(self.arrays, NAMES, strict=True):
            a.fill_(NOT_ARRIVED if n == "arrival" else 0.0)

    def update(self, t: float) -> None:
        self.backend.maxima(t, self.arrive, self.deep)

    def raw(self) -> dict[str, np.ndarray]:
        """The arrays in the reference state layout; halo entries hold the initial value, as the reference's do."""
        nt = self.model.grid.ntiles
        idx = _own_ref_index(nt)
        out = {}
        for n, a in zip(NAMES, self.arrays, strict=True):
            full = np.full(nt * STRIDE2, NOT_ARRIVED if n == "arrival" else 0.0, np.float32)
            full[idx] = a.cpu().numpy()[TILE2:]
            out[n] = full
        return out

    def restore(self, saved: dict[str, np.ndarray]) -> None:
        idx = _own_ref_index(self.model.grid.ntiles)
        torch = self.backend.torch
        for n, a in zip(NAMES, self.arrays, strict=True):
            a[TILE2:] = torch.as_tensor(np.asarray(saved[n], np.float32)[idx], device=a.device)

    def fields(self) -> dict[str, np.ndarray]:
        return {n: from_state(self.model.grid, a) for n, a in self.raw().items()}


class Tally:
    """Volume through a set of faces, m3, one FP64 total per face on the device, positive along the given signs."""

    def __init__(self, model, xfaces, xsign, yfaces, ysign) -> None:
        self.backend = model.backend
        face = np.concatenate((np.asarray(xfaces), np.asarray(yfaces))).astype(np.int64)
        axis = np.concatenate((np.zeros(len(xfaces)), np.ones(len(yfaces)))).astype(np.int32)
        sign = np.concatenate((np.asarray(xsign), np.asarray(ysign))).astype(np.float32)
        self.n = int(face.size)
        self.held = 0.0
        self.total = self.backend.set_tally(face, axis, sign)

    def add(self, dt: float) -> None:
        if self.n:
            self.backend.tally(dt)

    def volume(self) -> float:
        if self.n == 0:
            return self.held
        return self.held + float(self.total.sum().item())

    def restore(self, value: float) -> None:
        self.held = value
        if self.n:
            self.total.zero_()
