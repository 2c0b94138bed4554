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


class Lines:
    """Design lines: the discharge through each line's faces (wadi2d/engine/monitor.py:229-232), taken on the device
    at every step of the device loop, with its running peak |Q| and the time of the peak (the figures
    wadi2d/run.py:1839-1843 reads off the line series). ``lines``: per line (xfaces, xsign, yfaces, ysign), reference
    state indices and signs (+1: positive to the line's right), as wadi2d/forcing.py:411-425 gives them."""

    def __init__(self, model, lines: list) -> None:
        from wadi2d_b200 import _lib
        from wadi2d_b200.layout import native_of_ref

        b = model.backend
        torch = b.torch
        grid = model.grid
        start, face, axis, sign = [0], [], [], []
        for xf, xs, yf, ys in lines:
            f = np.concatenate((np.asarray(xf, np.int64), np.asarray(yf, np.int64)))
            face.append(native_of_ref(grid.tiles, f, grid.shape[1]))
            axis.append(np.concatenate((np.zeros(len(xf)), np.ones(len(yf)))))
            sign.append(np.concatenate((np.asarray(xs, np.float64), np.asarray(ys, np.float64))))
            start.append(start[-1] + f.size)
        n = len(lines)
        dev = b.device

        def put(a, dtype):
            return torch.as_tensor(np.ascontiguousarray(a), device=dev).to(dtype)

        cat = (lambda parts: np.concatenate(parts) if parts else np.zeros(0))  # noqa: E731
        self._t = (put(start, torch.int32), put(cat(face), torch.int32), put(cat(axis), torch.int32),
                   put(cat(sign), torch.float32), torch.zeros(max(n, 1), dtype=torch.float64, device=dev),
                   torch.zeros(max(n, 1), dtype=torch.float64, device=dev),
                   torch.zeros(max(n, 1), dtype=torch.float64, device=dev))  # fmt: skip
        self.n = n
        b._lines = self._t  # the handle keeps raw pointers: the backend keeps the tensors
        _lib.call("w2b_set_lines", b.handle, n, *[x.data_ptr() for x in self._t])

    def discharge(self) -> np.ndarray:
        """Each line's discharge after the last step, m3/s."""
        return self._t[4][: self.n].cpu().numpy()

    def discharge_device(self):
        """The same, as the device FP64 tensor (no copy to the host)."""
        return self._t[4][: self.n]

    def peaks(self) -> tuple[np.ndarray, np.ndarray]:
        """Each line's peak |Q| (m3/s) and the time it was reached (s)."""
        return self._t[5][: self.n].cpu().numpy(), self._t[6][: self.n].cpu().numpy()

    def reset(self) -> None:
        for x in self._t[4:]:
            x.zero_()


def faces_across(grid, j, i, axis: int, sign: float = 1.0):
    """A design line through cells (j, i) crossing their west faces (axis 1: x faces, eastward flow positive for
    sign +1) or their north faces (axis 0: y faces, southward flow positive), as the (xfaces, xsign, yfaces, ysign)
    of wadi2d/forcing.py:411-425. Faces with an inactive cell on either side are left out."""
    from wadi2d_b200.state import state_index

    j, i = np.atleast_1d(np.asarray(j, np.int64)), np.atleast_1d(np.asarray(i, np.int64))
    keep = grid.mask[j, i] & (grid.mask[j, i - 1] if axis == 1 else grid.mask[j - 1, i])
    f = np.asarray(state_index(grid, j[keep], i[keep]), np.int64)
    s = np.full(f.size, float(sign))
    none = (np.zeros(0, np.int64), np.zeros(0))
    return (f, s) + none if axis == 1 else none + (f, s)
