"""A momentum source on faces: the interface of the reference's ``FaceKick`` (wadi2d/solver/momentum.py:18-54), which
``Model.set_momentum`` takes and the host loop applies before every step (wadi2d/solver/stepper.py:111-112).

The face update reads us = (m - dt flux / L) / Abar, so a source of momentum flux S into a face's control volume is
m += dt S / L before the faces are stepped; ``rate`` holds S / L per face (m3/s2). The reference's own FaceKick works
on the B200 backend unchanged (its ``apply`` writes ``backend.mx[faces] += ...`` through the backend's index
adapters); this class gives the same numbers to callers that do not import the reference.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass
class FaceKick:
    """Source rates on x faces (``mx``, positive east) and y faces (``my``, positive south), at reference state
    indices, float32."""

    faces_x: np.ndarray
    rate_x: np.ndarray
    faces_y: np.ndarray
    rate_y: np.ndarray

    @staticmethod
    def build(faces_x, rate_x, faces_y, rate_y) -> FaceKick:
        """Merge repeated faces by summing their rates in FP64 (then float32), so that ``apply`` is one indexed add
        per axis."""
        out = []
        for faces, rate in ((faces_x, rate_x), (faces_y, rate_y)):
            f = np.asarray(faces, np.int64).ravel()
            r = np.broadcast_to(np.asarray(rate, np.float64), f.shape)
            uniq, inverse = np.unique(f, return_inverse=True)
            total = np.bincount(inverse, weights=r, minlength=uniq.size) if f.size else np.zeros(0)
            out += [uniq, total.astype(np.float32)]
        return FaceKick(*out)

    def on(self, backend) -> FaceKick:
        """The kick for a backend: the B200 backend takes host index arrays, so this is the kick itself."""
        return self

    def apply(self, backend, dt: float) -> None:
        """m += float32(dt) * rate on the kicked faces (float32 arithmetic, as the reference's numpy add)."""
        step = np.float32(dt)
        if self.faces_x.size:
            backend.mx[self.faces_x] += step * self.rate_x
        if self.faces_y.size:
            backend.my[self.faces_y] += step * self.rate_y
