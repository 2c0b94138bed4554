"""What sets the time step: the face whose wave speed the step rule read, and what stands there. The reference's
``step_limiter`` (wadi2d/solver/limiter.py:113-191) on the B200 backend, with the same report.

The leading tile is the one with the largest wave speed over its cell size (the per-tile maxima the face pass keeps
on refresh steps). Its faces are read on the device (w2b_face_waves: the face pass's own arithmetic for one tile,
writing nothing of the state), where the reference copies the tile to the host and runs its CPU twin; the numbers
are the same, since the face pass is the twin's arithmetic statement for statement. As in the reference, the state
read is the one after the last step, and nothing runs unless a caller asks.
"""

from __future__ import annotations

import numpy as np

from wadi2d_b200 import _lib
from wadi2d_b200.layout import HALO, STRIDE, TILE, TILE2, local_index

NEAR = 0.8
"""Tiles whose wave is within this share of the leading one are counted as limiting too."""


def tile_waves(backend, t: int, dt: float) -> tuple[np.ndarray, np.ndarray, np.ndarray, np.ndarray]:
    """(wx, wy, un_x, un_y) of tile ``t``: the wave speed its west and north faces would report in a step ``dt``
    (m/s) and the face velocities of that step, each (TILE, TILE)."""
    torch = backend.torch
    out = torch.zeros(4 * TILE2, dtype=torch.float32, device=backend.device)
    _lib.call("w2b_face_waves", backend.handle, int(t), float(np.float32(dt)), out.data_ptr(), backend._stream())
    a = out.cpu().numpy().reshape(4, TILE, TILE)
    return a[0], a[1], a[2], a[3]


def face_report(model, t: int, axis: int, j: int, i: int, waves, zmin=None) -> dict:
    """What stands at the west (axis 0) or north (axis 1) face of own cell (j, i) of tile ``t``
    (wadi2d/solver/limiter.py:84-157)."""
    b, grid = model.backend, model.grid
    num = b.num  # the backend's numerics record: g, h_cfl, lead, a_min as the kernels take them
    wx, wy, ux, vy = waves
    s = 1 if axis == 0 else STRIDE
    k = int(local_index(t, j + HALO, i + HALO))
    fid = t * TILE2 + j * TILE + i
    wave = float((wx if axis == 0 else wy)[j, i])
    un = float((ux if axis == 0 else vy)[j, i])
    cells = np.array([k - s, k], np.int64)
    d = b.d[cells].astype(np.float64)
    h = b.h[cells].astype(np.float64)
    om = b.om[cells].astype(np.float64)
    uf = float((b.u if axis == 0 else b.v)[np.array([k])][0])
    ax = "x" if axis == 0 else "y"
    fl, fr, cw = (float(b._t[n + ax][fid]) for n in ("fl", "fr", "cw"))
    e_l, e_r = float(np.float32(d[0]) - np.float32(fl)), float(np.float32(d[1]) - np.float32(fr))
    from_left = uf > 0.0 or (uf == 0.0 and e_l >= e_r)
    up, other = (0, 1) if from_left else (1, 0)
    plan = float(om[up])
    both = bool(d[other] > num.h_cfl)
    if both:
        plan = min(plan, float(om[other]))
    # the kernel's sum |u| + min(lead |du|, 2c) + c, taken apart: the jump term is lead |du| unless 2c was smaller
    jump = num.lead * abs(un - uf)
    rest = wave - abs(un)
    c = rest - jump if rest - jump >= 0.5 * jump else rest / 3.0
    used = max(plan, num.a_min)
    tj, ti = (int(a) for a in grid.tiles[t])
    own = (tj * TILE + j, ti * TILE + i)
    left = (own[0] - 1, own[1]) if axis == 1 else (own[0], own[1] - 1)
    pos = {"up": left if from_left else own, "other": own if from_left else left}
    xy = {key: grid.xy_of(*cell) for key, cell in pos.items()}
    slim = "other" if both and float(om[other]) < float(om[up]) else "up"
    at = up if slim == "up" else other
    out = {
        "tile": int(t), "axis": ax,
        "x": round(float(xy[slim][0]), 2), "y": round(float(xy[slim][1]), 2),
        "j": int(pos[slim][0]), "i": int(pos[slim][1]),
        "face_x": round(0.5 * float(xy["up"][0] + xy["other"][0]), 2),
        "face_y": round(0.5 * float(xy["up"][1] + xy["other"][1]), 2),
        "wave": round(wave, 3), "speed": round(abs(un), 3), "jump": round(max(rest - c, 0.0), 3),
        "celerity": round(c, 3), "depth": round(float(d[at]), 3), "mean_depth": round(float(h[at]), 4),
        "plan": round(float(om[at]), 4), "plan_floor": bool(plan < num.a_min),
        "upwind_depth": round(float(d[up]), 3), "upwind_plan": round(float(om[up]), 4),
        "face_depth": round(max(e_l, e_r), 3), "face_area": round(c * c / num.g * used * grid.dx, 3),
        "hydraulic_depth": round(c * c / num.g, 3), "crest": bool(cw != 0.0), "cell_dx": float(grid.dx),
    }  # fmt: skip
    if zmin is not None:
        jj, ii = pos[slim]
        if 0 <= jj < zmin.shape[0] and 0 <= ii < zmin.shape[1]:
            out["bed"] = round(float(zmin[jj, ii]), 3)
            out["level"] = round(out["bed"] + out["depth"], 3)
    return out


def step_limiter(model, tables=None) -> dict | None:
    """The face that sets the step now: where, what stands there, and the step without its tile; None on a dry run
    (wadi2d/solver/limiter.py:160-191, same keys)."""
    b, grid, st = model.backend, model.grid, model.stepper
    num = st.num
    wave = np.asarray(b.wave, np.float64)
    freq = wave / grid.dx
    freq[0] = 0.0
    t = int(np.argmax(freq))
    if not np.isfinite(freq[t]) or freq[t] <= 0.0:
        return None
    order = np.sort(freq)[::-1]
    floor = num.wave_floor / grid.dx
    strip = float(getattr(b, "extra_wave", 0.0)) / grid.dx
    lead = {
        "dt": round(float(st.dt), 5),
        "dt_tile": round(num.cfl / max(freq[t], floor), 5),
        "dt_without_tile": round(min(num.cfl / max(order[1], strip, floor), num.dt_max), 5),
        "tiles_near": int((freq >= NEAR * freq[t]).sum()),
        "tile_wave": round(float(wave[t]), 3),
    }
    if strip > freq[t]:
        return {"source": "strip", "wave": round(strip * grid.dx, 3), **lead}
    waves = tile_waves(b, t, st.dt)
    axis = 0 if waves[0].max() >= waves[1].max() else 1
    j, i = (int(a) for a in np.unravel_index(int(np.argmax(waves[axis])), (TILE, TILE)))
    zmin = getattr(tables, "zmin", None) if tables is not None else None
    return {"source": "tiles", **face_report(model, t, axis, j, i, waves, zmin), **lead}
