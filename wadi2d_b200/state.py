"""Host conversions between (ny, nx) grids and the reference's tile-with-halo state layout, and the FP64 host
references of the level and plan lookups (wadi2d/solver/state.py:14-174). The backend's own arrays are NATIVE; these
serve the reference-facing calls (``Model.set_depth``, ``set_velocity``, ``set_source``) and conversions."""

from __future__ import annotations

import numpy as np

from wadi2d_b200.grid import TileGrid
from wadi2d_b200.layout import HALO, STRIDE, STRIDE2, TILE, local_index


def to_state(grid: TileGrid, a: np.ndarray) -> np.ndarray:
    """A (ny, nx) grid into own cells and halos, halos read with clipped indices (wadi2d/solver/state.py:74-84)."""
    ny, nx = grid.shape
    t = np.arange(1, grid.ntiles)
    r = np.clip(grid.tiles[t, 0, None] * TILE + np.arange(STRIDE)[None, :] - HALO, 0, ny - 1)
    c = np.clip(grid.tiles[t, 1, None] * TILE + np.arange(STRIDE)[None, :] - HALO, 0, nx - 1)
    out = np.zeros((grid.ntiles, STRIDE, STRIDE), np.float32)
    out[1:] = np.asarray(a)[r[:, :, None], c[:, None, :]]
    return out.reshape(-1)


def from_state(grid: TileGrid, a: np.ndarray) -> np.ndarray:
    """Own cells of a tile-major array as a (ny, nx) grid."""
    own = np.asarray(a)[: grid.ntiles * STRIDE2].reshape(-1, STRIDE, STRIDE)[:, HALO : HALO + TILE, HALO : HALO + TILE]
    return grid.from_tiles(np.ascontiguousarray(own))


def state_index(grid: TileGrid, j, i):
    tile = grid.tile_of[np.asarray(j) // TILE, np.asarray(i) // TILE]
    return local_index(tile, np.asarray(j) % TILE + HALO, np.asarray(i) % TILE + HALO)


def level_of(h, hc, dtab):
    """Level above zmin for mean depths h, FP64 (wadi2d/solver/state.py:142-155)."""
    last = dtab.shape[-1] - 1
    out = np.array(h, dtype=np.float64)
    wet = hc > 0.0
    above = wet & (h >= hc)
    out[above] = dtab[above, last] + (h[above] - hc[above])
    mid = wet & ~above
    s = np.sqrt(h[mid] / hc[mid]) * last
    r = np.minimum(s.astype(int), last - 1)
    idx = np.arange(r.size)
    t = dtab[mid]
    out[mid] = t[idx, r] + (s - r) * (t[idx, r + 1] - t[idx, r])
    return out


def plan_of(h, hc, dtab):
    """Wet share of the cell plan, FP64 (wadi2d/solver/state.py:164-174)."""
    last = dtab.shape[-1] - 1
    out = np.ones(h.shape, np.float64)
    mid = (hc > 0.0) & (h < hc)
    s = np.sqrt(h[mid] / hc[mid]) * last
    r = np.minimum(s.astype(int), last - 1)
    idx = np.arange(r.size)
    t = dtab[mid]
    out[mid] = hc[mid] * (2 * r + 1) / last**2 / np.maximum(t[idx, r + 1] - t[idx, r], 1e-12)
    return out


def level_field(tables, h):
    g = tables.grid
    return level_of(h, g.from_tiles(tables.hc), g.from_tiles(tables.dtab))


def plan_field(tables, h):
    g = tables.grid
    return plan_of(h, g.from_tiles(tables.hc), g.from_tiles(tables.dtab))
