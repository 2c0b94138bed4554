"""The reference's array contract (wadi2d/solver/layout.py:19-50), kept so that reference state indices, tile
layouts and field names mean the same here; and the NATIVE dense layout of this package.

REF_TILE: tile-major with a 2-cell halo, ``k = t * STRIDE2 + j * STRIDE + i``; static arrays (ntiles, TILE, TILE).
NATIVE: the padded grid with GY guard rows and GX guard columns, pitch PX; cell (j, i) at ``(j + GY) * PX + i + GX``.
"""

from __future__ import annotations

import numpy as np

TILE = 32
HALO = 2
STRIDE = TILE + 2 * HALO
STRIDE2 = STRIDE * STRIDE
TILE2 = TILE * TILE
CLOSED = 1.0e9
"""Invert over zmin of a closed face (wadi2d/solver/layout.py:43)."""

STATE_ARRAYS = ("h", "d", "u", "v", "mx", "my", "qx", "qy")
WORK_ARRAYS = ("u1", "v1", "mx1", "my1", "qx1", "qy1", "r", "src", "res", "om")

GY = 4
GX = 32


def local_index(t, j, i):
    return t * STRIDE2 + j * STRIDE + i


def table_index(t, j, i):
    return t * TILE2 + (j - HALO) * TILE + (i - HALO)


def native_pitch(nx: int) -> int:
    return nx + 2 * GX


def native_size(ny: int, nx: int) -> int:
    return (ny + 2 * GY) * native_pitch(nx)


def native_of_ref(tiles: np.ndarray, ref_index, nx: int) -> np.ndarray:
    """NATIVE index of REF_TILE state indices; a halo entry maps to the neighbour cell it copies."""
    k = np.asarray(ref_index, np.int64)
    t = k // STRIDE2
    r = k % STRIDE2
    j = tiles[t, 0].astype(np.int64) * TILE + r // STRIDE - HALO
    i = tiles[t, 1].astype(np.int64) * TILE + r % STRIDE - HALO
    return (j + GY) * native_pitch(nx) + i + GX


def native_of_cell(j, i, nx: int) -> np.ndarray:
    return (np.asarray(j, np.int64) + GY) * native_pitch(nx) + np.asarray(i, np.int64) + GX
