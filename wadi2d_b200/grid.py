"""TileGrid: the reference's grid of compact 32 x 32 tiles over a padded raster-aligned mask
(wadi2d/grid/tiles.py:19-101), same attributes and methods."""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from wadi2d_b200.layout import TILE

NEIGHBOURS = ((-1, -1), (-1, 0), (-1, 1), (0, -1), (0, 1), (1, -1), (1, 0), (1, 1))


@dataclass
class TileGrid:
    """Grid geometry and tile bookkeeping. ``mask`` is True on active cells, shape (ny, nx); rows run south."""

    x0: float
    y0: float
    dx: float
    mask: np.ndarray
    tile_of: np.ndarray = field(init=False)
    tiles: np.ndarray = field(init=False)
    nbr: np.ndarray = field(init=False)

    def __post_init__(self) -> None:
        ny, nx = self.mask.shape
        if ny % TILE or nx % TILE:
            raise ValueError("mask shape must be a multiple of the tile size; use TileGrid.from_mask")
        nty, ntx = ny // TILE, nx // TILE
        occ = self.mask.reshape(nty, TILE, ntx, TILE).any(axis=(1, 3))
        self.tile_of = np.zeros((nty, ntx), dtype=np.int32)
        cells = np.argwhere(occ)
        self.tile_of[occ] = np.arange(1, cells.shape[0] + 1, dtype=np.int32)
        self.tiles = np.vstack([np.array([[-1, -1]], dtype=np.int32), cells.astype(np.int32)])
        padded = np.zeros((nty + 2, ntx + 2), np.int32)
        padded[1:-1, 1:-1] = self.tile_of
        tj, ti = self.tiles[1:, 0] + 1, self.tiles[1:, 1] + 1
        self.nbr = np.zeros((self.ntiles, 8), dtype=np.int32)
        for n, (dj, di) in enumerate(NEIGHBOURS):
            self.nbr[1:, n] = padded[tj + dj, ti + di]

    @classmethod
    def from_mask(cls, mask: np.ndarray, x0: float, y0: float, dx: float) -> TileGrid:
        """Pad ``mask`` to whole tiles with one cell of margin on every side (wadi2d/grid/tiles.py:52-64)."""
        ny, nx = mask.shape
        nyp = int(np.ceil((ny + 2) / TILE)) * TILE
        nxp = int(np.ceil((nx + 2) / TILE)) * TILE
        m = np.zeros((nyp, nxp), dtype=bool)
        m[1 : 1 + ny, 1 : 1 + nx] = mask
        return cls(x0 - dx, y0 + dx, dx, m)

    @property
    def ntiles(self) -> int:
        return int(self.tiles.shape[0])

    @property
    def shape(self) -> tuple[int, int]:
        return self.mask.shape

    def cell_of(self, x: float, y: float) -> tuple[int, int]:
        return int((self.y0 - y) // self.dx), int((x - self.x0) // self.dx)

    def xy_of(self, j, i):
        return self.x0 + (i + 0.5) * self.dx, self.y0 - (j + 0.5) * self.dx

    def locate(self, j: int, i: int) -> tuple[int, int, int]:
        return int(self.tile_of[j // TILE, i // TILE]), j % TILE, i % TILE

    def to_tiles(self, a: np.ndarray, dtype=np.float32) -> np.ndarray:
        """Cut a (ny, nx) grid into (ntiles, TILE, TILE); the void tile is zero."""
        ny, nx = self.shape
        blocks = np.asarray(a).reshape((ny // TILE, TILE, nx // TILE, TILE) + a.shape[2:]).swapaxes(1, 2)
        out = np.zeros((self.ntiles, TILE, TILE) + a.shape[2:], dtype=dtype)
        out[1:] = blocks[self.tiles[1:, 0], self.tiles[1:, 1]]
        return out

    def from_tiles(self, a: np.ndarray, fill: float = 0.0) -> np.ndarray:
        """Paste (ntiles, TILE, TILE) back into a (ny, nx) grid."""
        ny, nx = self.shape
        out = np.full((ny // TILE, nx // TILE, TILE, TILE) + a.shape[3:], fill, dtype=a.dtype)
        out[self.tiles[1:, 0], self.tiles[1:, 1]] = a[1:]
        return out.swapaxes(1, 2).reshape((ny, nx) + a.shape[3:])
