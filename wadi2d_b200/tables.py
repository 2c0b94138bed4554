"""Static tables of the step: the records of wadi2d/tables/builder.py:28-115 with the reference's field names, the
FP64 host inverse ``hbar_at_level`` (wadi2d/tables/builder.py:311-331), and ``build_tables``, which builds every
table on the GPU (wadi2d_b200.tablebuild)."""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from wadi2d_b200.grid import TileGrid


@dataclass
class ArrayBed:
    """A bed already in memory, pixels aligned to the grid origin (wadi2d/tables/builder.py:38-60)."""

    z: np.ndarray
    pixel: float
    row_offset: int = 0
    col_offset: int = 0

    def read(self, row0: int, col0: int, nrows: int, ncols: int) -> np.ndarray:
        r = np.clip(np.arange(row0, row0 + nrows) + self.row_offset, 0, self.z.shape[0] - 1)
        c = np.clip(np.arange(col0, col0 + ncols) + self.col_offset, 0, self.z.shape[1] - 1)
        return np.asarray(self.z[np.ix_(r, c)], dtype=np.float64)

    @property
    def span(self) -> int:
        return int(max(self.z.shape))


@dataclass
class CrestFaces:
    """Faces edited by terrain objects, (ny, nx) grids; NaN means untouched; a wall face is closed
    (wadi2d/tables/builder.py:62-80)."""

    xz: np.ndarray
    xlen: np.ndarray
    xc: np.ndarray
    yz: np.ndarray
    ylen: np.ndarray
    yc: np.ndarray
    xwall: np.ndarray | None = None
    ywall: np.ndarray | None = None

    @classmethod
    def empty(cls, shape: tuple[int, int]) -> CrestFaces:
        nan = np.full(shape, np.nan)
        return cls(nan.copy(), np.ones(shape), np.zeros(shape), nan.copy(), np.ones(shape), np.zeros(shape))


@dataclass
class GridTables:
    """Everything static; tile arrays (ntiles, TILE, TILE, ...); suffix x west faces, y north faces
    (wadi2d/tables/builder.py:83-115)."""

    grid: TileGrid
    zmin: np.ndarray
    zbar: np.ndarray
    hc: np.ndarray
    dtab: np.ndarray
    flx: np.ndarray
    frx: np.ndarray
    glx: np.ndarray
    grx: np.ndarray
    efx: np.ndarray
    cwx: np.ndarray
    ftabx: np.ndarray
    fly: np.ndarray
    fry: np.ndarray
    gly: np.ndarray
    gry: np.ndarray
    efy: np.ndarray
    cwy: np.ndarray
    ftaby: np.ndarray
    zcx: np.ndarray
    zcy: np.ndarray

    @property
    def rows(self) -> int:
        return int(self.dtab.shape[-1])

    @classmethod
    def from_dict(cls, grid: TileGrid, d: dict) -> GridTables:
        names = [f for f in cls.__dataclass_fields__ if f != "grid"]
        return cls(grid, **{n: np.asarray(d[n]) for n in names})


def hbar_at_level(level, zmin: np.ndarray, hc: np.ndarray, dtab: np.ndarray) -> np.ndarray:
    """Mean depth that gives exactly this level through the table (the inverse of the step's lookup), FP64."""
    rows = dtab.shape[-1]
    last = rows - 1
    d = np.maximum(np.asarray(level, dtype=np.float64) - zmin, 0.0)
    out = np.where(hc <= 0.0, d, 0.0)
    top = dtab[..., last]
    above = (hc > 0.0) & (d >= top)
    out = np.where(above, hc + (d - top), out)
    inside = (hc > 0.0) & (d < top) & (d > 0.0)
    if inside.any():
        di = d[inside]
        tab = dtab[inside]
        r = np.clip(np.sum(tab <= di[:, None], axis=1) - 1, 0, last - 1)
        idx = np.arange(tab.shape[0])
        lo, hi = tab[idx, r], tab[idx, r + 1]
        s = r + (di - lo) / np.maximum(hi - lo, 1e-30)
        out[inside] = hc[inside] * (s / last) ** 2
    return out


def build_tables(grid, bed, cfg=None, manning=0.035, crest=None, lining=None, device=None, npix=None):
    """Every static array of the step, built on the GPU from the bed's pixels (wadi2d/tables/builder.py:131-258)."""
    from wadi2d_b200.tablebuild import build_tables_gpu

    return build_tables_gpu(grid, bed, cfg, manning, crest, lining, device, npix)
