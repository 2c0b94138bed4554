"""CPU oracle of Wadi2D's uniform-grid shallow-water step. TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` may import this module; the
product package ``wadi2d_b200`` never does, and its CUDA path fails loudly rather than fall back to anything here.

It restates, in numpy plus the C file ``wadi_oracle.c`` (float32 kernels, float64 table builder), the reference's
own CPU path:

* grid and tiles          wadi2d/grid/tiles.py:19-101
* state layout, maps      wadi2d/solver/layout.py:19-50, wadi2d/solver/state.py:14-174
* table build             wadi2d/tables/builder.py:131-331, wadi2d/tables/core.py:16-371
* backend                 wadi2d/solver/cpu/backend.py:14-141
* stepper                 wadi2d/solver/stepper.py:24-133
* model                   wadi2d/solver/model.py:32-188
* envelope and tally      wadi2d/engine/maxima.py:75-192

Parity is pinned: ``tests/test_oracle_golden.py`` checks every array here bit for bit against vectors that
``tests/golden/make_golden.py`` made by running the reference itself.
"""

from __future__ import annotations

import ctypes
import subprocess
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "_build" / "liboracle.so"

TILE = 32
HALO = 2
STRIDE = TILE + 2 * HALO
STRIDE2 = STRIDE * STRIDE
TILE2 = TILE * TILE
CLOSED = 1.0e9
G = 9.80665
CRITICAL_WEIR_COEFF = 1.7046
NEIGHBOURS = ((-1, -1), (-1, 0), (-1, 1), (0, -1), (0, 1), (1, -1), (1, 0), (1, 1))
SLEEP_CHECKS = 2

_F32P = ctypes.POINTER(ctypes.c_float)
_F64P = ctypes.POINTER(ctypes.c_double)
_I32P = ctypes.POINTER(ctypes.c_int32)
_I64P = ctypes.POINTER(ctypes.c_int64)


def build(force: bool = False) -> Path:
    """Compile ``wadi_oracle.c`` with IEEE float arithmetic (no FMA contraction, no fast math) and OpenMP."""
    src = HERE / "wadi_oracle.c"
    if LIB_PATH.exists() and not force and LIB_PATH.stat().st_mtime >= src.stat().st_mtime:
        return LIB_PATH
    LIB_PATH.parent.mkdir(parents=True, exist_ok=True)
    cmd = [
        "gcc", "-O2", "-fopenmp", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-shared",
        "-o", str(LIB_PATH), str(src), "-lm",
    ]  # fmt: skip
    subprocess.run(cmd, check=True)
    return LIB_PATH


class OrParams(ctypes.Structure):
    _fields_ = [(n, ctypes.c_float) for n in ("g", "dx", "e_wet", "h_cfl", "u_max", "lead", "a_min")] + [
        (n, ctypes.c_int32) for n in ("rows", "second", "sheet", "mirror", "carry")
    ]


_ARRAY_FIELDS = (
    "h d u v mx my qx qy u1 v1 mx1 my1 qx1 qy1 r src res om zcx zcy Hc dtab "
    "flx frx glx grx efx cwx ftabx fly fry gly gry efy cwy ftaby wave"
).split()


class OrArrays(ctypes.Structure):
    _fields_ = [(n, _F32P) for n in _ARRAY_FIELDS] + [("wet", _I32P)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        path = build()
        L = ctypes.CDLL(str(path))
        P = ctypes.POINTER
        L.or_threads.argtypes = [ctypes.c_int]
        L.or_threads.restype = ctypes.c_int
        L.or_faces.argtypes = [P(OrArrays), P(OrParams), _I32P, ctypes.c_int, ctypes.c_float, ctypes.c_int]
        L.or_limit.argtypes = [P(OrArrays), P(OrParams), _I32P, ctypes.c_int, ctypes.c_float]
        L.or_update.argtypes = [P(OrArrays), P(OrParams), _I32P, ctypes.c_int, ctypes.c_float, ctypes.c_int]
        L.or_plan.argtypes = [P(OrArrays), P(OrParams), _I32P, ctypes.c_int]
        L.or_exchange.argtypes = [_I32P, ctypes.c_int, _I32P, _I32P, ctypes.c_int, _F32P]
        L.or_boundary.argtypes = [ctypes.c_int, _I32P, _I32P, _I32P, _F32P, _F32P, _F32P, _F32P]
        L.or_maxima.argtypes = [_I32P, ctypes.c_int] + [ctypes.c_float] * 3 + [_F32P] * 9
        L.or_tally.argtypes = [ctypes.c_int, ctypes.c_double, _I32P, _I32P, _F32P, _F32P, _F32P, _F64P]
        L.or_cell_table.argtypes = [_F64P, ctypes.c_int, ctypes.c_int, _F64P, _F64P, _F64P]
        L.or_tile_tables.argtypes = (
            [_F64P, ctypes.c_int, ctypes.c_int, ctypes.c_double, _F64P, _F64P, _F64P, _F64P, _F64P, _F64P]
            + [ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_double]
            + [_F64P] * 10
        )
        _lib = L
    return _lib


def threads(n: int = 0) -> int:
    """Set (n > 0) and return the OpenMP thread count of the C kernels."""
    return int(lib().or_threads(int(n)))


def _p(a, t=_F32P):
    return None if a is None else a.ctypes.data_as(t)


# ---------------------------------------------------------------------------------------------------- grid


@dataclass
class Grid:
    """Tiles of a padded raster-aligned grid (wadi2d/grid/tiles.py:19-64). Rows run south."""

    x0: float
    y0: float
    dx: float
    mask: np.ndarray
    tile_of: np.ndarray = field(init=False)
    tiles: np.ndarray = field(init=False)
    nbr: np.ndarray = field(init=False)

    def __post_init__(self) -> None:
        ny, nx = self.mask.shape
        assert ny % TILE == 0 and nx % TILE == 0
        nty, ntx = ny // TILE, nx // TILE
        occ = self.mask.reshape(nty, TILE, ntx, TILE).any(axis=(1, 3))
        self.tile_of = np.zeros((nty, ntx), np.int32)
        cells = np.argwhere(occ)
        self.tile_of[occ] = np.arange(1, cells.shape[0] + 1, dtype=np.int32)
        self.tiles = np.vstack([np.array([[-1, -1]], np.int32), cells.astype(np.int32)])
        self.nbr = np.zeros((self.ntiles, 8), np.int32)
        for t in range(1, self.ntiles):
            tj, ti = self.tiles[t]
            for n, (dj, di) in enumerate(NEIGHBOURS):
                j2, i2 = tj + dj, ti + di
                if 0 <= j2 < nty and 0 <= i2 < ntx:
                    self.nbr[t, n] = self.tile_of[j2, i2]

    @classmethod
    def from_mask(cls, mask: np.ndarray, x0: float, y0: float, dx: float) -> Grid:
        ny, nx = mask.shape
        nyp = int(np.ceil((ny + 2) / TILE)) * TILE
        nxp = int(np.ceil((nx + 2) / TILE)) * TILE
        m = np.zeros((nyp, nxp), bool)
        m[1 : 1 + ny, 1 : 1 + nx] = mask
        return cls(x0 - dx, y0 + dx, dx, m)

    @property
    def ntiles(self) -> int:
        return int(self.tiles.shape[0])

    @property
    def shape(self) -> tuple[int, int]:
        return self.mask.shape

    def to_tiles(self, a: np.ndarray, dtype=np.float32) -> np.ndarray:
        out = np.zeros((self.ntiles, TILE, TILE) + a.shape[2:], dtype=dtype)
        for t in range(1, self.ntiles):
            tj, ti = self.tiles[t]
            out[t] = a[tj * TILE : (tj + 1) * TILE, ti * TILE : (ti + 1) * TILE]
        return out

    def from_tiles(self, a: np.ndarray, fill: float = 0.0) -> np.ndarray:
        ny, nx = self.shape
        out = np.full((ny, nx) + a.shape[3:], fill, dtype=a.dtype)
        for t in range(1, self.ntiles):
            tj, ti = self.tiles[t]
            out[tj * TILE : (tj + 1) * TILE, ti * TILE : (ti + 1) * TILE] = a[t]
        return out


def exchange_map(grid: Grid) -> tuple[np.ndarray, np.ndarray]:
    """(dst, src) pairs filling every tile's halo from the owning tile (wadi2d/solver/state.py:14-48)."""
    nt = grid.ntiles
    if nt <= 1:
        return np.zeros(0, np.int32), np.zeros(0, np.int32)
    jj, ii = np.meshgrid(np.arange(STRIDE), np.arange(STRIDE), indexing="ij")
    own = (jj >= HALO) & (jj < HALO + TILE) & (ii >= HALO) & (ii < HALO + TILE)
    hj, hi = jj[~own], ii[~own]
    dj = np.where(hj < HALO, -1, np.where(hj >= HALO + TILE, 1, 0))
    di = np.where(hi < HALO, -1, np.where(hi >= HALO + TILE, 1, 0))
    sj, si = hj - dj * TILE, hi - di * TILE
    lookup = {d: n for n, d in enumerate(NEIGHBOURS)}
    nidx = np.array([lookup[(int(a), int(b))] for a, b in zip(dj, di, strict=True)])
    tiles = np.arange(1, nt)
    src_tile = grid.nbr[tiles][:, nidx]
    dst = tiles[:, None] * STRIDE2 + hj * STRIDE + hi
    src = src_tile * STRIDE2 + sj * STRIDE + si
    return dst.ravel().astype(np.int32), src.ravel().astype(np.int32)


def to_state(grid: Grid, a: np.ndarray) -> np.ndarray:
    """(ny, nx) grid into own cells and halos, halos read with clipped indices (wadi2d/solver/state.py:74-84)."""
    out = np.zeros(grid.ntiles * STRIDE2, np.float32)
    ny, nx = grid.shape
    for t in range(1, grid.ntiles):
        tj, ti = grid.tiles[t]
        r = np.clip(np.arange(STRIDE) - HALO + tj * TILE, 0, ny - 1)
        c = np.clip(np.arange(STRIDE) - HALO + ti * TILE, 0, nx - 1)
        out[t * STRIDE2 : (t + 1) * STRIDE2] = a[np.ix_(r, c)].ravel()
    return out


def tiles_to_state(grid: Grid, a: np.ndarray) -> np.ndarray:
    out = np.zeros(grid.ntiles * STRIDE2, np.float32)
    for t in range(1, grid.ntiles):
        out[t * STRIDE2 : (t + 1) * STRIDE2].reshape(STRIDE, STRIDE)[HALO : HALO + TILE, HALO : HALO + TILE] = a[t]
    return out


def static_cell_state(grid: Grid, a: np.ndarray) -> np.ndarray:
    """(ntiles, TILE, TILE) static array in state layout with its halos filled (wadi2d/solver/state.py:91-98)."""
    out = tiles_to_state(grid, np.asarray(a, np.float32))
    dst, src = exchange_map(grid)
    if dst.size:
        out[dst] = out[src]
    return out


def from_state(grid: Grid, a: np.ndarray) -> np.ndarray:
    ny, nx = grid.shape
    out = np.zeros((ny, nx), a.dtype)
    for t in range(1, grid.ntiles):
        tj, ti = grid.tiles[t]
        blk = a[t * STRIDE2 : (t + 1) * STRIDE2].reshape(STRIDE, STRIDE)[HALO : HALO + TILE, HALO : HALO + TILE]
        out[tj * TILE : (tj + 1) * TILE, ti * TILE : (ti + 1) * TILE] = blk
    return out


def state_index(grid: Grid, j, i):
    tile = grid.tile_of[np.asarray(j) // TILE, np.asarray(i) // TILE]
    return tile * STRIDE2 + (np.asarray(j) % TILE + HALO) * STRIDE + np.asarray(i) % TILE + HALO


def level_of(h, hc, dtab):
    """FP64 level above zmin from mean depth (wadi2d/solver/state.py:142-155)."""
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
    """FP64 wet share of the cell plan (wadi2d/solver/state.py:164-174)."""
    last = dtab.shape[-1] - 1
    out = np.ones(h.shape, np.float64)
    mid = (hc > 0.0) & (h < hc)
    s = np.sqrt(h[mid] / hc[mid]) * last
    r = np.minimum(s.astype(int), last - 1)
    idx = np.arange(r.size)
    t = dtab[mid]
    out[mid] = hc[mid] * (2 * r + 1) / last**2 / np.maximum(t[idx, r + 1] - t[idx, r], 1e-12)
    return out


def hbar_at_level(level, zmin, hc, dtab):
    """Mean depth giving this level through the table (wadi2d/tables/builder.py:311-331)."""
    last = dtab.shape[-1] - 1
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


# ---------------------------------------------------------------------------------------------------- tables


@dataclass
class Crest:
    """Faces edited by terrain objects, (ny, nx) grids, NaN = untouched (wadi2d/tables/builder.py:62-80)."""

    xz: np.ndarray
    xlen: np.ndarray
    xc: np.ndarray
    yz: np.ndarray
    ylen: np.ndarray
    yc: np.ndarray
    xwall: np.ndarray | None = None
    ywall: np.ndarray | None = None

    @classmethod
    def empty(cls, shape) -> Crest:
        nan, one, zero = np.full(shape, np.nan), np.ones(shape), np.zeros(shape)
        return cls(nan.copy(), one.copy(), zero.copy(), nan.copy(), one.copy(), zero.copy())


def read_bed(z: np.ndarray, row0: int, col0: int, nrows: int, ncols: int) -> np.ndarray:
    """A window of pixels with clipped indices (ArrayBed.read, wadi2d/tables/builder.py:47-50)."""
    r = np.clip(np.arange(row0, row0 + nrows), 0, z.shape[0] - 1)
    c = np.clip(np.arange(col0, col0 + ncols), 0, z.shape[1] - 1)
    return np.asarray(z[np.ix_(r, c)], dtype=np.float64)


def build_tables(
    grid: Grid,
    z: np.ndarray,
    pixel: float,
    manning=0.035,
    crest: Crest | None = None,
    rows: int = 16,
    face_depth_min: float = 8.0,
    face_depth_max: float = 16.0,
    local_radius: bool = True,
    beta: float = 9.0,
    crest_tolerance: float = 0.05,
    npix: np.ndarray | None = None,
) -> dict:
    """Every static array of the step (wadi2d/tables/builder.py:131-258, :290-308). ``npix`` is an optional
    per-pixel Manning grid aligned with ``z`` (NaN where the cell's own n holds)."""
    k = round(grid.dx / pixel)
    ny, nx = grid.shape
    crest = crest or Crest.empty((ny, nx))
    nman = np.full((ny, nx), float(manning)) if np.isscalar(manning) else np.asarray(manning, np.float64)
    nt = grid.ntiles
    zmin_g, rel_g, zfx_g, zfy_g = (np.zeros((ny, nx)) for _ in range(4))
    zcx_g, zcy_g = np.zeros((ny, nx)), np.zeros((ny, nx))
    hc = np.zeros((nt, TILE, TILE), np.float32)
    dtab = np.zeros((nt, TILE, TILE, rows), np.float32)
    efx = np.ones((nt, TILE, TILE), np.float32)
    efy = np.ones((nt, TILE, TILE), np.float32)
    ftabx = np.zeros((nt, TILE, TILE, rows, 2), np.float32)
    ftaby = np.zeros((nt, TILE, TILE, rows, 2), np.float32)
    margin = min(int(np.ceil(beta * face_depth_max / pixel)), int(max(z.shape))) if local_radius else 0
    W = TILE * k + 1
    L = lib()
    for t in range(1, nt):
        tj, ti = grid.tiles[t]
        j0, i0 = int(tj) * TILE, int(ti) * TILE
        zbig = np.ascontiguousarray(read_bed(z, j0 * k - 1 - margin, i0 * k - 1 - margin, W + 2 * margin, W + 2 * margin))
        lin = None
        if npix is not None:
            lin = np.ascontiguousarray(read_bed(npix, j0 * k - 1, i0 * k - 1, W, W))
        sl = (slice(j0, j0 + TILE), slice(i0, i0 + TILE))
        cell_in = [np.ascontiguousarray(a[sl], np.float64) for a in (nman, crest.xz, crest.xlen, crest.yz, crest.ylen)]
        w = {n: np.zeros((TILE, TILE)) for n in ("zmin", "rel", "hc", "zfx", "efx", "zfy", "efy")}
        w_dtab = np.zeros((TILE, TILE, rows))
        w_ftabx = np.zeros((TILE, TILE, rows, 2))
        w_ftaby = np.zeros((TILE, TILE, rows, 2))
        L.or_tile_tables(
            _p(zbig, _F64P), margin, k, float(pixel), *(_p(a, _F64P) for a in cell_in[:1]), _p(lin, _F64P),
            *(_p(a, _F64P) for a in cell_in[1:]), float(face_depth_min), float(face_depth_max), rows,
            int(local_radius), float(beta), _p(w["zmin"], _F64P), _p(w["rel"], _F64P), _p(w["hc"], _F64P),
            _p(w_dtab, _F64P), _p(w["zfx"], _F64P), _p(w["efx"], _F64P), _p(w_ftabx, _F64P), _p(w["zfy"], _F64P),
            _p(w["efy"], _F64P), _p(w_ftaby, _F64P),
        )  # fmt: skip
        zmin_g[sl], rel_g[sl], zfx_g[sl], zfy_g[sl] = w["zmin"], w["rel"], w["zfx"], w["zfy"]
        core = zbig[margin : margin + W, margin : margin + W]
        cx, cy = centre_beds(core, k)
        zcx_g[sl], zcy_g[sl] = cx - w["zmin"], cy - w["zmin"]
        hc[t], dtab[t], efx[t], efy[t], ftabx[t], ftaby[t] = w["hc"], w_dtab, w["efx"], w["efy"], w_ftabx, w_ftaby
    zbar_g = zmin_g + rel_g
    active = grid.mask
    zcx_g, zcy_g = (np.nan_to_num(np.maximum(a, 0.0), nan=0.0, posinf=0.0, neginf=0.0) for a in (zcx_g, zcy_g))
    fx = _faces(zfx_g, zmin_g, zbar_g, active, 1, crest.xc, crest_tolerance, crest.xwall)
    fy = _faces(zfy_g, zmin_g, zbar_g, active, 0, crest.yc, crest_tolerance, crest.ywall)
    out = dict(zmin=zmin_g, zbar=zbar_g, hc=hc, dtab=dtab, efx=efx, efy=efy, ftabx=ftabx, ftaby=ftaby)
    for name, a in zip(("flx", "frx", "glx", "grx", "cwx"), fx, strict=True):
        out[name] = grid.to_tiles(a)
    for name, a in zip(("fly", "fry", "gly", "gry", "cwy"), fy, strict=True):
        out[name] = grid.to_tiles(a)
    out["zcx"] = grid.to_tiles(zcx_g).astype(np.float32)
    out["zcy"] = grid.to_tiles(zcy_g).astype(np.float32)
    out["rows"] = rows
    return out


def centre_beds(z: np.ndarray, k: int):
    """Bed on each cell's centre lines (wadi2d/tables/core.py:267-279)."""
    c = np.asarray(z, np.float64)[1 : 1 + TILE * k, 1 : 1 + TILE * k].reshape(TILE, k, TILE, k)
    columns = c.min(axis=1)
    rows = c.min(axis=3)
    if k % 2:
        return columns[:, :, k // 2], rows[:, k // 2, :]
    return 0.5 * (columns[:, :, k // 2 - 1] + columns[:, :, k // 2]), 0.5 * (rows[:, k // 2 - 1, :] + rows[:, k // 2, :])


def _faces(zf, zmin, zbar, active, axis, crest_c, tol, wall=None):
    """Inverts, closed faces and natural crests (wadi2d/tables/builder.py:290-308)."""
    zmin_n = np.roll(zmin, 1, axis=axis)
    zbar_n = np.roll(zbar, 1, axis=axis)
    act_n = np.roll(active, 1, axis=axis)
    open_face = active & act_n
    if wall is not None:
        open_face = open_face & ~wall
    fl = np.where(open_face, zf - zmin_n, CLOSED)
    fr = np.where(open_face, zf - zmin, CLOSED)
    gl = np.where(open_face, zf - zbar_n, 0.0)
    gr = np.where(open_face, zf - zbar, 0.0)
    natural = open_face & (gl > tol) & (gr > tol)
    cw = np.where(crest_c != 0.0, crest_c, np.where(natural, CRITICAL_WEIR_COEFF, 0.0))
    cw = np.where(open_face, cw, 0.0)
    return fl, fr, gl, gr, cw


# ---------------------------------------------------------------------------------------------------- backend


@dataclass
class Numerics:
    """The fields of the reference's ``Numerics`` the uniform step reads (wadi2d/config/schema.py:457-519)."""

    cfl: float = 0.45
    second: bool = True
    sheet_flow: bool = True
    mirror_dry_faces: bool = True
    face_depth_carry: bool = True
    e_wet: float = 1e-4
    h_cfl: float = 0.01
    u_max: float = 25.0
    dt_max: float = 5.0
    dt_min: float = 1e-3
    dt_every: int = 8
    wave_floor: float = 3.0
    plan_min: float = 0.02
    active_every: int = 16


@dataclass
class Boundary:
    cell: np.ndarray
    ref: np.ndarray
    kind: np.ndarray
    d0: np.ndarray
    h0: np.ndarray

    @classmethod
    def empty(cls) -> Boundary:
        i = np.zeros(0, np.int32)
        f = np.zeros(0, np.float32)
        return cls(i, i.copy(), i.copy(), f, f.copy())


class NumericalFailure(RuntimeError):
    pass


class Backend:
    """The reference CPU backend's arrays and step (wadi2d/solver/cpu/backend.py:14-141)."""

    def __init__(self, grid: Grid, tables: dict, num: Numerics) -> None:
        self.grid, self.num, self.rows = grid, num, int(tables["rows"])
        n = grid.ntiles * STRIDE2
        for a in "h d u v mx my qx qy u1 v1 mx1 my1 qx1 qy1 r src res om".split():
            setattr(self, a, np.zeros(n, np.float32))
        c32 = lambda a: np.ascontiguousarray(a, np.float32).ravel()  # noqa: E731
        self.Hc, self.dtab = c32(tables["hc"]), c32(tables["dtab"])
        for ax in "xy":
            for f in ("fl", "fr", "gl", "gr", "ef", "cw", "ftab"):
                setattr(self, f + ax, c32(tables[f + ax]))
        self.zcx = static_cell_state(grid, tables["zcx"])
        self.zcy = static_cell_state(grid, tables["zcy"])
        self.wave = np.zeros(grid.ntiles, np.float32)
        self.wet = np.zeros(grid.ntiles, np.int32)
        dst, src = exchange_map(grid)
        self.nhalo = dst.size // max(grid.ntiles - 1, 1)
        self.slot = (dst[: self.nhalo] - STRIDE2).astype(np.int32)
        self.src_map = src
        self.bc = Boundary.empty()
        self.params = OrParams(
            G, grid.dx, num.e_wet, num.h_cfl, num.u_max, float(num.dt_every), num.plan_min, self.rows, int(num.second),
            int(num.sheet_flow), int(num.mirror_dry_faces), int(num.face_depth_carry),
        )  # fmt: skip
        self.set_active(np.arange(1, grid.ntiles, dtype=np.int32))

    def _arrays(self) -> OrArrays:
        a = OrArrays()
        for n in _ARRAY_FIELDS:
            setattr(a, n, _p(getattr(self, n)))
        a.wet = _p(self.wet, _I32P)
        return a

    def set_active(self, active: np.ndarray) -> None:
        self.active = np.ascontiguousarray(active, np.int32)
        self.active_tiles = self.active
        self.nact = int(active.size)

    def set_field(self, name: str, a: np.ndarray) -> None:
        getattr(self, name)[:] = a

    def get_field(self, name: str) -> np.ndarray:
        return getattr(self, name).copy()

    def set_boundary(self, bc: Boundary) -> None:
        self.bc = bc

    def _exch(self, *arrays) -> None:
        L = lib()
        for a in arrays:
            L.or_exchange(_p(self.active, _I32P), self.nact, _p(self.slot, _I32P), _p(self.src_map, _I32P), self.nhalo, _p(a))

    def refresh_plan(self, tiles: np.ndarray) -> None:
        if tiles.size:
            t = np.ascontiguousarray(tiles, np.int32)
            lib().or_plan(ctypes.byref(self._arrays()), ctypes.byref(self.params), _p(t, _I32P), int(t.size))

    def refresh_halos(self) -> None:
        if self.nact:
            self._exch(self.h, self.d, self.qx, self.qy, self.u, self.v, self.om)

    def step(self, dt: float, want_wave: bool, want_wet: bool) -> None:
        if want_wave:
            self.wave[:] = 0.0
        if self.nact == 0:
            return
        L = lib()
        dtf = float(np.float32(dt))
        arr, par, act = ctypes.byref(self._arrays()), ctypes.byref(self.params), _p(self.active, _I32P)
        L.or_faces(arr, par, act, self.nact, dtf, int(want_wave))
        self._exch(self.u1, self.v1, self.qx1, self.qy1)
        L.or_limit(arr, par, act, self.nact, dtf)
        self._exch(self.r)
        L.or_update(arr, par, act, self.nact, dtf, int(want_wave))
        if self.bc.cell.size:
            b = self.bc
            L.or_boundary(
                int(b.cell.size), _p(b.cell, _I32P), _p(b.ref, _I32P), _p(b.kind, _I32P), _p(b.d0), _p(b.h0),
                _p(self.h), _p(self.d),
            )  # fmt: skip
        self._exch(self.h, self.d, self.qx, self.qy)
        if want_wave:
            self._exch(self.om)
        self.u, self.u1 = self.u1, self.u
        self.v, self.v1 = self.v1, self.v
        self.mx, self.mx1 = self.mx1, self.mx
        self.my, self.my1 = self.my1, self.my

    def max_wave(self) -> float:
        return float(self.wave.max())

    def wet_flags(self) -> np.ndarray:
        return self.wet.copy()


class Model:
    """Tables + backend + the stepper's time loop (wadi2d/solver/model.py:32-188, wadi2d/solver/stepper.py:24-129)."""

    def __init__(self, grid: Grid, tables: dict, num: Numerics | None = None) -> None:
        self.grid, self.tables = grid, tables
        self.num = num or Numerics()
        self.backend = Backend(grid, tables, self.num)
        self.boundary_tiles = np.zeros(0, np.int64)
        self.t = 0.0
        self.nsteps = 0
        self.adaptive_active = True
        self.keep_active = np.zeros(grid.ntiles, bool)
        self.refresh_due = True
        self.dt = self.num.cfl * grid.dx / self.num.wave_floor
        self.idle = np.zeros(grid.ntiles, np.int32)
        self.dts: list[float] = []
        self.kick = None  # a momentum source on faces, applied before every step (wadi2d/solver/stepper.py:111-112)

    @property
    def stepper(self) -> Model:
        """The reference keeps t, dt and nsteps on ``Model.stepper``; here the model is its own stepper."""
        return self

    # host-side setters, wadi2d/solver/model.py:43-150
    def set_depth(self, hbar: np.ndarray) -> None:
        g = self.grid
        h = np.where(g.mask, hbar, 0.0)
        hc, dtab = g.from_tiles(self.tables["hc"]), g.from_tiles(self.tables["dtab"])
        self.backend.set_field("h", to_state(g, h))
        self.backend.set_field("d", to_state(g, level_of(h, hc, dtab)))
        self.backend.set_field("om", to_state(g, plan_of(h, hc, dtab)))
        self.backend.wet[:] = self._tile_wet(h)
        self.rebuild_active()

    def _tile_wet(self, h: np.ndarray) -> np.ndarray:
        out = np.zeros(self.grid.ntiles, np.int32)
        for t in range(1, self.grid.ntiles):
            tj, ti = self.grid.tiles[t]
            out[t] = int(np.any(h[tj * TILE : (tj + 1) * TILE, ti * TILE : (ti + 1) * TILE] > 0.0))
        return out

    def set_velocity(self, ucell: np.ndarray, vcell: np.ndarray) -> None:
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
        g = self.grid
        self.backend.set_field("src", to_state(g, np.where(g.mask, rate, 0.0)))
        self.keep_active[:] = False
        for t in range(1, g.ntiles):
            tj, ti = g.tiles[t]
            self.keep_active[t] = bool(np.any(rate[tj * TILE : (tj + 1) * TILE, ti * TILE : (ti + 1) * TILE] != 0.0))
        self.keep_active[self.boundary_tiles] = True
        self.rebuild_active(retain=True)
        self.refresh_due = True

    def set_source_cells(self, cells: np.ndarray, rate: np.ndarray) -> None:
        src = np.zeros(self.grid.ntiles * STRIDE2, np.float32)
        src[cells] = rate
        self.backend.set_field("src", src)
        self.keep_active[:] = False
        self.keep_active[cells[rate != 0.0] // STRIDE2] = True
        self.keep_active[self.boundary_tiles] = True
        self.rebuild_active(retain=True)
        self.refresh_due = True

    def set_boundary(self, bc: Boundary) -> None:
        self.backend.set_boundary(bc)
        self.boundary_tiles = np.unique(bc.cell // STRIDE2)
        self.keep_active[self.boundary_tiles] = True
        self.rebuild_active(retain=True)

    def set_momentum(self, kick) -> None:
        """A momentum source on faces for the steps until the next call (wadi2d/solver/model.py:128-132)."""
        self.kick = kick

    def cell_state_index(self, j: int, i: int) -> int:
        return int(state_index(self.grid, j, i))

    def field(self, name: str) -> np.ndarray:
        return from_state(self.grid, self.backend.get_field(name))

    def volume(self) -> float:
        return float(self.field("h").sum(dtype=np.float64) * self.grid.dx**2)

    # stepper, wadi2d/solver/stepper.py:56-129
    def rebuild_active(self, retain: bool = False, check: bool = False) -> None:
        g, b = self.grid, self.backend
        nt = g.ntiles
        if not self.adaptive_active:
            if int(b.nact) != nt - 1:
                b.set_active(np.arange(1, nt, dtype=np.int32))
            return
        wet = b.wet_flags().astype(bool) | self.keep_active
        wet[0] = False
        act = wet.copy()
        act[g.nbr[wet].ravel()] = True
        current = np.zeros(nt, bool)
        current[b.active_tiles] = True
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
        b.set_active(np.nonzero(act)[0].astype(np.int32))
        if (retain or check) and woken.any():
            b.refresh_plan(np.nonzero(woken)[0].astype(np.int32))
            b.refresh_halos()

    def advance(self, t_end: float, on_step=None) -> float:
        b, num, dx = self.backend, self.num, self.grid.dx
        while self.t < t_end - 1e-9:
            refresh = self.refresh_due or self.nsteps % num.dt_every == 0
            self.refresh_due = False
            activate = self.nsteps % num.active_every == 0
            dt = min(self.dt, t_end - self.t, num.dt_max)
            if self.kick is not None:
                self.kick.apply(b, dt)
            b.step(dt, refresh, activate)
            self.dts.append(dt)
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


class Maxima:
    """Envelope arrays in state layout (wadi2d/engine/maxima.py:103-146), CPU form."""

    NAMES = ("depth", "mean_depth", "speed", "hazard", "arrival")

    def __init__(self, model: Model, arrival_depth: float = 0.1, speed_depth: float = 0.05) -> None:
        self.model = model
        self.arrive, self.deep = float(arrival_depth), float(speed_depth)
        n = model.grid.ntiles * STRIDE2
        self.arrays = [np.zeros(n, np.float32) for _ in self.NAMES]
        self.arrays[-1][:] = -1.0

    def update(self, t: float) -> None:
        b = self.model.backend
        lib().or_maxima(
            _p(b.active, _I32P), b.nact, float(np.float32(t)), float(np.float32(self.arrive)),
            float(np.float32(self.deep)), _p(b.d), _p(b.h), _p(b.u), _p(b.v), *(_p(a) for a in self.arrays),
        )  # fmt: skip

    def raw(self) -> dict[str, np.ndarray]:
        return {n: a.copy() for n, a in zip(self.NAMES, self.arrays, strict=True)}

    def fields(self) -> dict[str, np.ndarray]:
        return {n: from_state(self.model.grid, a) for n, a in zip(self.NAMES, self.arrays, strict=True)}


class Tally:
    """FP64 volume through a set of faces, one total per face (wadi2d/engine/maxima.py:149-192, device form)."""

    def __init__(self, model: Model, xfaces, xsign, yfaces, ysign) -> None:
        self.model = model
        self.face = np.concatenate((xfaces, yfaces)).astype(np.int32)
        self.axis = np.concatenate((np.zeros(len(xfaces)), np.ones(len(yfaces)))).astype(np.int32)
        self.sign = np.concatenate((xsign, ysign)).astype(np.float32)
        self.total = np.zeros(self.face.size, np.float64)

    def add(self, dt: float) -> None:
        b = self.model.backend
        lib().or_tally(
            int(self.face.size), float(dt), _p(self.face, _I32P), _p(self.axis, _I32P), _p(self.sign), _p(b.qx),
            _p(b.qy), _p(self.total, _F64P),
        )  # fmt: skip

    def volume(self) -> float:
        return float(self.total.sum())
