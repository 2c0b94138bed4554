"""``build_tables`` on the GPU (w2b_build_tables): the reference's table build (wadi2d/tables/builder.py:131-258)
from an in-memory bed, with the same inputs (bed, Tables settings, Manning n as one value or a grid, CrestFaces,
per-pixel lining). The tables stay on the device; host copies are made the first time a field is read."""

from __future__ import annotations

import ctypes

import numpy as np

from wadi2d_b200 import _lib
from wadi2d_b200.config import Tables
from wadi2d_b200.grid import TileGrid

TILE_FIELDS = ("hc", "dtab", "efx", "efy", "ftabx", "ftaby", "zcx", "zcy", "flx", "frx", "glx", "grx", "cwx", "fly",
               "fry", "gly", "gry", "cwy")  # fmt: skip
GRID_FIELDS = ("zmin", "zbar")
WS_BYTES_MAX = 2 << 30


class TableIn(ctypes.Structure):
    _fields_ = (
        [("z", ctypes.c_void_p), ("zh", ctypes.c_int64), ("zw", ctypes.c_int64), ("row_offset", ctypes.c_int32),
         ("col_offset", ctypes.c_int32), ("npix", ctypes.c_void_p), ("nman", ctypes.c_void_p)]
        + [(n, ctypes.c_void_p) for n in ("xcrest", "xlen", "xc", "ycrest", "ylen", "yc", "xwall", "ywall", "mask",
                                          "tiles")]
        + [(n, ctypes.c_int32) for n in ("ntiles", "ny", "nx", "k", "rows", "local", "margin")]
        + [(n, ctypes.c_double) for n in ("pixel", "face_depth_min", "face_depth_max", "beta", "crest_tolerance")]
    )  # fmt: skip


class TableOut(ctypes.Structure):
    _fields_ = [(n, ctypes.c_void_p) for n in TILE_FIELDS + ("zmin", "rel", "zfx", "zfy", "ws")] + [
        ("ws_threads", ctypes.c_int64)
    ]


_L = _lib.lib()
_L.w2b_build_tables.argtypes = [ctypes.POINTER(TableIn), ctypes.POINTER(TableOut), ctypes.c_void_p]
_L.w2b_build_tables.restype = ctypes.c_int32


class DeviceGridTables:
    """GridTables whose arrays live on the device (``device_arrays``). Reading a field by name (``tables.hc``) gives
    a host numpy copy, made once; the B200 backend binds the device arrays without a copy."""

    def __init__(self, grid: TileGrid, rows: int, arrays: dict) -> None:
        self.grid = grid
        self._rows = rows
        self.device_arrays = arrays
        self._host: dict[str, np.ndarray] = {}

    @property
    def rows(self) -> int:
        return self._rows

    def __getattr__(self, name: str):
        if name.startswith("_") or name not in self.__dict__.get("device_arrays", {}):
            raise AttributeError(name)
        if name not in self._host:
            self._host[name] = self.device_arrays[name].cpu().numpy()
        return self._host[name]


def tile_margin(cfg: Tables, pixel: float, span: int) -> int:
    """Pixels a face's line reaches past its ends for the local radius (wadi2d/tables/builder.py:261-269)."""
    if cfg.face_conveyance != "local_radius":
        return 0
    return min(int(np.ceil(cfg.local_radius_beta * cfg.face_depth_max / pixel)), int(span))


def build_tables_gpu(grid: TileGrid, bed, cfg=None, manning=0.035, crest=None, lining=None, device=None,
                     npix=None) -> DeviceGridTables:  # fmt: skip
    import torch

    if not torch.cuda.is_available():
        raise RuntimeError("build_tables runs on the GPU; no CUDA device is available")
    cfg = cfg or Tables()
    dev = torch.device(device if device is not None else "cuda")
    pixel = float(bed.pixel)
    k = round(grid.dx / pixel)
    if abs(k * pixel - grid.dx) > 1e-6 * grid.dx:
        raise ValueError(f"cell size {grid.dx} is not a multiple of the pixel {pixel}")
    ny, nx = grid.shape
    nt, rows = grid.ntiles, int(cfg.rows)
    if isinstance(bed.z, torch.Tensor):
        zt = bed.z.to(device=dev, dtype=torch.float64).contiguous()
        zshape = tuple(zt.shape)
    else:
        z = np.asarray(bed.z, np.float64)
        zshape = z.shape
    if lining is not None and npix is None:
        npix = np.full(zshape, np.nan)
        lining(np.asarray(bed.z.cpu() if isinstance(bed.z, torch.Tensor) else z), npix, 0, 0)

    def d64(a):
        return torch.as_tensor(np.ascontiguousarray(a, np.float64), device=dev)

    def u8(a):
        return torch.as_tensor(np.ascontiguousarray(a, np.uint8), device=dev)

    if not isinstance(bed.z, torch.Tensor):
        zt = d64(z)
    npt = d64(npix) if npix is not None else None
    nman = d64(np.full((ny, nx), float(manning)) if np.isscalar(manning) else manning)
    if crest is None:
        nan = np.full((ny, nx), np.nan)
        cr = dict(xcrest=nan, xlen=np.ones((ny, nx)), xc=np.zeros((ny, nx)), ycrest=nan, ylen=np.ones((ny, nx)),
                  yc=np.zeros((ny, nx)))  # fmt: skip
        walls = (None, None)
    else:
        cr = dict(xcrest=crest.xz, xlen=crest.xlen, xc=crest.xc, ycrest=crest.yz, ylen=crest.ylen, yc=crest.yc)
        walls = (crest.xwall, crest.ywall)
    crt = {n: d64(a) for n, a in cr.items()}
    wt = [u8(w) if w is not None else None for w in walls]
    mask = u8(grid.mask)
    tiles = torch.as_tensor(np.ascontiguousarray(grid.tiles, np.int32), device=dev)

    out = {}
    for n in TILE_FIELDS:
        shape = {"dtab": (nt, 32, 32, rows), "ftabx": (nt, 32, 32, rows, 2), "ftaby": (nt, 32, 32, rows, 2)}.get(
            n, (nt, 32, 32)
        )
        out[n] = torch.full(shape, 1.0 if n in ("efx", "efy") else 0.0, dtype=torch.float32, device=dev)
    dense = {n: torch.zeros((ny, nx), dtype=torch.float64, device=dev) for n in ("zmin", "rel", "zfx", "zfy")}
    local = cfg.face_conveyance == "local_radius"
    margin = tile_margin(cfg, pixel, max(zshape))
    nmax = k + 2 * margin
    threads = 148 * 8 * 128
    per_thread = int(_L.w2b_table_workspace_doubles(nmax, 1)) * 8
    threads = max(128, min(threads, (WS_BYTES_MAX // per_thread) // 128 * 128))
    ws = torch.empty(int(_L.w2b_table_workspace_doubles(nmax, threads)) if local else 1, dtype=torch.float64,
                     device=dev)  # fmt: skip

    def ptr(t):
        return None if t is None else t.data_ptr()

    tin = TableIn(
        zt.data_ptr(), zshape[0], zshape[1], int(getattr(bed, "row_offset", 0)), int(getattr(bed, "col_offset", 0)),
        ptr(npt), nman.data_ptr(), *(crt[n].data_ptr() for n in ("xcrest", "xlen", "xc", "ycrest", "ylen", "yc")),
        ptr(wt[0]), ptr(wt[1]), mask.data_ptr(), tiles.data_ptr(), nt, ny, nx, k, rows, int(local), margin, pixel,
        float(cfg.face_depth_min), float(cfg.face_depth_max), float(cfg.local_radius_beta), float(cfg.crest_tolerance),
    )  # fmt: skip
    tout = TableOut(*(out[n].data_ptr() for n in TILE_FIELDS), *(dense[n].data_ptr() for n in ("zmin", "rel", "zfx", "zfy")),
                    ws.data_ptr(), threads if local else 0)  # fmt: skip
    stream = torch.cuda.current_stream(dev).cuda_stream
    status = int(_L.w2b_build_tables(ctypes.byref(tin), ctypes.byref(tout), stream))
    if status != _lib.OK:
        raise _lib.W2BError(status, "w2b_build_tables")
    torch.cuda.current_stream(dev).synchronize()
    del ws, zt, npt
    out["zmin"] = dense["zmin"]
    out["zbar"] = dense["zmin"] + dense["rel"]
    return DeviceGridTables(grid, rows, out)
