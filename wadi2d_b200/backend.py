"""The compute interface the reference's Model and Stepper drive (wadi2d/solver/backend.py:15-75), and
``B200Backend``: the duck-typed twin of CpuBackend / GpuBackend (wadi2d/solver/cpu/backend.py:14-141,
wadi2d/solver/gpu/backend.py:53-203) whose step runs in libwadi_b200 on a B200, with PyTorch tensors as its device
buffers.

State attributes (``h``, ``u``, ``mx``, ``qx`` ...) are ``Field`` adapters: indexed with reference state indices
(tile-with-halo layout) they read and write the device arrays, so ``Model.read_cells``, ``FaceKick.apply``
(``backend.mx[faces] += ...``) and tests that poke faces between steps work unchanged. There is no ``cp`` attribute:
callers that look for CuPy take their host path, and this package's own Maxima and Tally run on the device.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from wadi2d_b200 import _lib
from wadi2d_b200.config import G, Numerics
from wadi2d_b200.layout import STRIDE2, TILE, TILE2, native_of_ref
from wadi2d_b200.tables import GridTables


@dataclass(frozen=True)
class NumericsRecord:
    """The run-time numbers kernels read (wadi2d/solver/backend.py:15-39)."""

    g: float
    dx: float
    e_wet: float
    h_cfl: float
    u_max: float
    lead: float
    a_min: float
    second: bool
    sheet: bool
    mirror: bool
    carry: bool = True
    level_fp64: bool = False
    arith: str = "exact"

    @classmethod
    def from_config(cls, num: Numerics, dx: float) -> NumericsRecord:
        lead = float(max(num.dt_every, 1 << num.lts_levels) if num.local_time_stepping else num.dt_every)
        return cls(
            G, dx, num.e_wet, num.h_cfl, num.u_max, lead, num.plan_min, num.limiter != "none", num.sheet_flow,
            num.mirror_dry_faces, num.face_depth_carry, bool(getattr(num, "level_fp64", False)),
            str(getattr(num, "arithmetic", "exact")),
        )  # fmt: skip


@dataclass
class BoundaryCells:
    """Cells whose level is prescribed after every update. kind: 0 fixed, 1 free, 2 follows ``ref`` plus d0."""

    cell: np.ndarray
    ref: np.ndarray
    kind: np.ndarray
    d0: np.ndarray
    h0: np.ndarray

    @classmethod
    def empty(cls) -> BoundaryCells:
        i = np.zeros(0, np.int32)
        f = np.zeros(0, np.float32)
        return cls(i, i.copy(), i.copy(), f, f.copy())


def select_backend(name: str, tables: GridTables, num: NumericsRecord):
    """``b200``, ``gpu`` and ``auto`` give the B200 backend; there is no CPU backend in this package."""
    if name not in ("auto", "gpu", "b200"):
        raise ValueError(f"backend {name!r}: this package has only the B200 backend")
    return B200Backend(tables, num)


class Field:
    """A state array seen through reference state indices (tile-with-halo layout)."""

    def __init__(self, backend: B200Backend, name: str) -> None:
        self.b, self.name = backend, name

    def _tensor(self):
        return self.b.native(self.name)

    def _index(self, idx):
        if isinstance(idx, slice) or idx is Ellipsis:
            raise TypeError("index a state field with reference state indices, or use get_field/set_field")
        return self.b.torch.as_tensor(native_of_ref(self.b.grid.tiles, idx, self.b.grid.shape[1]), device=self.b.device)

    def __getitem__(self, idx) -> np.ndarray:
        return self._tensor()[self._index(idx)].cpu().numpy()

    def __setitem__(self, idx, value) -> None:
        t = self._tensor()
        t[self._index(idx)] = self.b.torch.as_tensor(np.asarray(value, np.float32), device=self.b.device)

    def __array__(self, dtype=None, copy=None):
        a = self.b.get_field(self.name)
        return a if dtype is None else a.astype(dtype)

    def copy(self) -> np.ndarray:
        return self.b.get_field(self.name)

    @property
    def size(self) -> int:
        return self.b.grid.ntiles * STRIDE2


class TileFlags:
    """The per-tile wet flags: a device array that accepts ``wet[:] = host_flags`` (wadi2d/solver/model.py:52)."""

    def __init__(self, backend: B200Backend) -> None:
        self.b = backend

    def __setitem__(self, idx, value) -> None:
        self.b._t["wet"][idx] = self.b.torch.as_tensor(np.asarray(value, np.int32), device=self.b.device)

    def __getitem__(self, idx):
        return self.b._t["wet"].cpu().numpy()[idx]

    def __array__(self, dtype=None, copy=None):
        a = self.b._t["wet"].cpu().numpy()
        return a if dtype is None else a.astype(dtype)


STATE = ("h", "d", "u", "v", "mx", "my", "qx", "qy", "u1", "v1", "mx1", "my1", "qx1", "qy1", "src", "res", "om",
         "zcx", "zcy")  # fmt: skip
ENVELOPE = ("depth", "mean_depth", "speed", "hazard", "arrival")
MOMENTUM_FIELDS = ("u", "v", "mx", "my", "u1", "v1", "mx1", "my1")  # read or written only with the momenta in place


class B200Backend:
    """Owns the device buffers (PyTorch CUDA tensors) and a libwadi_b200 handle bound to them."""

    name = "b200"

    def __init__(self, tables: GridTables, num: NumericsRecord, device=None, tile_run=None, nruns: int = 1,
                 grid=None, table_tile=None) -> None:  # fmt: skip
        """``grid`` (default ``tables.grid``) is the grid stepped; with ``table_tile`` (one entry a tile of it) the
        tables hold only distinct tiles and tile t reads table tile ``table_tile[t]`` (a batch's runs on one catchment
        sharing one copy)."""
        import torch

        self.torch = torch
        if not torch.cuda.is_available():
            raise RuntimeError("B200Backend needs a CUDA device; this package has no CPU fallback")
        self.device = torch.device(device if device is not None else "cuda")
        self.grid = tables.grid if grid is None else grid
        self.num = num
        self.rows = tables.rows
        g = self.grid
        ny, nx = g.shape
        nt = g.ntiles
        rows = self.rows
        self.nruns = int(nruns)
        self._desc = _lib.GridDesc(ny, nx, nt, rows, self.nruns)
        lay = _lib.Layout()
        _lib.call("w2b_layout", ctypes.byref(self._desc), ctypes.byref(lay))
        self.px, self.ncells = int(lay.px), int(lay.ncells)
        dev = self.device

        def f32(n, fill=0.0):
            return torch.full((int(n),), fill, dtype=torch.float32, device=dev)

        def i32(n):
            return torch.zeros(int(n), dtype=torch.int32, device=dev)

        def up(a, dtype=torch.float32):
            if isinstance(a, torch.Tensor):
                return a.reshape(-1).to(device=dev, dtype=dtype).contiguous()
            return torch.as_tensor(np.ascontiguousarray(a).reshape(-1), device=dev).to(dtype).contiguous()

        on_device = getattr(tables, "device_arrays", None) or {}

        def tab(name):
            """A table array: the builder's device tensor when there is one, else an upload of the host array."""
            return up(on_device[name] if name in on_device else getattr(tables, name))

        t = {}
        for n in ("h", "u", "v", "mx", "my"):
            t[n] = f32(2 * self.ncells).view(2, self.ncells)
        for n in ("d", "qx", "qy", "qx1", "qy1", "res", "src", "om", "zcx", "zcy"):
            t[n] = f32(self.ncells)
        t["hc"] = tab("hc")
        for ax in "xy":
            for f in ("fl", "fr", "gl", "gr", "ef", "cw"):
                t[f + ax] = tab(f + ax)
        ntab = t["hc"].numel() // TILE2  # tiles of the static arrays: nt, or the distinct tiles under table_tile
        if table_tile is None and ntab != nt:
            raise ValueError(f"tables of {ntab} tiles for a grid of {nt}")
        t["dtab2"] = f32(ntab * (rows - 1) * TILE2 * 2)
        t["ftab4x"] = f32(ntab * (rows - 1) * TILE2 * 4)
        t["ftab4y"] = f32(ntab * (rows - 1) * TILE2 * 4)
        t["tiles"] = up(g.tiles, torch.int32)
        t["tile_of"] = up(g.tile_of, torch.int32)
        t["nbr"] = up(g.nbr, torch.int32)
        for n in ("active", "wet", "keep", "idle", "is_act", "woken", "work"):
            t[n] = i32(nt)
        t["wave"] = f32(nt)
        t["scratch"] = i32(2 * nt)
        t["bmark"] = i32(nt * TILE)
        t["env"] = [f32(nt * TILE2, -1.0 if n == "arrival" else 0.0) for n in ENVELOPE]
        t["ctl"] = torch.zeros(_lib.CTL_BYTES // 8, dtype=torch.int64, device=dev)
        nbytes = int(_lib.lib().w2b_run_table_bytes(self.nruns))
        t["runs"] = torch.zeros((nbytes + 7) // 8, dtype=torch.int64, device=dev)
        t["tile_run"] = (torch.zeros(nt, dtype=torch.int32, device=dev) if tile_run is None
                         else torch.as_tensor(np.ascontiguousarray(tile_run, np.int32), device=dev))  # fmt: skip
        t["stage"] = f32(nt * STRIDE2)
        t["lpair"] = f32(nt * TILE2 * 2)  # the update pass's level cache (w2b_create marks it empty)
        t["lrow"] = torch.full((nt * TILE2,), 255, dtype=torch.uint8, device=dev)
        if table_tile is not None:
            tt = np.ascontiguousarray(table_tile, np.int32)
            if tt.shape != (nt,) or tt.min() < 0 or tt.max() >= ntab or tt[0] != 0:
                raise ValueError("table_tile: one entry a tile, in [0, table tiles), the void tile on tile 0")
            t["table_tile"] = torch.as_tensor(tt, device=dev)
        self._t = t
        # own cells of every allocated tile, NATIVE index in tile-layout order (fid = t * 1024 + j * 32 + i)
        jj, ii = np.divmod(np.arange(TILE2), TILE)
        j = g.tiles[1:, 0, None].astype(np.int64) * TILE + jj[None, :]
        i = g.tiles[1:, 1, None].astype(np.int64) * TILE + ii[None, :]
        self._own = torch.as_tensor(((j + 4) * self.px + i + 32).reshape(-1), device=dev)
        for zc in ("zcx", "zcy"):
            z = tab(zc)
            if table_tile is not None:
                z = z.view(ntab, TILE2)[t["table_tile"][1:].long()].reshape(-1)
            else:
                z = z[TILE2:]
            t[zc][self._own] = z
        dtab, fx, fy = tab("dtab"), tab("ftabx"), tab("ftaby")
        stream = self._stream()
        tab_desc = _lib.GridDesc(ny, nx, ntab, rows, self.nruns)
        _lib.call("w2b_pack_tables", ctypes.byref(tab_desc), dtab.data_ptr(), fx.data_ptr(), fy.data_ptr(),
                  t["dtab2"].data_ptr(), t["ftab4x"].data_ptr(), t["ftab4y"].data_ptr(), stream)  # fmt: skip
        torch.cuda.current_stream(dev).synchronize()
        del dtab, fx, fy

        B = _lib.Buffers()
        for n in ("h", "u", "v", "mx", "my"):
            getattr(B, n)[0] = t[n][0].data_ptr()
            getattr(B, n)[1] = t[n][1].data_ptr()
        for n in ("d", "qx", "qy", "qx1", "qy1", "res", "src", "om", "zcx", "zcy", "hc", "dtab2", "tiles", "tile_of",
                  "nbr", "active", "wave", "wet", "keep", "idle", "is_act", "woken", "work", "scratch", "bmark", "ctl",
                  "runs", "tile_run", "stage", "lpair", "lrow"):  # fmt: skip
            setattr(B, n, t[n].data_ptr())
        for a, ax in enumerate("xy"):
            for f in ("fl", "fr", "gl", "gr", "ef", "cw"):
                getattr(B, f)[a] = t[f + ax].data_ptr()
            B.ftab4[a] = t["ftab4" + ax].data_ptr()
        for e in range(5):
            B.env[e] = t["env"][e].data_ptr()
        B.table_tile = t["table_tile"].data_ptr() if "table_tile" in t else None
        self._buffers = B
        self._params = self._make_params(num)
        handle = ctypes.c_void_p()
        _lib.call("w2b_create", ctypes.byref(self._desc), ctypes.byref(self._params), ctypes.byref(B),
                  ctypes.byref(handle))  # fmt: skip
        self.handle = handle
        self.bc = BoundaryCells.empty()
        self._bc_tensors = None
        self.hooks = None
        self.extra_wave = 0.0
        self.wet = TileFlags(self)
        self.set_active(np.arange(1, nt, dtype=np.int32))

    # ------------------------------------------------------------------ plumbing

    @staticmethod
    def _make_params(num: NumericsRecord) -> _lib.Params:
        return _lib.Params(
            num.g, num.dx, num.e_wet, num.h_cfl, num.u_max, num.lead, num.a_min, int(num.second), int(num.sheet),
            int(num.mirror), int(num.carry), int(getattr(num, "level_fp64", False)),
            _lib.ARITH[getattr(num, "arith", "exact")],
        )  # fmt: skip

    def _stream(self) -> int:
        return self.torch.cuda.current_stream(self.device).cuda_stream

    def native(self, name: str):
        """The current device tensor of a field, NATIVE layout (for the velocities and momenta, with the momenta put in
        their arrays first: w2b_sync_momentum)."""
        if name in MOMENTUM_FIELDS:
            self.sync_momentum()
        p = ctypes.c_void_p()
        _lib.call("w2b_field_ptr", self.handle, _lib.FIELD_ID[name], ctypes.byref(p))
        for key in ("h", "u", "v", "mx", "my"):
            pair = self._t[key]
            for half in (0, 1):
                if pair[half].data_ptr() == p.value:
                    return pair[half]
        key = name
        return self._t[key]

    def sync_momentum(self) -> None:
        """The face momenta into their arrays, on the current stream, before the state is read or written directly
        (the steps form them from the mean depths and face velocities instead of storing them)."""
        _lib.call("w2b_sync_momentum", self.handle, self._stream())

    def __getattr__(self, name: str):
        if name in STATE:
            return Field(self, name)
        raise AttributeError(name)

    def __del__(self) -> None:
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            try:
                _lib.lib().w2b_destroy(h)
            except Exception:
                pass
            self.handle = ctypes.c_void_p()

    # ------------------------------------------------------------------ the reference backend interface

    def set_active(self, active: np.ndarray) -> None:
        self.active_tiles = np.ascontiguousarray(active, np.int32)
        self.nact = int(self.active_tiles.size)
        torch = self.torch
        act = self._t["active"]
        if self.nact:
            act[: self.nact] = torch.as_tensor(self.active_tiles, device=self.device)
        flags = np.zeros(self.grid.ntiles, np.int32)
        flags[self.active_tiles] = 1
        self._t["is_act"].copy_(torch.as_tensor(flags, device=self.device))
        _lib.call("w2b_set_active", self.handle, act.data_ptr(), self.nact, self._stream())

    @property
    def active(self):
        return self._t["active"][: self.nact]

    def set_field(self, name: str, a: np.ndarray) -> None:
        """A host array in the reference state layout (ntiles * 1296) into the field's own cells."""
        a = np.ascontiguousarray(a, np.float32)
        if a.size != self.grid.ntiles * STRIDE2:
            raise ValueError(f"set_field {name}: {a.size} values for {self.grid.ntiles * STRIDE2}")
        _lib.call("w2b_set_field", self.handle, _lib.FIELD_ID[name], a.ctypes.data, _lib.LAYOUT_REF_TILE, 1,
                  self._stream())  # fmt: skip

    def get_field(self, name: str) -> np.ndarray:
        """The field in the reference state layout; halo entries hold the neighbour cells they copy."""
        out = np.empty(self.grid.ntiles * STRIDE2, np.float32)
        _lib.call("w2b_get_field", self.handle, _lib.FIELD_ID[name], out.ctypes.data, _lib.LAYOUT_REF_TILE, 1,
                  self._stream())  # fmt: skip
        return out

    def set_boundary(self, bc: BoundaryCells) -> None:
        torch = self.torch
        self.bc = bc
        n = int(bc.cell.size)
        nx = self.grid.shape[1]
        cell = native_of_ref(self.grid.tiles, bc.cell, nx).astype(np.int32)
        ref = native_of_ref(self.grid.tiles, bc.ref, nx).astype(np.int32) if n else cell

        def dev(a, dtype):
            return torch.as_tensor(np.ascontiguousarray(a), device=self.device).to(dtype).contiguous()

        self._bc_tensors = (dev(cell, torch.int32), dev(ref, torch.int32), dev(bc.kind, torch.int32),
                            dev(bc.d0, torch.float32), dev(bc.h0, torch.float32))  # fmt: skip
        ptrs = [x.data_ptr() if n else None for x in self._bc_tensors]
        torch.cuda.current_stream(self.device).synchronize()
        _lib.call("w2b_set_boundary", self.handle, n, *ptrs)
        torch.cuda.synchronize(self.device)

    def refresh_plan(self, tiles: np.ndarray) -> None:
        if tiles.size:
            lst = self.torch.as_tensor(np.ascontiguousarray(tiles, np.int32), device=self.device)
            _lib.call("w2b_refresh_plan", self.handle, lst.data_ptr(), int(lst.numel()), self._stream())

    def refresh_halos(self) -> None:
        """Nothing to do: the NATIVE layout has no halo copies."""

    def step(self, dt: float, want_wave: bool, want_wet: bool) -> None:
        _lib.call("w2b_step", self.handle, float(np.float32(dt)), int(want_wave), int(want_wet), self._stream())

    def loop_config(self) -> dict:
        """The device loop's launch schedule (w2b_loop_config): the face and update passes' CTAs a SM and the loop
        steps a captured graph (while the tuner runs: the next graph launch's), whether it is still tuning, and each
        pass's resident CTAs a SM."""
        out = np.zeros(9, np.int32)
        _lib.call("w2b_loop_config", self.handle, out.ctypes.data)
        keys = ("faces_per_sm", "update_per_sm", "steps_per_graph", "tuning", "faces_occupancy", "update_occupancy",
                "strips", "strips16_occupancy", "strips8_occupancy")  # fmt: skip
        return {k: int(v) for k, v in zip(keys, out, strict=True)}

    def set_loop(self, tune: bool = True, faces_per_sm: int = 0, update_per_sm: int = 0, steps: int = 0,
                 strips: int = 0) -> None:  # fmt: skip
        """Start the launch tuner again (``tune``), or fix the device loop's launch schedule (w2b_loop_tuning): the face
        pass's CTAs a SM in its tile form, or with ``strips`` (16 or 8) in its strip form of that many rows, the
        update pass's CTAs a SM, steps a graph."""
        if strips not in (0, 8, 16):
            raise ValueError("strips: 0 (the tile form), 16 or 8")
        code = 1 if tune else {0: 0, 16: 2, 8: 3}[strips]
        _lib.call("w2b_loop_tuning", self.handle, code, int(faces_per_sm), int(update_per_sm), int(steps))

    def max_wave(self) -> float:
        w = ctypes.c_float()
        _lib.call("w2b_max_wave", self.handle, ctypes.byref(w), self._stream())
        return max(float(w.value), float(self.extra_wave))

    def wet_flags(self) -> np.ndarray:
        out = np.empty(self.grid.ntiles, np.int32)
        _lib.call("w2b_wet_flags", self.handle, out.ctypes.data, self._stream())
        return out

    def synchronize(self) -> None:
        self.torch.cuda.synchronize(self.device)

    @property
    def wave(self) -> np.ndarray:
        return self._t["wave"].cpu().numpy()

    # ------------------------------------------------------------------ envelope, tally, device loop

    def maxima(self, t: float, arrive: float, deep: float) -> None:
        _lib.call("w2b_maxima", self.handle, float(np.float32(t)), float(np.float32(arrive)), float(np.float32(deep)),
                  self._stream())  # fmt: skip

    def envelope(self) -> list:
        return self._t["env"]

    def set_tally(self, face_ref: np.ndarray, axis: np.ndarray, sign: np.ndarray):
        torch = self.torch
        n = int(face_ref.size)
        face = native_of_ref(self.grid.tiles, face_ref, self.grid.shape[1]).astype(np.int32)
        self._tally = (torch.as_tensor(face, device=self.device), torch.as_tensor(np.asarray(axis, np.int32), device=self.device),
                       torch.as_tensor(np.asarray(sign, np.float32), device=self.device),
                       torch.zeros(max(n, 1), dtype=torch.float64, device=self.device))  # fmt: skip
        ptrs = [x.data_ptr() if n else None for x in self._tally]
        _lib.call("w2b_set_tally", self.handle, n, *ptrs)
        return self._tally[3][:n]

    def tally(self, dt: float) -> None:
        _lib.call("w2b_tally", self.handle, float(dt), self._stream())

    def advance_device(self, cfg: _lib.Stepper, t_end: float, max_steps: int, clock: _lib.Clock) -> int:
        """The device-resident step loop (w2b_advance); returns the status (0, or a failure code)."""
        return int(_lib.lib().w2b_advance(self.handle, ctypes.byref(cfg), float(t_end), int(max_steps),
                                          ctypes.byref(clock), self._stream()))  # fmt: skip
