"""The FP64 run. TEST INFRASTRUCTURE ONLY: only tests/ use it, as a checker.

``wadi_oracle.c`` compiled with ``-DOR_REAL_DOUBLE`` carries out the oracle's step (the reference's statements,
wadi2d/solver/cpu/kernels.py:19-334) with every operation in double: the same constants, the same float32 table
values and initial state, widened exactly. ``Model64`` drives it with a given time-step sequence (the float32 run's
own), so the two runs differ only by arithmetic precision, and ``field_errors`` reports, field by field, how far a
float32 result lies from the FP64 one. The reference's step has no FP64 form of its own; this run is the yardstick
for the float32 arithmetic that both the reference and the CUDA path use.
"""

from __future__ import annotations

import ctypes
import subprocess

import numpy as np

from oracle import oracle as O

LIB64_PATH = O.HERE / "_build" / "liboracle64.so"
_F64P = ctypes.POINTER(ctypes.c_double)
_I32P = ctypes.POINTER(ctypes.c_int32)

STATE_ARRAYS = "h d u v mx my qx qy u1 v1 mx1 my1 qx1 qy1 r src res om".split()
STATIC_ARRAYS = ["Hc", "dtab", "zcx", "zcy"] + [f + ax for ax in "xy" for f in ("fl", "fr", "gl", "gr", "ef", "cw", "ftab")]


def build64(force: bool = False):
    """Compile the double form of ``wadi_oracle.c`` (no FMA contraction, no fast math, OpenMP)."""
    src = O.HERE / "wadi_oracle.c"
    if LIB64_PATH.exists() and not force and LIB64_PATH.stat().st_mtime >= src.stat().st_mtime:
        return LIB64_PATH
    LIB64_PATH.parent.mkdir(parents=True, exist_ok=True)
    cmd = [
        "gcc", "-O2", "-fopenmp", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-shared", "-DOR_REAL_DOUBLE",
        "-o", str(LIB64_PATH), str(src), "-lm",
    ]  # fmt: skip
    subprocess.run(cmd, check=True)
    return LIB64_PATH


class OrParams64(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in ("g", "dx", "e_wet", "h_cfl", "u_max", "lead", "a_min")] + [
        (n, ctypes.c_int32) for n in ("rows", "second", "sheet", "mirror", "carry")
    ]


class OrArrays64(ctypes.Structure):
    _fields_ = [(n, _F64P) for n in O._ARRAY_FIELDS] + [("wet", _I32P)]


_lib64 = None


def lib64():
    global _lib64
    if _lib64 is None:
        L = ctypes.CDLL(str(build64()))
        P = ctypes.POINTER
        d = ctypes.c_double
        L.or_faces.argtypes = [P(OrArrays64), P(OrParams64), _I32P, ctypes.c_int, d, ctypes.c_int]
        L.or_limit.argtypes = [P(OrArrays64), P(OrParams64), _I32P, ctypes.c_int, d]
        L.or_update.argtypes = [P(OrArrays64), P(OrParams64), _I32P, ctypes.c_int, d, ctypes.c_int]
        L.or_plan.argtypes = [P(OrArrays64), P(OrParams64), _I32P, ctypes.c_int]
        L.or_exchange.argtypes = [_I32P, ctypes.c_int, _I32P, _I32P, ctypes.c_int, _F64P]
        L.or_boundary.argtypes = [ctypes.c_int, _I32P, _I32P, _I32P, _F64P, _F64P, _F64P, _F64P]
        L.or_maxima.argtypes = [_I32P, ctypes.c_int] + [d] * 3 + [_F64P] * 9
        L.or_tally.argtypes = [ctypes.c_int, d, _I32P, _I32P, _F64P, _F64P, _F64P, _F64P]
        _lib64 = L
    return _lib64


def _p(a, t=_F64P):
    return None if a is None else a.ctypes.data_as(t)


class Backend64(O.Backend):
    """The oracle backend on float64 arrays and the double kernels."""

    def __init__(self, grid, tables: dict, num) -> None:
        super().__init__(grid, tables, num)
        for name in STATE_ARRAYS + STATIC_ARRAYS + ["wave"]:
            setattr(self, name, np.asarray(getattr(self, name), np.float64).copy())
        self.params = OrParams64(
            O.G, grid.dx, num.e_wet, num.h_cfl, num.u_max, float(num.dt_every), num.plan_min, self.rows,
            int(num.second), int(num.sheet_flow), int(num.mirror_dry_faces), int(num.face_depth_carry),
        )  # fmt: skip
        self.bc64 = None

    def _arrays(self) -> OrArrays64:
        a = OrArrays64()
        for n in O._ARRAY_FIELDS:
            setattr(a, n, _p(getattr(self, n)))
        a.wet = _p(self.wet, _I32P)
        return a

    def set_boundary(self, bc) -> None:
        self.bc = bc
        self.bc64 = (np.asarray(bc.d0, np.float64).copy(), np.asarray(bc.h0, np.float64).copy())

    def _exch(self, *arrays) -> None:
        L = lib64()
        for a in arrays:
            L.or_exchange(_p(self.active, _I32P), self.nact, _p(self.slot, _I32P), _p(self.src_map, _I32P), self.nhalo,
                          _p(a))  # fmt: skip

    def refresh_plan(self, tiles: np.ndarray) -> None:
        if tiles.size:
            t = np.ascontiguousarray(tiles, np.int32)
            lib64().or_plan(ctypes.byref(self._arrays()), ctypes.byref(self.params), _p(t, _I32P), int(t.size))

    def step(self, dt: float, want_wave: bool, want_wet: bool) -> None:
        if want_wave:
            self.wave[:] = 0.0
        if self.nact == 0:
            return
        L = lib64()
        arr, par, act = ctypes.byref(self._arrays()), ctypes.byref(self.params), _p(self.active, _I32P)
        L.or_faces(arr, par, act, self.nact, float(dt), int(want_wave))
        self._exch(self.u1, self.v1, self.qx1, self.qy1)
        L.or_limit(arr, par, act, self.nact, float(dt))
        self._exch(self.r)
        L.or_update(arr, par, act, self.nact, float(dt), int(want_wave))
        if self.bc.cell.size:
            b = self.bc
            L.or_boundary(
                int(b.cell.size), _p(b.cell, _I32P), _p(b.ref, _I32P), _p(b.kind, _I32P), _p(self.bc64[0]),
                _p(self.bc64[1]), _p(self.h), _p(self.d),
            )  # fmt: skip
        self._exch(self.h, self.d, self.qx, self.qy)
        if want_wave:
            self._exch(self.om)
        self.u, self.u1 = self.u1, self.u
        self.v, self.v1 = self.v1, self.v
        self.mx, self.mx1 = self.mx1, self.mx
        self.my, self.my1 = self.my1, self.my


class Model64(O.Model):
    """The oracle model on ``Backend64``, stepped through a given dt sequence (``replay``)."""

    def __init__(self, grid, tables: dict, num=None) -> None:
        super().__init__(grid, tables, num)
        self.backend = Backend64(grid, tables, self.num)

    def replay(self, dts, on_step=None) -> float:
        """The stepper's loop (wadi2d/solver/stepper.py:106-129) with each step's dt taken from ``dts``: the same
        refresh and sleeping-tile schedule, no dt rule."""
        b, num = self.backend, self.num
        for dt in dts:
            refresh = self.refresh_due or self.nsteps % num.dt_every == 0
            self.refresh_due = False
            activate = self.nsteps % num.active_every == 0
            if self.kick is not None:
                self.kick.apply(b, float(dt))
            b.step(float(dt), refresh, activate)
            self.dts.append(float(dt))
            self.t += float(dt)
            self.nsteps += 1
            if activate and self.adaptive_active:
                self.rebuild_active(check=True)
            if on_step is not None:
                on_step(self)
        return self.t


class Maxima64(O.Maxima):
    """The envelope on the FP64 run's arrays."""

    def __init__(self, model: Model64, arrival_depth: float = 0.1, speed_depth: float = 0.05) -> None:
        super().__init__(model, arrival_depth, speed_depth)
        self.arrays = [np.asarray(a, np.float64).copy() for a in self.arrays]

    def update(self, t: float) -> None:
        b = self.model.backend
        lib64().or_maxima(
            _p(b.active, _I32P), b.nact, float(t), self.arrive, self.deep, _p(b.d), _p(b.h), _p(b.u), _p(b.v),
            *(_p(a) for a in self.arrays),
        )  # fmt: skip


class Tally64(O.Tally):
    """The outfall tally on the FP64 run's discharges."""

    def __init__(self, model: Model64, xfaces, xsign, yfaces, ysign) -> None:
        super().__init__(model, xfaces, xsign, yfaces, ysign)
        self.sign = self.sign.astype(np.float64)

    def add(self, dt: float) -> None:
        b = self.model.backend
        lib64().or_tally(
            int(self.face.size), float(dt), _p(self.face, _I32P), _p(self.axis, _I32P), _p(self.sign), _p(b.qx),
            _p(b.qy), _p(self.total),
        )  # fmt: skip


def field_errors(f32: np.ndarray, f64: np.ndarray) -> dict:
    """How far float32 results lie from the FP64 run: the largest absolute difference, the field's scale (its
    largest magnitude in the FP64 run) and their ratio."""
    a = np.asarray(f32, np.float64)
    b = np.asarray(f64, np.float64)
    diff = float(np.abs(a - b).max()) if a.size else 0.0
    scale = float(np.abs(b).max()) if b.size else 0.0
    return {"max_abs": diff, "scale": scale, "rel_to_scale": diff / scale if scale > 0 else 0.0}
