"""ctypes binding of libwadi_b200.so (include/wadi_b200.h). Loading fails loudly: there is no fallback."""

from __future__ import annotations

import ctypes
from pathlib import Path

LIB_PATH = Path(__file__).resolve().with_name("libwadi_b200.so")

c_i32, c_i64, c_f32, c_f64, c_vp = ctypes.c_int32, ctypes.c_int64, ctypes.c_float, ctypes.c_double, ctypes.c_void_p

OK, EINVAL, ECUDA, ENONFINITE, EDTMIN, ETIMEOUT = 0, -1, -2, -3, -4, -5
LAYOUT_REF_TILE, LAYOUT_NATIVE = 0, 1
ARITH_EXACT, ARITH_FAST = 0, 1
ARITH = {"exact": ARITH_EXACT, "fast": ARITH_FAST}
FIELDS = ("h", "d", "u", "v", "mx", "my", "qx", "qy", "u1", "v1", "mx1", "my1", "qx1", "qy1", "src", "res", "om",
          "zcx", "zcy")  # fmt: skip
FIELD_ID = {n: i for i, n in enumerate(FIELDS)}
CTL_BYTES = 1024


class W2BError(RuntimeError):
    """A libwadi_b200 call returned a status other than W2B_OK."""

    def __init__(self, status: int, what: str) -> None:
        names = {EINVAL: "bad argument", ECUDA: "CUDA error", ENONFINITE: "non-finite wave speed",
                 EDTMIN: "time step below the minimum", ETIMEOUT: "device wait timed out"}  # fmt: skip
        super().__init__(f"{what}: {names.get(status, 'status')} ({status})")
        self.status = status


class GridDesc(ctypes.Structure):
    _fields_ = [("ny", c_i32), ("nx", c_i32), ("ntiles", c_i32), ("rows", c_i32), ("nruns", c_i32)]


class Layout(ctypes.Structure):
    _fields_ = [("gy", c_i32), ("gx", c_i32), ("px", c_i32), ("ncells", c_i64)]


class Params(ctypes.Structure):
    _fields_ = [(n, c_f32) for n in ("g", "dx", "e_wet", "h_cfl", "u_max", "lead", "a_min")] + [
        (n, c_i32) for n in ("second", "sheet", "mirror", "carry", "level_fp64", "arith")
    ]


class Buffers(ctypes.Structure):
    _fields_ = (
        [(n, c_vp * 2) for n in ("h", "u", "v", "mx", "my")]
        + [(n, c_vp) for n in ("d", "qx", "qy", "qx1", "qy1", "res", "src", "om", "zcx", "zcy", "hc")]
        + [(n, c_vp * 2) for n in ("fl", "fr", "gl", "gr", "ef", "cw")]
        + [("dtab2", c_vp), ("ftab4", c_vp * 2)]
        + [(n, c_vp) for n in ("tiles", "tile_of", "nbr", "active", "wave", "wet", "keep", "idle", "is_act", "woken",
                               "work", "scratch", "bmark")]  # fmt: skip
        + [("env", c_vp * 5), ("ctl", c_vp), ("runs", c_vp), ("tile_run", c_vp), ("stage", c_vp), ("table_tile", c_vp)]
        + [("lpair", c_vp), ("lrow", c_vp)]
    )


class Stepper(ctypes.Structure):
    _fields_ = [(n, c_f64) for n in ("cfl", "wave_floor", "dt_max", "dt_min")] + [
        (n, c_i32) for n in ("dt_every", "active_every", "adaptive", "max_every")
    ] + [("arrive", c_f32), ("deep", c_f32)]


class Rain(ctypes.Structure):
    _fields_ = [("n", c_i64), ("cells", c_vp), ("depth", c_vp), ("loss", c_i32), ("s_mm", c_vp), ("ia_mm", c_vp),
                ("fc_mm_h", c_f64), ("partial", c_vp)]  # fmt: skip


PARTIALS = 296
INFLOWS_MAX, INFLOW_CELLS_MAX = 64, 4096


class Inflow(ctypes.Structure):
    _fields_ = [("n", c_i32), ("start", c_vp), ("lowest", c_vp), ("min_depth", c_vp), ("cells", c_vp),
                ("rained", c_vp), ("area", c_f64), ("volume", c_vp)]  # fmt: skip


class Clock(ctypes.Structure):
    _fields_ = [("t", c_f64), ("dt", c_f64), ("nsteps", c_i64), ("refresh_due", c_i32), ("status", c_i32),
                ("wave_max", c_f32), ("nact", c_i32)]  # fmt: skip


_SIGNATURES = {
    "w2b_version": [],
    "w2b_selftest_cbrt": [ctypes.c_uint32, ctypes.c_uint32, c_vp, c_vp],
    "w2b_selftest_wait": [ctypes.c_uint32, c_vp, c_vp],
    "w2b_layout": [ctypes.POINTER(GridDesc), ctypes.POINTER(Layout)],
    "w2b_ref_to_native": [ctypes.POINTER(GridDesc), c_vp, c_i64, c_vp, c_vp],
    "w2b_create": [ctypes.POINTER(GridDesc), ctypes.POINTER(Params), ctypes.POINTER(Buffers), ctypes.POINTER(c_vp)],
    "w2b_destroy": [c_vp],
    "w2b_set_params": [c_vp, ctypes.POINTER(Params)],
    "w2b_pack_tables": [ctypes.POINTER(GridDesc), c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp],
    "w2b_set_active": [c_vp, c_vp, c_i32, c_vp],
    "w2b_set_boundary": [c_vp, c_i32, c_vp, c_vp, c_vp, c_vp, c_vp],
    "w2b_set_tally": [c_vp, c_i32, c_vp, c_vp, c_vp, c_vp],
    "w2b_step": [c_vp, c_f32, c_i32, c_i32, c_vp],
    "w2b_step_timed": [c_vp, c_f32, c_i32, c_i32, c_vp, ctypes.POINTER(c_f32)],
    "w2b_max_wave": [c_vp, ctypes.POINTER(c_f32), c_vp],
    "w2b_wet_flags": [c_vp, c_vp, c_vp],
    "w2b_refresh_plan": [c_vp, c_vp, c_i32, c_vp],
    "w2b_field_ptr": [c_vp, c_i32, ctypes.POINTER(c_vp)],
    "w2b_sync_momentum": [c_vp, c_vp],
    "w2b_get_field": [c_vp, c_i32, c_vp, c_i32, c_i32, c_vp],
    "w2b_set_field": [c_vp, c_i32, c_vp, c_i32, c_i32, c_vp],
    "w2b_maxima": [c_vp, c_f32, c_f32, c_f32, c_vp],
    "w2b_tally": [c_vp, c_f64, c_vp],
    "w2b_advance": [c_vp, ctypes.POINTER(Stepper), c_f64, c_i64, ctypes.POINTER(Clock), c_vp],
    "w2b_build_tables": [c_vp, c_vp, c_vp],
    "w2b_build_tables_noalloc": [c_vp, c_vp, c_vp],
    "w2b_table_workspace_doubles": [c_i32, c_i64],
    "w2b_run_table_bytes": [c_i32],
    "w2b_set_run_dx": [c_vp, c_vp, c_i32],
    "w2b_run_halves": [c_vp, c_vp, c_vp],
    "w2b_face_waves": [c_vp, c_i32, c_f32, c_vp, c_vp],
    "w2b_loop_tuning": [c_vp, c_i32, c_i32, c_i32, c_i32],
    "w2b_loop_config": [c_vp, c_vp],
    "w2b_mma_gemm": [c_vp, c_vp, c_i32, c_i32, c_i32, c_vp, c_vp, c_vp, c_vp],
    "w2b_bf16_act": [c_vp, c_i64, c_i32, c_vp, c_vp],
    "w2b_relu_back": [c_vp, c_vp, c_i64, c_vp, c_vp],
    "w2b_transpose_bf16": [c_vp, c_i32, c_i32, c_i32, c_vp, c_vp],
    "w2b_mse_grad": [c_vp, c_vp, c_i32, c_i32, c_i32, c_f32, c_vp, c_vp, c_vp],
    "w2b_colsum_bf16": [c_vp, c_i32, c_i32, c_vp, c_vp],
    "w2b_adam": [c_vp, c_vp, c_vp, c_vp, c_i64, c_f32, c_f32, c_f32, c_f32, c_vp, c_vp],
    "w2b_adam_table": [c_vp, c_vp, c_vp, c_vp, c_i64, c_vp, c_vp, c_f32, c_f32, c_f32, c_vp, c_vp],
    "w2b_source_runs": [c_vp, c_i64, c_vp, c_vp, c_vp],
    "w2b_set_lines": [c_vp, c_i32, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp],
    "w2b_advance_runs": [c_vp, ctypes.POINTER(Stepper), c_vp, c_i64, c_vp, c_vp],
    "w2b_cell_size": [c_vp, ctypes.POINTER(c_f32)],
    "w2b_rain_window": [c_vp, c_vp, c_f64, c_f64, c_f64, c_f64, c_vp, c_vp],
    "w2b_inflow_window": [c_vp, c_vp, c_vp, c_f64, c_f64, c_vp],
    "w2b_storage": [c_vp, c_i64, c_vp, c_vp, c_vp, c_vp],
}

_RETURNS_SIZE = ("w2b_run_table_bytes", "w2b_table_workspace_doubles")  # int64 sizes, not status codes

_lib = None


def lib() -> ctypes.CDLL:
    """The loaded library. Raises if it was not built: the package has no other implementation."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(
                f"{LIB_PATH.name} is not built; run `python -m wadi2d_b200.build` (nvcc, sm_100a). The package has no "
                "CPU or library fallback."
            )
        L = ctypes.CDLL(str(LIB_PATH))
        for name, args in _SIGNATURES.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = c_i64 if name in _RETURNS_SIZE else c_i32
        _lib = L
    return _lib


def call(name: str, *args) -> int:
    """Call an entry point; raise W2BError on a failing status."""
    status = int(getattr(lib(), name)(*args))
    if status != OK:
        raise W2BError(status, name)
    return status
