"""The run folder on the B200 backend: ``checkpoint.h5`` (enough to continue a run) and ``results.h5`` (maxima, map
snapshots, series and the balance), in the reference's layouts (wadi2d/io/checkpoint.py:23-86,
wadi2d/io/results.py:1-99): the same dataset paths, attribute names and semantics, read from and written to this
package's device state.

The files are HDF5 through h5py where h5py is installed (as on a machine that runs ``wadi2d run``). Without h5py the
same layout goes to a ``.npz`` archive at the same path: one array per dataset path (``state/h``, ``maxima/depth``,
``maps/t000000600/depth``, ...) and the attributes of the root and of each group as JSON under ``__attrs__``.
"""

from __future__ import annotations

import json
import re
from dataclasses import asdict
from pathlib import Path

import numpy as np

FORMAT_VERSION = "1.0"
CHECKPOINT_FORMAT = "2"
BALANCE = "balance_"
SAVED_ARRAYS = ("h", "d", "u", "v", "mx", "my", "qx", "qy", "res", "om")
"""The state, the cells' rounding residuals, and the wet share of the cell plan (wadi2d/io/checkpoint.py:19-20)."""
ATTRS = "__attrs__"


def _h5py():
    try:
        import h5py

        return h5py
    except ImportError:
        return None


def safe_name(name: str) -> str:
    """A name fit for a file: letters, digits, dot, dash and underscore (wadi2d/io/results.py:31-33)."""
    return re.sub(r"[^A-Za-z0-9._-]+", "_", name).strip("_") or "unnamed"


class Store:
    """Datasets by path and attributes by group path, kept in HDF5 (h5py) or in a ``.npz`` archive."""

    def __init__(self, path: str | Path, mode: str = "r") -> None:
        self.path = Path(path)
        self.mode = mode
        h5 = _h5py()
        self.h5 = h5.File(self.path, mode) if h5 is not None else None
        self.data: dict[str, np.ndarray] = {}
        self.attrs: dict[str, dict] = {}
        if self.h5 is None and mode in ("r", "a") and self.path.exists():
            with np.load(self.path, allow_pickle=False) as z:
                self.data = {k: z[k] for k in z.files if k != ATTRS}
                self.attrs = json.loads(str(z[ATTRS])) if ATTRS in z.files else {}

    def put(self, name: str, a) -> None:
        a = np.asarray(a)
        if self.h5 is not None:
            if name in self.h5:
                del self.h5[name]
            kw = {"compression": "gzip", "compression_opts": 1} if a.ndim == 2 else {}
            self.h5.create_dataset(name, data=a, **kw)
        else:
            self.data[name] = a.copy()

    def get(self, name: str) -> np.ndarray:
        return self.h5[name][()] if self.h5 is not None else self.data[name]

    def has(self, name: str) -> bool:
        if self.h5 is not None:
            return name in self.h5
        return name in self.data or any(k.startswith(name + "/") for k in self.data)

    def children(self, group: str) -> list[str]:
        if self.h5 is not None:
            return list(self.h5[group]) if group in self.h5 else []
        pre = group + "/"
        return sorted({k[len(pre) :].split("/")[0] for k in self.data if k.startswith(pre)})

    def set_attr(self, group: str, key: str, value) -> None:
        if isinstance(value, np.generic):
            value = value.item()
        if self.h5 is not None:
            (self.h5 if group == "" else self.h5.require_group(group)).attrs[key] = value
        else:
            self.attrs.setdefault(group, {})[key] = value

    def attr(self, group: str, key: str, default=None):
        if self.h5 is not None:
            obj = self.h5 if group == "" else self.h5[group]
            v = obj.attrs.get(key, default)
            return v.item() if isinstance(v, np.generic) else v
        return self.attrs.get(group, {}).get(key, default)

    def group_attrs(self, group: str) -> dict:
        if self.h5 is not None:
            obj = self.h5 if group == "" else self.h5[group]
            return {k: (v.item() if isinstance(v, np.generic) else v) for k, v in obj.attrs.items()}
        return dict(self.attrs.get(group, {}))

    def close(self) -> None:
        if self.h5 is not None:
            self.h5.close()
            return
        if self.mode != "r":
            tmp = self.path.with_name(self.path.name + ".part")
            with open(tmp, "wb") as f:
                np.savez(f, **self.data, **{ATTRS: np.array(json.dumps(self.attrs))})
            tmp.replace(self.path)


# ------------------------------------------------------------------------------------------------ checkpoint


def save_checkpoint(path: str | Path, model, maxima, tally, balance, job_hash: str, times=(), series=(),
                    next_series: float = 0.0, next_map: float = 0.0) -> Path:  # fmt: skip
    """Write a checkpoint through a temporary name, so that a crash during the write leaves the last good one
    (wadi2d/io/checkpoint.py:23-50). ``series``: the columns of each recorded series, in the monitor's order."""
    out = Path(path)
    tmp = out.with_name(out.name + ".tmp")
    st = model.stepper
    model.backend.synchronize()
    volume = tally.volume() if tally is not None else 0.0
    balance.outflow = volume
    f = Store(tmp, "w")
    try:
        f.set_attr("", "format", CHECKPOINT_FORMAT)
        f.set_attr("", "job_hash", job_hash)
        f.set_attr("", "tally", volume)
        f.set_attr("", "t", float(st.t))
        f.set_attr("", "dt", float(st.dt))
        f.set_attr("", "nsteps", int(st.nsteps))
        f.set_attr("", "next_series", float(next_series))
        f.set_attr("", "next_map", float(next_map))
        for name in SAVED_ARRAYS:
            f.put(f"state/{name}", model.backend.get_field(name))
        if maxima is not None:
            for name, a in maxima.raw().items():
                f.put(f"maxima/{name}", a)
        for key, value in asdict(balance).items():
            f.set_attr("", f"{BALANCE}{key}", float(value))
        f.put("times", np.asarray(times, np.float64))
        for n, columns in enumerate(series):
            for key, values in columns.items():
                f.put(f"series/{n}/{key}", np.asarray(values, np.float64))
    finally:
        f.close()
    tmp.replace(out)
    return out


def checkpoint_job(path: str | Path) -> str | None:
    """The hash of the job that wrote this checkpoint; None for a file too old or damaged to say
    (wadi2d/io/checkpoint.py:53-61)."""
    try:
        f = Store(path, "r")
        try:
            if f.attr("", "format") != CHECKPOINT_FORMAT:
                return None
            return str(f.attr("", "job_hash"))
        finally:
            f.close()
    except (OSError, KeyError, ValueError):
        return None


def load_checkpoint(path: str | Path, model, maxima, tally, balance_type) -> dict:
    """Put a saved run back into a freshly built model of the same job (wadi2d/io/checkpoint.py:64-86): the state,
    the envelope, the clock and the tally; the tiles' wet flags and the active list are rebuilt from the depths.
    Returns the balance (a ``balance_type``), the recorded times and series columns, and the next series and map
    times."""
    f = Store(path, "r")
    try:
        for name in SAVED_ARRAYS:
            model.backend.set_field(name, f.get(f"state/{name}"))
        if maxima is not None:
            maxima.restore({name: f.get(f"maxima/{name}") for name in f.children("maxima")})
        st = model.stepper
        st.t, st.dt, st.nsteps = float(f.attr("", "t")), float(f.attr("", "dt")), int(f.attr("", "nsteps"))
        saved = {k[len(BALANCE) :]: v for k, v in f.group_attrs("").items() if k.startswith(BALANCE)}
        balance = balance_type(**saved)
        if tally is not None:
            tally.restore(float(f.attr("", "tally", balance.outflow)))
        times = list(f.get("times"))
        series = [{key: list(f.get(f"series/{n}/{key}")) for key in f.children(f"series/{n}")}
                  for n in sorted(int(x) for x in f.children("series"))]  # fmt: skip
        out = {"balance": balance, "times": times, "series": series,
               "next_series": float(f.attr("", "next_series")), "next_map": float(f.attr("", "next_map"))}  # fmt: skip
    finally:
        f.close()
    model.backend.wet[:] = model._tile_wet(model.field("h"))
    model.stepper.rebuild_active()
    return out


# ------------------------------------------------------------------------------------------------ results


class Results:
    """An open results file; snapshots append, so a stopped run keeps what it wrote (wadi2d/io/results.py:37-99).
    ``grid`` None: a run with no grid, series only."""

    def __init__(self, path: str | Path, grid, crs_wkt: str = "", config_json: str = "{}", append: bool = False):
        self.path = Path(path)
        self.f = Store(self.path, "a" if append and self.path.exists() else "w")
        if self.f.has("mask"):
            return
        self.f.set_attr("", "format_version", FORMAT_VERSION)
        self.f.set_attr("", "crs", crs_wkt)
        self.f.set_attr("", "config", config_json)
        if grid is None:
            self.f.set_attr("", "lumped_only", True)
            return
        for key, value in (("x0", grid.x0), ("y0", grid.y0), ("dx", grid.dx)):
            self.f.set_attr("", key, float(value))
        self.f.put("mask", np.asarray(grid.mask))

    def snapshot(self, t: float, fields: dict[str, np.ndarray]) -> None:
        group = f"maps/t{round(t):09d}"
        self.f.set_attr(group, "t_s", float(t))
        for name, a in fields.items():
            if not self.f.has(f"{group}/{name}"):
                self.f.put(f"{group}/{name}", np.asarray(a, np.float32))

    def maxima(self, fields: dict[str, np.ndarray]) -> None:
        for name, a in fields.items():
            self.f.put(f"maxima/{name}", np.asarray(a, np.float32))

    def series(self, kind: str, name: str, t, columns: dict) -> None:
        group = f"series/{kind}/{safe_name(name)}"
        self.f.set_attr(group, "name", name)
        for key, a in {"t_s": t, **columns}.items():
            self.f.put(f"{group}/{key}", np.asarray(a, np.float64))

    def attributes(self, values: dict) -> None:
        for key, value in values.items():
            self.f.set_attr("", key, value)

    def close(self) -> None:
        self.f.close()


def read_results(path: str | Path) -> Store:
    """A results file opened for reading (either form)."""
    return Store(path, "r")
