"""Make the golden vectors that pin the oracle: run the reference's own CPU engine on small seeded cases.

Run in a container that holds the reference source tree (read-only is fine):

    WADI2D_REFERENCE=<the reference source tree> NUMBA_CACHE_DIR=/tmp/numba_cache PYTHONDONTWRITEBYTECODE=1 \
        python tests/golden/make_golden.py

It imports ``wadi2d`` from that tree and drives ``Model(..., "cpu")`` (the Numba twin of the reference's GPU
kernels) through the cases of ``tests/golden/cases.py``, the calls its own tests make. It writes, per case,
``<case>.npz`` (final state arrays in the reference tile-with-halo layout, every step size, the envelope, the
boundary tally and, for ``c1_small``, the FP64 host helpers) and ``<case>.json`` (SHA-256 of every table array, bit
for bit, and of the seeded inputs, so a drift in the generator shows). Nothing on the GPU side reads the reference:
these files are the only thing that travels.
"""

from __future__ import annotations

import hashlib
import json
import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1]))
sys.path.insert(0, str(HERE))
if not os.environ.get("WADI2D_REFERENCE"):
    sys.exit("set WADI2D_REFERENCE to the reference source tree")
sys.path.insert(0, os.environ["WADI2D_REFERENCE"])

from wadi2d.config.schema import Numerics, Tables  # noqa: E402
from wadi2d.engine.maxima import Maxima, Tally  # noqa: E402
from wadi2d.grid import TileGrid  # noqa: E402
from wadi2d.solver.backend import BoundaryCells  # noqa: E402
from wadi2d.solver.model import Model  # noqa: E402
from wadi2d.solver.state import level_field, plan_field  # noqa: E402
from wadi2d.tables import ArrayBed, build_tables  # noqa: E402
from wadi2d.tables.builder import CrestFaces, hbar_at_level  # noqa: E402

import cases  # noqa: E402

TABLES = ("hc", "dtab", "flx", "frx", "glx", "grx", "efx", "cwx", "ftabx", "fly", "fry", "gly", "gry", "efy", "cwy",
          "ftaby", "zcx", "zcy", "zmin", "zbar")  # fmt: skip


def digest(a: np.ndarray) -> str:
    a = np.ascontiguousarray(a)
    return hashlib.sha256(a.dtype.str.encode() + str(a.shape).encode() + a.tobytes()).hexdigest()


class ReferenceApi:
    """The adapter of tests/golden/cases.py onto the reference's own classes."""

    def __init__(self) -> None:
        self.dts: list[float] = []

    def grid(self, mask, x0, y0, dx):
        return TileGrid.from_mask(mask, x0, y0, dx)

    def tables(self, grid, z, pixel, manning, local, crest, npix):
        lining = None
        if npix is not None:

            def lining(zz, n, row0, col0):
                r = np.clip(np.arange(row0, row0 + zz.shape[0]), 0, npix.shape[0] - 1)
                c = np.clip(np.arange(col0, col0 + zz.shape[1]), 0, npix.shape[1] - 1)
                n[:] = npix[np.ix_(r, c)]

        cfg = Tables(face_conveyance="local_radius" if local else "strips")
        return build_tables(grid, ArrayBed(z, pixel), cfg, manning, crest=crest, lining=lining)

    def model(self, grid, tables, numerics):
        m = Model(tables, Numerics.model_construct(**numerics), "cpu")
        step = m.backend.step

        def logged(dt, want_wave, want_wet):
            self.dts.append(float(dt))
            step(dt, want_wave, want_wet)

        m.backend.step = logged
        return m

    def boundary(self, cell, ref, kind, d0, h0):
        return BoundaryCells(cell, ref, kind, d0, h0)

    def maxima(self, m, arrive, deep):
        return Maxima(m, arrive, deep)

    def tally(self, m, xf, xs, yf, ys):
        return Tally(m, xf, xs, yf, ys)

    def hbar_at_level(self, level, zmin, hc, dtab):
        return hbar_at_level(level, zmin, hc, dtab)

    def from_tiles(self, grid, tables, name):
        return grid.from_tiles(getattr(tables, name))

    def zmin(self, tables):
        return tables.zmin

    def crest(self, shape):
        return CrestFaces.empty(shape)


def main(names) -> None:
    for name in names:
        api = ReferenceApi()
        arrays, ctx = cases.CASES[name](api)
        arrays["dts"] = np.asarray(api.dts, np.float64)
        tables = ctx["tables"]
        if name == "c1_small":
            rng = np.random.default_rng(5)
            grid = ctx["grid"]
            hb = np.where(grid.mask, rng.random(grid.shape) ** 3 * 3.0, 0.0)
            arrays["fp64_hb_in"] = hb
            arrays["fp64_level"] = level_field(tables, hb)
            arrays["fp64_plan"] = plan_field(tables, hb)
            levels = tables.zmin + rng.random(grid.shape) * 3.0
            arrays["fp64_levels_in"] = levels
            hc, dtab = grid.from_tiles(tables.hc), grid.from_tiles(tables.dtab)
            arrays["fp64_hbar"] = hbar_at_level(levels, tables.zmin, hc, dtab)
        np.savez_compressed(HERE / f"{name}.npz", **arrays)
        meta = {
            "case": name,
            "tables": {n: digest(getattr(tables, n)) for n in TABLES},
            "inputs": {"z": digest(ctx["z"])},
            "nsteps": int(arrays["nsteps"]),
            "t": float(arrays["t"]),
        }
        (HERE / f"{name}.json").write_text(json.dumps(meta, indent=1, sort_keys=True) + "\n")
        print(name, "steps", int(arrays["nsteps"]), "volume", float(arrays["state_h"].sum()))


if __name__ == "__main__":
    main(sys.argv[1:] or list(cases.CASES))
