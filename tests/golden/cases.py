"""The golden cases, written once and driven through any implementation of the reference's Model API.

An ``api`` object supplies ``grid(mask, x0, y0, dx)``, ``tables(grid, z, pixel, manning, local, crest, npix)``,
``model(grid, tables, numerics: dict)``, ``boundary(cell, ref, kind, d0, h0)``, ``maxima(model, arrive, deep)``,
``tally(model, xfaces, xsign, yfaces, ysign)``, ``hbar_at_level(level, zmin, hc, dtab)``, ``from_tiles(grid, a)``,
``zmin(tables)`` and ``crest(shape)`` (an empty crest-face record with the reference's field names). The reference
(tests/golden/make_golden.py), the oracle and the CUDA path each provide one, so the three run the same calls the
reference's own tests make (tests/solver/harness.py, tests/solver/test_subgrid.py).
"""

from __future__ import annotations

import numpy as np

from wadi2d_b200 import workloads

STATE = ("h", "d", "u", "v", "mx", "my", "qx", "qy", "res", "om", "src")
MAXIMA = ("depth", "mean_depth", "speed", "hazard", "arrival")


def _record(m, extra: dict) -> dict:
    out = {f"state_{n}": m.backend.get_field(n) for n in STATE}
    out["wet"] = np.asarray(m.backend.wet_flags(), np.int32)
    out["active"] = np.asarray(m.backend.active_tiles, np.int32)
    out["nsteps"] = np.int64(m.stepper.nsteps)
    out["t"] = np.float64(m.stepper.t)
    out["dt_next"] = np.float64(m.stepper.dt)
    out.update(extra)
    return out


def c1_small_inputs(api, n: int = 64):
    w = workloads.v_channel_plane(n=n, dx=10.0, k=5, seed=0)
    grid = api.grid(np.ones((w.ny, w.nx), bool), 0.0, 0.0, w.dx)
    return grid, (w.z, w.dx / w.k, w.manning, True, None, None), w


def c1_small(api, t_end: float = 600.0, n: int = 64) -> tuple[dict, dict]:
    """Configuration 1 at n x n: rain on a V-channel plane, free outfall east, CFL 0.9, sleeping tiles on."""
    grid, targs, w = c1_small_inputs(api, n)
    tables = api.tables(grid, *targs)
    m = api.model(grid, tables, {"cfl": w.cfl})
    rows, cols = w.outfall
    cells = np.array([m.cell_state_index(int(j), int(i)) for j, i in zip(rows, cols, strict=True)], np.int32)
    k = cells.size
    m.set_boundary(api.boundary(cells, np.zeros(k, np.int32), np.ones(k, np.int32), np.zeros(k, np.float32),
                                np.zeros(k, np.float32)))  # fmt: skip
    rate = np.zeros(grid.shape)
    rate[1 : 1 + w.ny, 1 : w.nx] = w.rain_mm_h / 3.6e6
    m.set_source(rate)
    maxima = api.maxima(m, 0.1, 0.05)
    tally = api.tally(m, cells.astype(np.int64), np.ones(k), np.zeros(0, np.int64), np.zeros(0))
    last = [0.0]

    def on_step(st):
        tally.add(st.t - last[0])
        last[0] = st.t
        if st.nsteps % 4 == 0:
            maxima.update(st.t)

    m.advance(t_end, on_step)
    env = maxima.raw()
    extra = {f"max_{name}": env[name] for name in MAXIMA}
    extra["tally"] = np.float64(tally.volume())
    return _record(m, extra), {"z": w.z, "tables": tables, "grid": grid, "model": m}


def dambreak_inputs(api):
    nx, ny, k, dx = 60, 40, 6, 10.0
    grid = api.grid(np.ones((ny, nx), bool), 0.0, 0.0, dx)
    z = workloads.rough_dam_break_bed(nx, ny, k, dx, seed=3)
    return grid, (z, dx / k, 0.03, False, None, None), None


def dambreak(api, t_end: float = 20.0) -> tuple[dict, dict]:
    """The reference's rough dam break (tests/solver/test_subgrid.py:95-116) on strips tables, a fixed 0.2 s step."""
    grid, targs, _ = dambreak_inputs(api)
    z = targs[0]
    tables = api.tables(grid, *targs)
    m = api.model(grid, tables, {"dt_every": 1, "dt_max": 0.2})
    h0 = np.zeros(grid.shape)
    h0[:, :30] = 2.0
    m.set_depth(h0)
    m.advance(t_end)
    return _record(m, {}), {"z": z, "tables": tables, "grid": grid, "model": m}


CREST_DIMS = (56, 40, 4, 5.0)


def crest_inputs(api):
    """A sloping valley with a crest line of terrain objects, a wall, a lined channel strip and a natural ridge."""
    nx, ny, k, dx = CREST_DIMS
    grid = api.grid(np.ones((ny, nx), bool), 0.0, 0.0, dx)
    pny, pnx = grid.shape
    p = dx / k
    x = (np.arange(pnx * k) + 0.5) * p - dx
    y = (np.arange(pny * k) + 0.5) * p - dx
    X, Y = np.meshgrid(x, y)
    z = 50.0 + 0.004 * (nx * dx - X) + 0.02 * np.abs(Y - 0.5 * ny * dx)
    z += workloads.fractal_noise(z.shape, 0.7, 0.05, 11)
    ridge = (X > 40 * dx) & (X < 40 * dx + p)
    z[ridge] += 0.6
    crest = api.crest(grid.shape)
    ci = 24
    crest.xz[1 : 1 + ny, ci] = 51.2
    crest.xc[1 : 1 + ny // 2, ci] = 1.5
    crest.xc[1 + ny // 2 : 1 + ny, ci] = -1.2
    crest.xlen[1 : 1 + ny, ci] = 0.8
    crest.xwall = np.zeros(grid.shape, bool)
    crest.xwall[1:6, 30] = True
    crest.ywall = np.zeros(grid.shape, bool)
    crest.ywall[20, 10:16] = True
    yc = 0.5 * ny * dx
    npix = np.full(z.shape, np.nan)
    npix[np.abs(y - yc) < 3.0, :] = 0.015
    return grid, z, crest, npix, (nx, ny, k, dx)


def crest(api, t_end: float = 150.0) -> tuple[dict, dict]:
    """Crest caps (positive and negative coefficients), walls, lined pixels, fixed-stage and follow boundaries,
    initial velocities, point sources, sleeping tiles waking as the water spreads."""
    grid, z, crest_faces, npix, (nx, ny, k, dx) = crest_inputs(api)
    tables = api.tables(grid, z, dx / k, 0.04, True, crest_faces, npix)
    m = api.model(grid, tables, {})
    hc, dtab = api.from_tiles(grid, tables, "hc"), api.from_tiles(grid, tables, "dtab")
    zmin = api.zmin(tables)
    stage = 51.6
    h0 = np.where(grid.mask, api.hbar_at_level(np.full(grid.shape, stage), zmin, hc, dtab), 0.0)
    h0[:, 20:] = 0.0
    m.set_depth(h0)
    m.set_velocity(np.where(h0 > 0, 0.3, 0.0), np.where(h0 > 0, -0.05, 0.0))
    jj = np.arange(1, 1 + ny)
    west = np.array([m.cell_state_index(int(j), 1) for j in jj], np.int32)
    east = np.array([m.cell_state_index(int(j), nx) for j in jj], np.int32)
    east_ref = np.array([m.cell_state_index(int(j), nx - 1) for j in jj], np.int32)
    d0w = np.maximum(stage - zmin[jj, 1], 0.0)
    h0w = api.hbar_at_level(stage, zmin[jj, 1], hc[jj, 1], dtab[jj, 1])
    d0e = np.minimum(zmin[jj, nx - 1] - zmin[jj, nx] - 0.001 * dx, 0.0)
    m.set_boundary(api.boundary(
        np.concatenate((west, east)), np.concatenate((west, east_ref)),
        np.concatenate((np.zeros(ny, np.int32), np.full(ny, 2, np.int32))),
        np.concatenate((d0w, d0e)).astype(np.float32), np.concatenate((h0w, np.zeros(ny))).astype(np.float32),
    ))  # fmt: skip
    src_cells = np.array([m.cell_state_index(30, 10), m.cell_state_index(31, 10), m.cell_state_index(8, 44)], np.int64)
    m.set_source_cells(src_cells, np.array([2e-3, 1e-3, 5e-4], np.float32))
    m.advance(t_end)
    return _record(m, {}), {"z": z, "tables": tables, "grid": grid, "model": m}


def crest_table_inputs(api):
    grid, z, crest_faces, npix, (nx, ny, k, dx) = crest_inputs(api)
    return grid, (z, dx / k, 0.04, True, crest_faces, npix), None


CASES = {"c1_small": c1_small, "dambreak": dambreak, "crest": crest}
TABLE_INPUTS = {"c1_small": c1_small_inputs, "dambreak": dambreak_inputs, "crest": crest_table_inputs}
