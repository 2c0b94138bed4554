#!/usr/bin/env python
"""Benchmark of the uniform-grid shallow-water step on B200: cell-steps/s on configuration 3.

Workload (one rank): 4096 x 4096 cells at 30 m (16.8 M domain cells, 16,641 tiles of 32 x 32), 4 x 4 pixels a cell,
the seeded fractal catchment of ``wadi2d_b200.workloads.catchment`` with its tables built on the GPU; a wet start
(0.05 m of mean depth everywhere) under the storm's peak rain excess, five free outfalls; every tile stepped (the
reference's "adaptive_active off" headline mode); the envelope every 4 steps and the FP64 outfall tally every step,
as the reference's monitor takes them. A step is one time step of the whole grid (the device-resident loop,
graph-captured). Inputs stay resident in HBM (about 15 GB, far beyond the 126 MB L2).

The step is the fast build by default (``--arith``), the launch schedule and the face pass's form (tiles or strips)
chosen by the library's tuner before the timed steps. JSON line (rank 0): value = domain cell-steps per second over
all ranks (ranks run independent replicas: weak scaling, no collective in the data path); roofline of the dominant
kernel (the face pass) from CUDA events; parity = the timed build against the oracle on a block of the workload;
cpu_baseline = the oracle (a C restatement of the reference's CPU step) on that block; e2e = the same metric through
the C-ABI with host buffers (per 30 s window, as the reference's run driver and monitor take a run: the window's rain
uploaded from pinned memory a window ahead, the window stepped, the clock, active list, design-line discharge, outfall
volume and storage read back; the envelope maps at the end); sweep = the critical-duration search at a reduced size.

``--impl reference`` times the reference's CPU step (its restatement, the oracle, with every host thread) on the
same bounded block and prints the same line with "impl": "reference".
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

# Algorithmic bytes per cell-step, the problem's fixed figure (the reference's state and tables): the whole step 44 B
# of state read (h d u v mx my qx qy om res src), 40 B written, 60 B of static scalars, 40 B of table values, 10 B of
# envelope (5 arrays read and written every 4 steps). The face pass's share: d h u v mx my qx qy read (32 B) + om on
# refresh steps (4 B / 8), zcx zcy (8 B), 12 face scalars (48 B), two table quads (32 B); u v mx my qx qy written
# (24 B). The roofline's achieved GB/s counts these.
ALG_STEP = 194.0
ALG_FACES = 32.0 + 0.5 + 8.0 + 48.0 + 32.0 + 24.0
# The bytes this implementation's step needs: the face momenta are formed from the last step's mean depth and the
# face velocities instead of read and written (4 B read in place of 16 B read and written).
IMPL_STEP = ALG_STEP - 12.0
IMPL_FACES = ALG_FACES - 12.0
FALLBACK_HBM_GBS = 6650.0
# DRAM bytes a tile cell of the face pass (dram__bytes_read.sum + dram__bytes_write.sum of two launches, divided by
# their tile cells), from an ncu capture of fast::strips_kernel<8> (the form the tuner keeps) on configuration 3's
# catchment at 1024 x 1024 cells (1,115,136 tile cells a launch, beyond L2): profiles/strips8_kernel_fast_config3_1024.md.
# The traffic grows with the tile cells a launch processes, so it scales to this launch by them.
FACES_DRAM_BYTES_PER_CELL = 165.5
CPU_BLOCK_TILES = 32  # the CPU sample: a 32 x 32-tile block (1,044,484 active cells) from the middle of the grid


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=200)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", default="b200", choices=("b200", "reference"))
    p.add_argument("--arith", default="fast", choices=("exact", "fast"),
                   help="the step's build: fast (the default: FMA contraction, approximate division, square root and "
                        "powers in the face pass, held to the step's accuracy bounds against the oracle and the FP64 "
                        "run) or exact (the reference's float32 bits)")
    p.add_argument("--form", default="tuned", choices=("tuned", "tiles", "strips16", "strips8"),
                   help="the face pass's form: the one the launch tuner keeps (the default), or fixed (the tile form, or "
                        "strips of 16 or 8 rows, each at its resident CTAs a SM)")
    p.add_argument("--parity-steps", type=int, default=200,
                   help="steps of the CUDA path against the oracle on the CPU sample block (0: none)")
    p.add_argument("--n", type=int, default=4096, help="domain side in cells (configuration 3: 4096)")
    p.add_argument("--cpu-seconds", type=float, default=15.0)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--e2e-windows", type=int, default=64,
                   help="30 s windows of the end-to-end leg (a 36 h run has 4,320; the envelope maps are read once, "
                        "at the end, as a run reads them)")
    p.add_argument("--full-run", action="store_true",
                   help="the whole 36 h run of configuration 3 from dry ground, with its mass balance")
    p.add_argument("--sim-hours", type=float, default=36.0, help="--full-run: simulated hours (configuration 3: 36)")
    p.add_argument("--ensemble", action="store_true",
                   help="configuration 4: the storm sweep as one batch against the same runs one after another")
    p.add_argument("--runs", type=int, default=64, help="runs of the ensemble")
    p.add_argument("--side-max", type=int, default=2048, help="largest side of an ensemble run, cells")
    p.add_argument("--recession-min", type=float, default=30.0, help="simulated time after each storm, minutes")
    p.add_argument("--time-scale", type=float, default=1.0, help="share of each run's simulated time to step")
    p.add_argument("--skip-plain", action="store_true", help="the batch only (no one-after-another sweep)")
    p.add_argument("--arf-study", action="store_true",
                   help="the depth-area (ARF) study: every storm area of one catchment as one batch, against one run "
                        "after another")
    p.add_argument("--study-n", type=int, default=1024, help="--arf-study: catchment cells a side")
    p.add_argument("--config2-run", action="store_true",
                   help="configuration 2 end to end: 1024 x 1024, crests, lumped inflows, a reservoir, 6 h")
    p.add_argument("--host-inflows", action="store_true",
                   help="--config2-run: share the inflows on the host (levels read back each window, the window's "
                        "source uploaded) instead of on the device")
    p.add_argument("--table-build", action="store_true",
                   help="the GPU table build of configuration 2 (1024 x 1024, 1 m pixels) and 3 (4096 x 4096, 7.5 m)")
    p.add_argument("--critical", action="store_true",
                   help="configuration 5: the critical-duration search, screened by the network, against the sweep")
    p.add_argument("--candidates", type=int, default=400, help="--critical: candidate storms")
    p.add_argument("--train-runs", type=int, default=96, help="--critical: solver runs the network learns from")
    p.add_argument("--plain-sample", type=int, default=8, help="--critical: runs timed one after another")
    p.add_argument("--critical-dx", type=float, default=10.0, help="--critical: cell size, m")
    p.add_argument("--critical-relief", type=float, default=None,
                   help="--critical: relief of the catchment, m (default 3 %% of its length)")
    p.add_argument("--no-sweep", action="store_true", help="leave the bounded storm sweep out of the default line")
    return p.parse_args()


def peaks() -> tuple[float, str]:
    f = ROOT / "MEASURED_PEAKS.json"
    if f.exists():
        return float(json.loads(f.read_text())["hbm_gbs"]), "measured"
    return FALLBACK_HBM_GBS, "fallback"


class Clocks:
    """nvidia-smi sampled every 200 ms during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")  # fmt: skip

    def __init__(self, index: int) -> None:
        self.index = index
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.proc = None

    def start(self) -> None:
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", str(self.index)], stdout=self.file, stderr=subprocess.DEVNULL,
            )  # fmt: skip
        except OSError:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        self.proc.wait(timeout=10)
        self.file.seek(0)
        rows = [r.split(",") for r in self.file.read().strip().splitlines() if r.strip()]
        sm, mx, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx.append(float(r[2]))
            except (ValueError, IndexError):
                continue
            for name, v in zip(names, r[5:9], strict=False):
                if v.strip().lower() == "active":
                    reasons.add(name)
        os.unlink(self.file.name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}  # fmt: skip


def build_workload(n: int, device, arith: str = "exact"):
    """Configuration 3 on the GPU: catchment, tables, model, outfalls, wet start under peak rain."""
    from wadi2d_b200 import workloads
    from wadi2d_b200.backend import BoundaryCells
    from wadi2d_b200.config import Numerics, Tables
    from wadi2d_b200.grid import TileGrid
    from wadi2d_b200.maxima import Maxima, Tally
    from wadi2d_b200.model import Model
    from wadi2d_b200.tables import ArrayBed, build_tables

    c = workloads.catchment(n=n, device=device)
    grid = TileGrid.from_mask(np.ones((n, n), bool), 0.0, 0.0, c.dx)
    tables = build_tables(grid, ArrayBed(c.z, c.dx / c.k), Tables(), c.manning, device=device)
    cut_block(c, grid)
    del c.z
    m = Model(tables, Numerics(arithmetic=arith))
    m.stepper.adaptive_active = False
    rows, cols = c.boundary_cells()
    cells = np.array([m.cell_state_index(int(j), int(i)) for j, i in zip(rows, cols, strict=True)], np.int32)
    nb = cells.size
    m.set_boundary(BoundaryCells(cells, cells.copy(), np.ones(nb, np.int32), np.zeros(nb, np.float32),
                                 np.zeros(nb, np.float32)))  # fmt: skip
    m.set_depth(np.where(grid.mask, 0.05, 0.0))
    rate = peak_rate(c)
    m.set_source(np.where(grid.mask, rate, 0.0))
    # outflow faces of the outfall cells (east/south faces of the rim cells are their own west/north faces)
    maxima = Maxima(m, 0.1, 0.05, every=4)
    tally = Tally(m, cells.astype(np.int64), np.ones(nb), np.zeros(0, np.int64), np.zeros(0))
    return m, c, grid, tables, maxima, tally, rate


def peak_rate(c) -> np.ndarray:
    """Rain excess at the hyetograph's peak (2 D / T), less the constant loss, m/s, on the padded grid."""
    peak_mm_h = 2.0 * c.rain_mm / (c.storm_s / 3600.0)
    return np.maximum(peak_mm_h - c.constant_loss_mm_h, 0.0) / 3.6e6


def cut_block(c, grid) -> None:
    """Keep the CPU sample block's pixels, with the one-pixel rim the table builder reads, on the host
    (``c.block_z``)."""
    j0, i0, M = cpu_block(grid)
    c.block_z = c.z[j0 * c.k : (j0 + M) * c.k + 2, i0 * c.k : (i0 + M) * c.k + 2].double().cpu().numpy()


def cpu_block(grid) -> tuple[int, int, int]:
    """First row and column (padded cells) and side of the CPU sample: a 32 x 32-tile block from the middle of the
    grid, smaller on a grid of fewer than 33 tiles a side (a tile short of its side, so that the block's pixels with
    their rim lie inside the bed)."""
    nty, ntx = grid.tile_of.shape
    B = max(1, min(CPU_BLOCK_TILES, nty - 1, ntx - 1))
    return (nty - B) // 2 * 32, (ntx - B) // 2 * 32, B * 32


def block_inputs(c, grid, rate):
    """The CPU sample block as the reference's CPU path takes it: the oracle's grid of the block (every cell active but
    the outer ring, walls on its edge), its tables from the oracle's table builder (the reference's builder restated) on the block's
    own pixels (``c.block_z``, cut from the catchment's bed; faces at the block's edge see the block's pixels), and the
    source rates of the block's cells."""
    from oracle import oracle as O

    j0, i0, M = cpu_block(grid)
    # the reference's padded grid of the block (wadi2d/grid/tiles.py:52-64): its outer ring of cells inactive, so every
    # face at the block's edge is closed, as on any grid the reference builds
    og = O.Grid.from_mask(np.ones((M - 2, M - 2), bool), 0.0, 0.0, grid.dx)
    tables = O.build_tables(og, c.block_z, c.dx / c.k, c.manning, local_radius=True)
    return og, tables, rate[j0 : j0 + M, i0 : i0 + M]


def cpu_sample(block, seconds: float, threads: int, steps: int | None = None, warmup: int = 1):
    """The oracle on the CPU sample block (``block_inputs``), 0.05 m of water everywhere under the block's rates.
    Returns cell-steps/s on ``threads`` host threads over about ``seconds`` (or exactly ``steps``) of stepping, the
    steps, the seconds and the cells."""
    from oracle import oracle as O

    og, tables, rate = block
    O.threads(threads)
    m = O.Model(og, tables, O.Numerics())
    m.adaptive_active = False
    m.set_depth(np.full(og.mask.shape, 0.05))
    m.set_source(rate)
    cells = int(og.mask.sum())
    for _ in range(warmup):
        m.advance(m.t + m.dt * 0.999)
    n0, t0 = m.nsteps, time.perf_counter()
    while True:
        m.advance(m.t + m.dt * 0.999)
        done = m.nsteps - n0
        el = time.perf_counter() - t0
        if (steps is not None and done >= steps) or (steps is None and el >= seconds and done >= 3):
            break
    return cells * done / el, done, el, cells


class _Stop(Exception):
    pass


def _steps(model, n: int) -> None:
    """n steps of a model's host-driven loop (the reference's Stepper.advance, dt rule and refresh cadence)."""

    def cb(st):
        if st.nsteps >= n:
            raise _Stop

    try:
        model.advance(1e12, cb)
    except _Stop:
        pass


def block_parity(block, arith: str, steps: int, threads: int) -> dict:
    """The CUDA step against the oracle on the CPU sample block: the same tables (the oracle's), 0.05 m of water under
    the block's peak rain, ``steps`` steps of each's host-driven loop at the reference's dt rule, then the step's
    accuracy bounds: the dt sequence, the wet set (h > 0), depth within 1e-5 m or 1e-4 relative, unit discharge within
    1e-4 of its field's scale; and whether every state field is equal bit for bit."""
    from oracle import oracle as O
    from wadi2d_b200.config import Numerics
    from wadi2d_b200.grid import TileGrid
    from wadi2d_b200.model import Model
    from wadi2d_b200.tables import GridTables

    og, tables, rate = block
    O.threads(threads)
    ref = O.Model(og, tables, O.Numerics())
    ref.adaptive_active = False
    grid = TileGrid(og.x0, og.y0, og.dx, og.mask)
    m = Model(GridTables.from_dict(grid, tables), Numerics(arithmetic=arith))
    m.stepper.adaptive_active = False
    dts = []
    step = m.backend.step

    def logged(dt, want_wave, want_wet):
        dts.append(float(dt))
        step(dt, want_wave, want_wet)

    m.backend.step = logged
    for model in (ref, m):
        model.set_depth(np.full(og.mask.shape, 0.05))
        model.set_source(rate)
        _steps(model, steps)
    out = {"arith": arith, "steps": int(m.stepper.nsteps), "cells": int(og.mask.sum()),
           "dt_identical": dts == [float(x) for x in ref.dts],
           "dt_max_rel_diff": float(np.max(np.abs(np.array(dts) / np.array(ref.dts) - 1.0))) if dts else 0.0}  # fmt: skip
    f = {n: (m.field(n), ref.field(n)) for n in ("h", "d", "u", "v", "mx", "my", "qx", "qy", "res", "om")}
    out["bit_identical"] = all(np.array_equal(a, b) for a, b in f.values())
    h, hr = (x.astype(np.float64) for x in f["h"])
    diff = np.abs(h - hr)
    out["wet_set_identical"] = bool(np.array_equal(h > 0, hr > 0))
    out["depth_max_abs_err_m"] = float(diff.max())
    out["depth_within"] = bool(np.all((diff <= 1e-5) | (diff <= 1e-4 * np.abs(hr))))
    rel = {}
    for n in ("qx", "qy", "u", "v", "d"):
        a, b = (x.astype(np.float64) for x in f[n])
        rel[n] = float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-30))
    out["rel_to_scale"] = rel
    out["discharge_within"] = rel["qx"] <= 1e-4 and rel["qy"] <= 1e-4
    out["within_bounds"] = out["wet_set_identical"] and out["depth_within"] and out["discharge_within"]
    del m
    return out


def run_reference(args) -> None:
    """The reference arm: its CPU step (the oracle) on every host thread, on the bounded block."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import torch

    from wadi2d_b200 import workloads
    from wadi2d_b200.grid import TileGrid

    threads = os.cpu_count() or 1
    dev = torch.device("cuda", 0) if torch.cuda.is_available() else torch.device("cpu")
    c = workloads.catchment(n=args.n, device=dev)  # the seeded bed, generated with torch
    grid = TileGrid.from_mask(np.ones((args.n, args.n), bool), 0.0, 0.0, c.dx)
    cut_block(c, grid)
    del c.z
    block = block_inputs(c, grid, peak_rate(c))
    value, done, el, cells = cpu_sample(block, 0.0, threads, steps=args.steps, warmup=args.warmup)
    B = cpu_block(grid)[2] // 32
    sample = f"{B}x{B} tiles ({cells} cells) of the workload, {done} steps"
    line = {
        "impl": "reference", "metric": "cell-steps/s", "value": value, "unit": "cell-steps/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * el / max(done, 1),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded fractal catchment, lognormal storm)",
        "config": {"workload": f"configuration 3, {args.n}x{args.n} cells at 30 m, bounded CPU sample", "sample": sample},
        "cpu_baseline": {"value": value, "unit": "cell-steps/s", "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": "cell-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }  # fmt: skip
    print(json.dumps(line), flush=True)


def full_run(args) -> None:
    """Configuration 3 end to end: 36 h from dry ground, the lognormal storm over its 12 h triangular hyetograph with
    the initial-and-constant loss rated on the device each 30 s window, sleeping tiles on, the envelope every 4 steps,
    the FP64 outfall tally every step; the books as the reference's monitor keeps them."""
    import torch

    from wadi2d_b200 import forcing as F
    from wadi2d_b200 import workloads
    from wadi2d_b200.backend import BoundaryCells
    from wadi2d_b200.config import Numerics, Tables
    from wadi2d_b200.grid import TileGrid
    from wadi2d_b200.maxima import Maxima, Tally
    from wadi2d_b200.model import Model
    from wadi2d_b200.run import DeviceRain, DeviceStorage, run_windows
    from wadi2d_b200.state import state_index
    from wadi2d_b200.tables import ArrayBed, build_tables

    dev = torch.device("cuda", 0)
    t0 = time.perf_counter()
    c = workloads.catchment(n=args.n, device=dev)
    grid = TileGrid.from_mask(np.ones((args.n, args.n), bool), 0.0, 0.0, c.dx)
    tables = build_tables(grid, ArrayBed(c.z, c.dx / c.k), Tables(), c.manning, device=dev)
    del c.z
    m = Model(tables, Numerics(arithmetic=args.arith))
    rows, cols = c.boundary_cells()
    cells = state_index(grid, rows, cols).astype(np.int32)
    nb = cells.size
    m.set_boundary(BoundaryCells(cells, cells.copy(), np.ones(nb, np.int32), np.zeros(nb, np.float32),
                                 np.zeros(nb, np.float32)))  # fmt: skip
    taken = np.zeros(grid.shape, bool)
    taken[rows, cols] = True
    inner = grid.mask & ~taken
    jj, ii = np.nonzero(inner)
    interior = state_index(grid, jj, ii).astype(np.int64)
    (xf, xs), (yf, ys) = F.open_faces(grid, inner, taken)
    tally = Tally(m, xf, xs, yf, ys)
    maxima = Maxima(m, 0.1, 0.05, every=4)
    storm = F.TriangularStorm(1.0, c.storm_s / 60.0)
    rain = DeviceRain(m, storm, interior, multiplier=c.rain_mm[jj, ii],
                      loss=F.InitialConstantLoss(c.initial_loss_mm, c.constant_loss_mm_h))  # fmt: skip
    storage = DeviceStorage(m, interior)
    setup = time.perf_counter() - t0
    torch.cuda.synchronize(dev)
    w0 = time.perf_counter()
    t_end = min(c.t_end, args.sim_hours * 3600.0)
    out = run_windows(m, t_end, rain=rain, window=30.0, maxima=maxima, tally=tally, storage=storage)
    torch.cuda.synchronize(dev)
    wall = time.perf_counter() - w0
    b = out.balance
    env = maxima.fields()
    line = {
        "run": f"configuration 3, {t_end / 3600.0:g} h", "cells": args.n * args.n, "steps": out.steps, "windows": out.windows,
        "wall_s": wall, "setup_s": setup, "runs_per_h": 3600.0 / (wall + setup),
        "cell_steps_per_s": args.n * args.n * out.steps / wall,
        "rain_m3": b.rain, "outflow_m3": b.outflow, "storage_m3": b.storage, "mass_error": b.relative,
        "peak_depth_m": float(env["depth"].max()), "peak_speed_m_s": float(env["speed"].max()),
        "wet_cells_end": int((m.field("h") > 0).sum()),
    }  # fmt: skip
    print(json.dumps(line), flush=True)


def ensemble_inputs(spec, dev):
    """One run of configuration 4 on the GPU: fan, tables, outfalls, tally faces, rained interior cells."""
    from wadi2d_b200 import forcing as F
    from wadi2d_b200 import workloads
    from wadi2d_b200.backend import BoundaryCells
    from wadi2d_b200.config import Tables
    from wadi2d_b200.grid import TileGrid
    from wadi2d_b200.state import state_index
    from wadi2d_b200.tables import ArrayBed, build_tables

    n = spec.side
    c = workloads.catchment(n=n, dx=spec.dx, k=4, seed=spec.seed, relief=spec.relief, device=dev)
    grid = TileGrid.from_mask(np.ones((n, n), bool), 0.0, 0.0, spec.dx)
    tables = build_tables(grid, ArrayBed(c.z, spec.dx / 4), Tables(), c.manning, device=dev)
    del c.z
    rows, cols = c.boundary_cells()
    cells = state_index(grid, rows, cols).astype(np.int32)
    nb = cells.size
    bc = BoundaryCells(cells, cells.copy(), np.ones(nb, np.int32), np.zeros(nb, np.float32), np.zeros(nb, np.float32))
    taken = np.zeros(grid.shape, bool)
    taken[rows, cols] = True
    inner = grid.mask & ~taken
    jj, ii = np.nonzero(inner)
    (xf, xs), (yf, ys) = F.open_faces(grid, inner, taken)
    return grid, tables, bc, state_index(grid, jj, ii).astype(np.int64), (xf, xs, yf, ys)


def ensemble_run(args) -> None:
    """Configuration 4: 64 runs of uneven size, cell size and storm (uniform rain, each run its own depth, duration
    and ARF factor), each from dry ground to the end of its storm plus a recession, the envelope every 4 steps and
    the FP64 outfall tally every step. Timed twice: as one batch (w2b_advance_runs) and one run after another (the
    plain per-run device loop); both give every run the same steps and the same envelope. Under torchrun the runs
    are split over the ranks by estimated cell-steps (no exchange while they step); the times are CUDA events, the
    max over ranks, and rank 0 gathers the per-run records."""
    import torch
    import torch.distributed as dist

    from wadi2d_b200 import sweep, workloads
    from wadi2d_b200.batch import Batch
    from wadi2d_b200.config import Numerics
    from wadi2d_b200.maxima import Maxima, Tally
    from wadi2d_b200.model import Model
    from wadi2d_b200.run import DeviceRain, run_windows

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=900))
    specs = workloads.ensemble(args.runs, side_max=args.side_max)
    t_all = np.array([(sp.duration_min + args.recession_min) * 60.0 * args.time_scale for sp in specs])
    costs = [sweep.run_cost(sp.side**2, t_all[r], sp.dx) for r, sp in enumerate(specs)]
    mine = sweep.partition(costs, world)[rank]
    stream = torch.cuda.current_stream(dev)

    def timed(fn):
        """fn() between CUDA events on the current stream; the max over ranks, seconds."""
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize(dev)
        e0.record(stream)
        out = fn()
        e1.record(stream)
        torch.cuda.synchronize(dev)
        sec = e0.elapsed_time(e1) / 1e3
        if world > 1:
            t = torch.tensor([sec], device=dev, dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            sec = float(t.item())
        return out, sec

    t0 = time.perf_counter()
    inputs = [ensemble_inputs(specs[r], dev) for r in mine]
    torch.cuda.synchronize(dev)
    setup = time.perf_counter() - t0
    num = Numerics(arithmetic=args.arith)
    t_end = t_all[mine]
    storms = [specs[r].storm() for r in mine]
    cells = np.array([int(i[0].mask.sum()) for i in inputs], np.float64)
    records = {r: {"side": specs[r].side, "cells": int(cells[n]), "simulated_h": float(t_end[n]) / 3600.0}
               for n, r in enumerate(mine)}  # fmt: skip
    plain_s = None
    if not args.skip_plain:

        def plain_sweep():
            for n, (grid, tables, bc, interior, tspec) in enumerate(inputs):
                m = Model(tables, num)
                m.set_boundary(bc)
                m.set_depth(np.zeros(grid.shape))
                tally = Tally(m, *tspec)
                maxima = Maxima(m, 0.1, 0.05, every=4)
                rain = DeviceRain(m, storms[n], interior)
                run_windows(m, t_end[n], rain=rain, window=30.0, maxima=maxima, tally=tally)
                rec = records[mine[n]]
                rec["plain_steps"] = int(m.stepper.nsteps)
                rec["plain_peak_depth"] = float(maxima.fields()["depth"].max())
                del m, tally, maxima, rain

        _, plain_s = timed(plain_sweep)
    b0 = time.perf_counter()
    B = Batch([i[0] for i in inputs], [i[1] for i in inputs], num)
    B.set_boundary([i[2] for i in inputs])
    B.set_depth([np.zeros(i[0].shape) for i in inputs])
    B.set_tally([i[4] for i in inputs])
    B.reset_envelope()
    rc = [B.native_of(n, i[3]) for n, i in enumerate(inputs)]
    torch.cuda.synchronize(dev)
    pack_s = time.perf_counter() - b0
    books, batch_s = timed(lambda: B.run_windows(t_end, storms, window=30.0, max_every=4, cells=rc))
    for n, r in enumerate(mine):
        rec = records[r]
        rec["steps"] = int(B.nsteps[n])
        rec["peak_depth"] = float(B.envelope(n)["depth"].max())
        rec["rain_m3"] = books[n].rain
        rec["outflow_m3"] = books[n].outflow
    allrec = sweep.gather_results(records, world, rank)
    if rank == 0:
        recs = list(allrec.values())
        cs = float(sum(x["cells"] * x["steps"] for x in recs))
        line = {
            "run": "configuration 4 ensemble", "runs": len(recs), "n_gpus": world, "cells": int(sum(x["cells"] for x in recs)),
            "setup_s_rank0": setup, "pack_s_rank0": pack_s,
            "batch": {"s": batch_s, "runs_per_h": 3600.0 * len(recs) / batch_s, "cell_steps_per_s": cs / batch_s,
                      "tiles_rank0": int(B.grid.ntiles - 1), "loop_steps_rank0": int(B.nsteps.max())},
            "plain": None if plain_s is None else {"s": plain_s, "runs_per_h": 3600.0 * len(recs) / plain_s,
                                                   "cell_steps_per_s": cs / plain_s},
            "speedup": None if plain_s is None else plain_s / batch_s,
            "same_steps": None if plain_s is None else all(x["steps"] == x["plain_steps"] for x in recs),
            "same_peak_depth": None if plain_s is None else all(x["peak_depth"] == x["plain_peak_depth"] for x in recs),
            "rain_m3": float(sum(x["rain_m3"] for x in recs)), "outflow_m3": float(sum(x["outflow_m3"] for x in recs)),
            "imbalance": sweep.imbalance(costs, sweep.partition(costs, world)),
            "per_run": [[x["side"], round(x["simulated_h"], 3), x["steps"]] for x in recs],
        }  # fmt: skip
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def critical_search(n: int, candidates: int, train_runs: int, plain_sample: int, dx: float = 10.0,
                    relief: float | None = None, seed: int = 17, storm_seed: int = 5, iters: int = 3000,
                    arith: str = "exact") -> dict:
    """Configuration 5 on an n x n catchment at dx (relief by default 3 % of its length): which of ``candidates``
    storms (0.5-48 h log-uniform, 20-200 mm, ARF 0.6-1.0, patterns a seeded convex mix of 4 alternating-block
    hyetographs) gives the largest peak flow at the main design point. Three ways, timed with CUDA events: every
    candidate through the solver as batches (the exhaustive sweep), the network's screen (solver runs of
    ``train_runs`` candidates, training, ranking, solver runs of the top 5 %), and one solver run after another on a
    sample of ``plain_sample`` candidates, whose time per simulated hour gives the one-after-another sweep's runs/h.
    A non-learned screen (the same share ranked by peak block intensity, with the same training runs) shows what the
    network adds."""
    import torch

    from wadi2d_b200 import critical as C
    from wadi2d_b200.config import Numerics
    from wadi2d_b200.maxima import Lines, Tally
    from wadi2d_b200.model import Model
    from wadi2d_b200.run import DeviceRain, run_windows

    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream(dev)

    def timed(fn):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize(dev)
        e0.record(stream)
        out = fn()
        e1.record(stream)
        torch.cuda.synchronize(dev)
        return out, e0.elapsed_time(e1) / 1e3

    num = Numerics(arithmetic=arith)
    t0 = time.perf_counter()
    cat = C.prepare(n=n, dx=dx, k=4, seed=seed, relief=relief, device=dev)
    setup = time.perf_counter() - t0
    storms = C.candidates(candidates, seed=storm_seed)
    x = C.features(storms)
    rec = 1.0
    sim_h = np.array([s.duration_h + rec for s in storms])
    full, full_s = timed(lambda: C.solve(cat, storms, recession_h=rec, num=num))
    point = 0
    crit = int(np.argmax(full["peak_q"][:, point]))
    rng = np.random.default_rng(11)
    train = rng.choice(len(storms), size=train_runs, replace=False)
    res_tr, tr_s = timed(lambda: C.solve(cat, [storms[i] for i in train], recession_h=rec, num=num))
    y_tr = C.targets(res_tr)
    (order, pred, losses), fit_s = timed(lambda: C.screen(x[train], y_tr, x, top=0.05, point=point, iters=iters))
    rerun = [int(i) for i in order if i not in set(train.tolist())]
    res_rr, rr_s = timed(lambda: C.solve(cat, [storms[i] for i in rerun], recession_h=rec, num=num) if rerun else None)
    solved = {int(i): float(res_tr["peak_q"][k, point]) for k, i in enumerate(train)}
    for k, i in enumerate(rerun):
        solved[i] = float(res_rr["peak_q"][k, point])
    found = max(solved, key=solved.get)
    screen_s = tr_s + fit_s + rr_s
    # the same share ranked without the network: by the storm's peak block intensity (descriptor 9)
    k = len(order)
    by_intensity = np.argsort(x[:, 9])[::-1][:k]
    naive = set(by_intensity.tolist()) | set(train.tolist())
    naive_found = max(naive, key=lambda i: full["peak_q"][i, point])
    held = np.setdiff1d(np.arange(len(storms)), train)
    truth = np.log1p(full["peak_q"][held, point])
    r2 = 1.0 - np.mean((pred[held, point] - truth) ** 2) / np.var(truth)
    # one run after another, on a sample
    sample = rng.choice(len(storms), size=plain_sample, replace=False)

    def plain():
        out = []
        for i in sample:
            m = Model(cat.tables, num)
            m.set_boundary(cat.boundary)
            m.set_depth(np.zeros(cat.grid.shape))
            tally = Tally(m, *cat.tally)
            lines = Lines(m, [ln[:4] for ln in cat.lines])
            rain = DeviceRain(m, storms[i], cat.rained)
            run_windows(m, sim_h[i] * 3600.0, rain=rain, window=30.0, tally=tally)
            out.append(float(lines.peaks()[0][point]))
        return out

    plain_q, plain_s = timed(plain)
    same = all(plain_q[j] == full["peak_q"][i, point] for j, i in enumerate(sample))
    plain_per_h = plain_s / sim_h[sample].sum()  # seconds of one-after-another solving per simulated hour
    plain_sweep_s = plain_per_h * sim_h.sum()
    return {
        "run": "configuration 5 critical-duration search", "cells": n * n, "dx_m": dx, "relief_m": cat.relief,
        "arith": arith, "candidates": len(storms), "design_points": len(cat.lines), "train_runs": int(train_runs),
        "top": k, "rerun_top": len(rerun), "setup_s": setup,
        "critical_in_training_runs": bool(crit in set(train.tolist())),
        "exhaustive_batched": {"s": full_s, "runs_per_h": 3600.0 * len(storms) / full_s,
                               "critical": crit, "peak_q": float(full["peak_q"][crit, point]),
                               "duration_h": storms[crit].duration_h, "depth_mm": storms[crit].total_depth},
        "screened": {"s": screen_s, "solver_s": tr_s + rr_s, "train_s": fit_s,
                     "runs_per_h": 3600.0 * len(storms) / screen_s, "critical": found,
                     "peak_q": solved[found], "same_critical": found == crit,
                     "critical_in_top": bool(crit in set(order.tolist())),
                     "peak_q_error": solved[found] / float(full["peak_q"][crit, point]) - 1.0,
                     "held_out_r2_log_peak": float(r2), "loss_first_last": [losses[0], losses[-1]]},
        "intensity_screen": {"critical": int(naive_found), "same_critical": int(naive_found) == crit,
                             "critical_in_top": bool(crit in set(by_intensity.tolist())),
                             "peak_q_error": float(full["peak_q"][naive_found, point] / full["peak_q"][crit, point])
                             - 1.0},
        "plain_one_after_another": {"sample": len(sample), "s_sample": plain_s, "s_per_simulated_h": plain_per_h,
                                    "sweep_s_estimate": plain_sweep_s,
                                    "runs_per_h": 3600.0 * len(storms) / plain_sweep_s, "same_peaks_as_batch": same},
        "speedup_screened_vs_plain": plain_sweep_s / screen_s,
        "speedup_batched_vs_plain": plain_sweep_s / full_s,
    }  # fmt: skip


def critical_run(args) -> None:
    """``critical_search`` at the command line's sizes (256 x 256 cells by default; the configuration names 1024)."""
    n = args.n if args.n != 4096 else 256
    line = critical_search(n, args.candidates, args.train_runs, args.plain_sample, dx=args.critical_dx,
                           relief=args.critical_relief, arith=args.arith)  # fmt: skip
    print(json.dumps(line), flush=True)


def config2_run(args) -> None:
    """Configuration 2 end to end: 1024 x 1024 cells at 10 m, 10 x 10 pixels a cell (tables on the GPU), 40 breakline
    crests, Manning patches, the 200 x 50 m reservoir started 4 m above its downstream bed (its depths through
    hbar_at_level), three lumped inflows at the channel heads shared over their cells by depth each 30 s window
    (wadi2d/forcing.py:667-695, depths read from the device), a free outfall on the south edge; 6 h on the device loop
    with sleeping tiles, the envelope every 4 steps and the FP64 outfall tally every step; the books."""
    import torch

    from wadi2d_b200 import forcing as F
    from wadi2d_b200 import workloads
    from wadi2d_b200.backend import BoundaryCells
    from wadi2d_b200.config import Numerics, Tables
    from wadi2d_b200.grid import TileGrid
    from wadi2d_b200.maxima import Maxima, Tally
    from wadi2d_b200.model import Model
    from wadi2d_b200.run import DeviceInflow, DeviceStorage, run_windows
    from wadi2d_b200.state import state_index
    from wadi2d_b200.tables import ArrayBed, build_tables, hbar_at_level

    dev = torch.device("cuda", 0)
    t0 = time.perf_counter()
    n = 1024
    c = workloads.crest_valley(n=n)
    grid = TileGrid.from_mask(np.ones((n, n), bool), 0.0, 0.0, c.dx)
    tables = build_tables(grid, ArrayBed(torch.as_tensor(c.z, device=dev), c.dx / c.k), Tables(), c.manning,
                          crest=c.crest, device=dev)  # fmt: skip
    del c.z
    m = Model(tables, Numerics(arithmetic=args.arith))
    rows, cols = c.outfall
    cells = state_index(grid, rows, cols).astype(np.int32)
    nb = cells.size
    m.set_boundary(BoundaryCells(cells, cells.copy(), np.ones(nb, np.int32), np.zeros(nb, np.float32),
                                 np.zeros(nb, np.float32)))  # fmt: skip
    rr, rc, level = c.reservoir
    hc, dtab = grid.from_tiles(tables.hc), grid.from_tiles(tables.dtab)
    zmin = np.asarray(tables.zmin)
    h0 = np.zeros(grid.shape)
    h0[rr, rc] = hbar_at_level(np.full(rr.size, level), zmin[rr, rc], hc[rr, rc], dtab[rr, rc])
    m.set_depth(h0)
    taken = np.zeros(grid.shape, bool)
    taken[rows, cols] = True
    inner = grid.mask & ~taken
    jj, ii = np.nonzero(inner)
    interior = state_index(grid, jj, ii).astype(np.int64)
    (xf, xs), (yf, ys) = F.open_faces(grid, inner, taken)
    tally = Tally(m, xf, xs, yf, ys)
    maxima = Maxima(m, 0.1, 0.05, every=4)
    pos = {int(k): p for p, k in enumerate(interior)}
    injections = []
    for q, (ir, icol, low, times, flows) in enumerate(c.inflows):
        idx = state_index(grid, ir, icol).astype(np.int64)
        injections.append(F.Injection(f"inflow {q}", np.array([pos[int(k)] for k in idx]), idx, low, times, flows,
                                      0.1))  # fmt: skip
    storage = DeviceStorage(m, interior)
    if args.host_inflows:
        forcing = F.Forcing(interior, c.dx**2, injections=injections,
                            depth_reader=lambda inj: m.read_cells("d", inj.index))  # fmt: skip
        sources = {"host_forcing": forcing}
    else:
        sources = {"inflow": DeviceInflow(m, injections, c.dx**2)}
    setup = time.perf_counter() - t0
    torch.cuda.synchronize(dev)
    w0 = time.perf_counter()
    out = run_windows(m, c.t_end, window=30.0, maxima=maxima, tally=tally, storage=storage, **sources)
    torch.cuda.synchronize(dev)
    wall = time.perf_counter() - w0
    b = out.balance
    env = maxima.fields()
    qx, qy = m.field("qx"), m.field("qy")
    crest_x = np.isfinite(c.crest.xz) & grid.mask
    line = {
        "run": "configuration 2, 6 h", "cells": n * n, "steps": out.steps, "windows": out.windows, "wall_s": wall,
        "setup_s": setup, "cell_steps_per_s": n * n * out.steps / wall, "inflow_m3": b.inflow,
        "reservoir_m3": b.storage0, "outflow_m3": b.outflow, "storage_m3": b.storage, "mass_error": b.relative,
        "peak_depth_m": float(env["depth"].max()), "peak_speed_m_s": float(env["speed"].max()),
        "wet_cells_end": int((m.field("h") > 0).sum()), "crest_x_faces": int(crest_x.sum()),
        "crest_x_faces_flowing_end": int((crest_x & (qx != 0.0)).sum()),
    }  # fmt: skip
    print(json.dumps(line), flush=True)


def table_build(args) -> None:
    """The sub-grid tables built on the GPU (w2b_build_tables), timed with CUDA events: configuration 2 (1024 x 1024
    cells at 10 m, 10 x 10 pixels a cell, 40 breakline crests, Manning patches; face lines of 298 pixels for the
    local radius) and configuration 3 (4096 x 4096 at 30 m, 4 x 4 pixels; lines of 44 pixels)."""
    import torch

    from wadi2d_b200 import workloads
    from wadi2d_b200.config import Tables
    from wadi2d_b200.grid import TileGrid
    from wadi2d_b200.tables import ArrayBed, build_tables

    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream(dev)
    out = {}
    for name, make in (("configuration 2", lambda: workloads.crest_valley(n=1024)),
                       ("configuration 3", lambda: workloads.catchment(n=4096, device=dev))):  # fmt: skip
        g0 = time.perf_counter()
        c = make()
        gen = time.perf_counter() - g0
        n = c.n
        grid = TileGrid.from_mask(np.ones((n, n), bool), 0.0, 0.0, c.dx)
        crest = getattr(c, "crest", None)
        z = c.z if isinstance(c.z, torch.Tensor) else torch.as_tensor(c.z, device=dev)
        small = TileGrid.from_mask(np.ones((62, 62), bool), 0.0, 0.0, c.dx)  # a first build, for the kernels' set-up
        build_tables(small, ArrayBed(z[: 64 * c.k, : 64 * c.k], c.dx / c.k), Tables(), 0.035, device=dev)
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        tables = build_tables(grid, ArrayBed(z, c.dx / c.k), Tables(), c.manning, crest=crest, device=dev)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        ms = e0.elapsed_time(e1)
        out[name] = {"cells": n * n, "pixels_per_cell": c.k * c.k, "pixel_m": c.dx / c.k, "build_s": ms / 1e3,
                     "cells_per_s": n * n / (ms / 1e3), "generate_s": gen,
                     "rows": tables.rows}  # fmt: skip
        del tables, z, c
        torch.cuda.empty_cache()
    print(json.dumps({"run": "GPU table build", **out}), flush=True)


def arf_study(args) -> None:
    """The depth-area study (the reference's ``wadi2d arf``): configuration 5's catchment (a seeded fractal fan at
    10 m with 4 x 4 pixels, 8 design lines on its channels), six storm areas log-spaced from 0.1 to 30 km2, a uniform
    60 mm storm over 2 h read through an area-reduction table at each, 3 h from dry ground; all storm areas as one
    batch against one run after another, CUDA-event time around the runs."""
    import torch

    from wadi2d_b200 import critical as C
    from wadi2d_b200 import study as S
    from wadi2d_b200.forcing import ArfTable, UniformStorm

    t0 = time.perf_counter()
    cat = C.prepare(n=args.study_n, dx=10.0, k=4, seed=17)
    cell, line_a = S.drainage_km2(cat)
    areas = S.storm_areas(list(line_a), n_areas=6, area_min_km2=0.1, area_max_km2=30.0)
    torch.cuda.synchronize()
    setup = time.perf_counter() - t0
    arf = ArfTable(np.array([0.1, 1.0, 10.0, 100.0, 1000.0]), np.array([1.0, 0.95, 0.86, 0.72, 0.55]))
    storm = UniformStorm(60.0, 120.0, arf=arf)
    names = [f"line{n}" for n in range(len(cat.lines))]
    kw = dict(t_end=3 * 3600.0, window=30.0, every=4, kind="storm-centred")
    b = S.run_study(cat, storm, areas, names, list(line_a), cell, batched=True, **kw)
    p = S.run_study(cat, storm, areas, names, list(line_a), cell, batched=False, **kw)
    cells = int(cat.grid.mask.sum())
    n = len(areas)
    line = {
        "run": "ARF depth-area study", "cells": cells, "storm_areas_km2": [round(a, 4) for a in areas],
        "lines": len(cat.lines), "setup_s": setup,
        "batch": {"s": b.seconds, "runs_per_h": 3600.0 * n / b.seconds,
                  "cell_steps_per_s": float(cells * b.steps.sum() / b.seconds)},
        "plain": {"s": p.seconds, "runs_per_h": 3600.0 * n / p.seconds,
                  "cell_steps_per_s": float(cells * p.steps.sum() / p.seconds)},
        "speedup": p.seconds / b.seconds,
        "same_steps": bool(np.array_equal(b.steps, p.steps)),
        "same_table": b.table == p.table,
        "same_composites": all(np.array_equal(b.composite[k], p.composite[k]) for k in S.COMPOSITE_MAPS),
        "steps": [int(x) for x in b.steps],
        "table": [{k: (round(v, 4) if isinstance(v, float) else v) for k, v in r.items()
                   if k in ("design_point", "drainage_area_km2", "design_peak_m3s", "time_of_peak_s")}
                  for r in b.table],
        "composite_max": {k: float(v.max()) for k, v in b.composite.items()},
    }  # fmt: skip
    print(json.dumps(line), flush=True)


def main() -> None:
    args = parse()
    if args.impl == "reference":
        run_reference(args)
        return
    if args.full_run:
        full_run(args)
        return
    if args.ensemble:
        ensemble_run(args)
        return
    if args.critical:
        critical_run(args)
        return
    if args.table_build:
        table_build(args)
        return
    if args.config2_run:
        config2_run(args)
        return
    if args.arf_study:
        arf_study(args)
        return
    import torch
    import torch.distributed as dist

    from wadi2d_b200 import _lib

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
    m, c, grid, tables, maxima, tally, rate = build_workload(args.n, dev, args.arith)
    b = m.backend
    cells = args.n * args.n
    tile_cells = (grid.ntiles - 1) * 1024
    stream = torch.cuda.current_stream(dev)

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize(dev)

    # warm-up: the graph capture and the first steps; then the launch tuner settles (its candidate schedules give the
    # same bits and differ only in time), so the timed steps run the schedule it kept
    if args.form != "tuned":
        lc = b.loop_config()
        strips = {"tiles": 0, "strips16": 16, "strips8": 8}[args.form]
        occ = {0: lc["faces_occupancy"], 16: lc["strips16_occupancy"], 8: lc["strips8_occupancy"]}[strips]
        b.set_loop(False, occ, lc["update_occupancy"], 16, strips)
    m.run(1e12, maxima=maxima, tally=tally, max_steps=max(args.warmup, 3))
    tune_steps = 0
    while b.loop_config()["tuning"] and tune_steps < 4096:
        m.run(1e12, maxima=maxima, tally=tally, max_steps=64)
        tune_steps += 64
    barrier()
    phys = os.environ.get("CUDA_VISIBLE_DEVICES", "").split(",")
    clocks = Clocks(int(phys[local]) if len(phys) > local and phys[local].strip().isdigit() else local)
    clocks.start()
    time.sleep(0.4)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    n0 = m.stepper.nsteps
    e0.record(stream)
    m.run(1e12, maxima=maxima, tally=tally, max_steps=args.steps)
    e1.record(stream)
    barrier()
    clk = clocks.stop()
    ran = m.stepper.nsteps - n0
    ms = e0.elapsed_time(e1)
    if world > 1:
        t = torch.tensor([ms], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    value = world * cells * ran / (ms / 1e3)

    # the face pass on its own, CUDA events on its stream (the same state, continuing)
    import ctypes

    times = (ctypes.c_float * 3)()
    faces_ms, update_ms = [], []
    for s in range(16):
        want_wave = s % 8 == 0
        dt = float(np.float32(m.stepper.dt))
        _lib.call("w2b_step_timed", b.handle, dt, int(want_wave), 0, stream.cuda_stream, times)
        faces_ms.append(times[0])
        update_ms.append(times[1])
    faces = statistics.mean(faces_ms)
    hbm, peak_kind = peaks()
    achieved = ALG_FACES * tile_cells / (faces / 1e3) / 1e9
    traffic = FACES_DRAM_BYTES_PER_CELL * tile_cells
    form = b.loop_config()["strips"]
    kernel = f"{args.arith}::strips_kernel<{form}>" if form else f"{args.arith}::faces_kernel"
    roofline = {"kernel": kernel, "bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                "frac": achieved / hbm, "peak_kind": peak_kind, "traffic": traffic,
                # the DRAM bytes the launch moves (traffic, from the capture) over its time, against the same peak
                "traffic_frac": traffic / (faces / 1e3) / 1e9 / hbm,
                "alg_bytes_per_cell": ALG_FACES, "impl_bytes_per_cell": IMPL_FACES, "launch_ms": faces,
                "update_kernel_ms": statistics.mean(update_ms),
                "step_alg_bytes_per_cell": ALG_STEP, "step_impl_bytes_per_cell": IMPL_STEP,
                "step_frac": (cells * ran / (ms / 1e3)) * ALG_STEP / 1e9 / hbm}  # fmt: skip

    # end to end through the C-ABI with host buffers, as the reference's run driver and monitor take a run: per 30 s
    # window the window's rain from pinned memory (uploaded on a side stream while the window before steps, then put
    # in place by a device copy: run.SourceStager), the window stepped, then what the monitor reads each window (the
    # clock and the active list, the design line's discharge, the outfall volume, the FP64 storage); at the end the
    # five envelope maps
    from wadi2d_b200.maxima import Lines, faces_across
    from wadi2d_b200.run import DeviceStorage, MonitorReads, SourceStager
    from wadi2d_b200.state import state_index

    rows, cols = c.boundary_cells()
    main = rows == rows.max()
    line = Lines(m, [faces_across(grid, rows[main], cols[main], axis=0)])  # the main outfall's row, southward
    jj, ii = np.nonzero(grid.mask)
    storage = DeviceStorage(m, np.asarray(state_index(grid, jj, ii), np.int64))
    del jj, ii
    src_native = b.native("src").cpu().pin_memory()
    stager = SourceStager(m)
    env_host = [torch.empty(a.shape, dtype=a.dtype).pin_memory() for a in maxima.arrays]  # the maps' host buffers
    win = 30.0
    h2d = d2h = 0
    # the monitor's reads once before the timed region, as the steps are warmed: their kernels' first launches (about
    # 20 ms, once a process) belong to a run's set-up, not to each of its thousands of windows
    monitor = MonitorReads(m, line, tally, storage)  # the three reads behind one synchronisation
    monitor()
    torch.cuda.synchronize(dev)
    w0 = time.perf_counter()
    s0 = m.stepper.nsteps
    series = []
    if args.e2e_windows:
        h2d += stager.stage(src_native)  # the first window's rates
    for w in range(args.e2e_windows):
        stager.commit()
        if w + 1 < args.e2e_windows:
            h2d += stager.stage(src_native)  # the next window's, crossing while this one steps
        m.run(m.stepper.t + win, maxima=maxima, tally=tally)
        d2h += ctypes.sizeof(_lib.Clock) + 4 * (int(b.nact) + grid.ntiles)  # the clock, the active list, idle counts
        q, outflow, stored = monitor()
        series.append((m.stepper.t, float(q[0]), outflow, stored))
        d2h += monitor.host.numel() * 8
    for dst, a in zip(env_host, maxima.arrays, strict=True):
        dst.copy_(a, non_blocking=True)
    d2h += sum(a.numel() * a.element_size() for a in env_host)
    torch.cuda.synchronize(dev)
    e2e_s = time.perf_counter() - w0
    e2e_steps = m.stepper.nsteps - s0
    e2e = {"value": world * cells * e2e_steps / e2e_s, "unit": "cell-steps/s",
           "h2d_bytes_per_step": h2d / max(e2e_steps, 1), "d2h_bytes_per_step": d2h / max(e2e_steps, 1),
           "windows": args.e2e_windows, "steps": e2e_steps,
           "upload": "each window's rain from pinned host memory on a side stream while the window before steps, "
                     "then a device copy into place (run.SourceStager)",
           "read_back": "per window: clock, active list, design-line discharge, outfall volume, storage; at the end: "
                        "the five envelope maps",
           "last_window": {"t_s": series[-1][0], "line_q_m3s": series[-1][1], "outflow_m3": series[-1][2],
                           "storage_m3": series[-1][3]} if series else None}  # fmt: skip
    del env_host

    wet_fraction = float((m.field("h") > 0).sum()) / cells
    launch = b.loop_config()
    cfl = m.num.cfl
    memory_gb = torch.cuda.memory_allocated(dev) / 1e9
    cpu = parity = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        block = block_inputs(c, grid, rate)
        if args.parity_steps > 0:
            parity = block_parity(block, args.arith, args.parity_steps, threads)
        cv, done, el, ccells = cpu_sample(block, args.cpu_seconds, threads)
        B = cpu_block(grid)[2] // 32
        cpu = {"value": cv, "unit": "cell-steps/s", "cores": threads, "kind": "port",
               "sample": f"{B}x{B} tiles ({ccells} cells) of the workload, {done} steps in {el:.1f} s"}  # fmt: skip
    sweep = None
    if rank == 0 and world == 1 and not args.no_sweep:
        # the other half of the metric, bounded: the critical-duration storm sweep at 128 x 128 cells, 100 candidates
        del m, b, maxima, tally, tables
        torch.cuda.empty_cache()
        try:
            r = critical_search(128, 100, 32, 4, iters=1500, arith=args.arith)
            sweep = {"workload": f"configuration 5 reduced: {r['cells']} cells at {r['dx_m']} m, {r['candidates']} "
                                 f"candidate storms, {r['train_runs']} training runs, top {r['top']} re-run",
                     "runs_per_h": {"screened": r["screened"]["runs_per_h"],
                                    "exhaustive_batched": r["exhaustive_batched"]["runs_per_h"],
                                    "plain_one_after_another": r["plain_one_after_another"]["runs_per_h"]},
                     "speedup_screened_vs_plain": r["speedup_screened_vs_plain"],
                     "same_critical": r["screened"]["same_critical"],
                     "peak_q_error": r["screened"]["peak_q_error"],
                     "critical_in_network_top": r["screened"]["critical_in_top"],
                     "critical_in_intensity_top": r["intensity_screen"]["critical_in_top"],
                     "same_peaks_one_after_another": r["plain_one_after_another"]["same_peaks_as_batch"]}  # fmt: skip
        except Exception as exc:  # the sweep is reported, never the reason the line is missing
            sweep = {"error": f"{type(exc).__name__}: {exc}"}
    if world > 1:
        dist.barrier()
    if rank == 0:
        wet = wet_fraction
        line = {
            "metric": "cell-steps/s", "value": value, "unit": "cell-steps/s", "n_gpus": world, "steps": ran,
            "warmup": args.warmup, "ms_per_step": ms / ran, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded fractal catchment, lognormal storm)",
            "config": {"workload": f"configuration 3: {args.n}x{args.n} cells at 30 m, 4x4 pixels, wet start under peak "
                                   "rain, every tile stepped, envelope every 4 steps, FP64 tally every step",
                       "cells": cells, "tiles": grid.ntiles - 1, "wet_fraction": wet, "cfl": cfl,
                       "l2": f"inputs larger than L2 ({memory_gb:.1f} GB resident)",
                       "parallelism": f"replicas x{world}",
                       "arith": args.arith, "loop": "device-resident, CUDA graphs", "launch": launch,
                       "tuning_steps": tune_steps},
            "roofline": roofline, "cpu_baseline": cpu, "parity": parity, "e2e": e2e, "sweep": sweep, "clocks": clk,
            # the device loop's launches: the work list and the first step's settings, then graphs of 16 steps of
            # six kernels (faces, update, envelope, boundary, control, plan)
            "gpu_launches": 2 + 6 * launch["steps_per_graph"] * -(-ran // launch["steps_per_graph"]),
        }  # fmt: skip
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
