"""The critical-duration search with a learned screen (configuration 5): which storm of a candidate set gives the
largest peak flow at a catchment's design points.

- Candidate storms: durations, depths and areal reduction factors drawn as the configuration says, each with a
  temporal pattern that is a seeded convex mix of four alternating-block hyetographs. A storm's cumulative depth is a
  percent graph interpolated linearly in time, as the reference's hypothetical storm (wadi2d/storm/hypothetical.py:
  24-62) reads one; here the interpolation is written out so that the batched form is the same arithmetic.
- The solver: every run is this package's step on the same catchment, as a batch (``Batch``: one run per storm, the
  catchment's tables copied into each), the design lines' peak discharge and its time taken on the device every step.
- The screen: the network of ``surrogate.Network`` maps a storm's 16 descriptors to the peak flow and time to peak at
  the 8 design points. It is trained on solver runs of a sample of the candidates, ranks all of them, and only the
  top-ranked ones get solver runs; every reported design value comes from the solver.
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

N_BLOCKS = 48
PEAK_AT = (0.2, 0.4, 0.6, 0.8)
"""Where the largest block of each base pattern sits, as a share of the storm."""


def alternating_block(n: int = N_BLOCKS, peak_at: float = 0.5, b: float = 0.1, c: float = 0.7) -> np.ndarray:
    """The cumulative share of depth at the n + 1 block edges of an alternating-block hyetograph: the depth of the
    most intense k blocks follows a dimensionless intensity-duration curve, P(k) = (k / n) (k / n + b)^-c; the block
    increments, largest first, go to the peak block and then alternately after and before it."""
    k = np.arange(n + 1) / n
    P = k * (k + b) ** (-c)
    inc = np.sort(np.diff(P))[::-1]
    p = int(round(peak_at * (n - 1)))
    order = [p]
    lo, hi = p - 1, p + 1
    while len(order) < n:
        if hi < n:
            order.append(hi)
            hi += 1
        if lo >= 0 and len(order) < n:
            order.append(lo)
            lo -= 1
    blocks = np.zeros(n)
    blocks[order] = inc
    F = np.concatenate(([0.0], np.cumsum(blocks)))
    return F / F[-1]


BASE = np.stack([alternating_block(peak_at=r) for r in PEAK_AT])


@dataclass
class MixedStorm:
    """``depth_mm`` reduced by ``arf`` over ``duration_h``, its cumulative share a convex mix of the base patterns."""

    depth_mm: float
    duration_h: float
    arf: float
    weights: np.ndarray
    F: np.ndarray = field(init=False, repr=False)

    def __post_init__(self) -> None:
        self.weights = np.asarray(self.weights, np.float64)
        self.F = self.weights @ BASE

    @property
    def total_depth(self) -> float:
        return self.depth_mm * self.arf

    def cumulative_depth(self, minutes) -> np.ndarray:
        """Depth fallen by each time, mm."""
        m = np.asarray(minutes, np.float64)
        return cumulative(np.full(m.shape, self.total_depth), np.full(m.shape, self.duration_h),
                          np.broadcast_to(self.F, m.shape + self.F.shape), m)  # fmt: skip

    @staticmethod
    def stack(storms: list[MixedStorm]) -> tuple:
        """The arrays of ``cumulative_many`` for a list of storms."""
        return (np.array([s.total_depth for s in storms]), np.array([s.duration_h for s in storms]),
                np.stack([s.F for s in storms]))  # fmt: skip

    @staticmethod
    def cumulative_many(stacked: tuple, minutes) -> np.ndarray:
        """Each storm's depth fallen by its own time (one a storm), mm: element for element cumulative_depth."""
        total, duration_h, F = stacked
        return cumulative(total, duration_h, F, minutes)


def cumulative(total, duration_h, F, minutes) -> np.ndarray:
    """Depth fallen by ``minutes`` (any shape; F has one more axis, the n + 1 block edges), mm: the percent graph
    interpolated linearly between block edges, zero before and the whole depth after."""
    n = F.shape[-1] - 1
    u = np.clip(np.asarray(minutes, np.float64) / (duration_h * 60.0), 0.0, 1.0) * n
    j = np.minimum(np.floor(u).astype(np.int64), n - 1)
    f = u - j
    f0 = np.take_along_axis(F, j[..., None], axis=-1)[..., 0]
    f1 = np.take_along_axis(F, (j + 1)[..., None], axis=-1)[..., 0]
    return total * (f0 + f * (f1 - f0))


def candidates(n: int, seed: int = 5, hours=(0.5, 48.0), depth=(20.0, 200.0), arf=(0.6, 1.0)) -> list[MixedStorm]:
    """n storms: durations log-uniform, depths and ARF factors uniform, pattern weights from a flat Dirichlet."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        d = float(np.exp(rng.uniform(np.log(hours[0]), np.log(hours[1]))))
        out.append(MixedStorm(float(rng.uniform(*depth)), d, float(rng.uniform(*arf)), rng.dirichlet(np.ones(4))))
    return out


def features(storms: list[MixedStorm]) -> np.ndarray:
    """16 descriptors a storm: log duration, depth, ARF, the four pattern weights, the reduced depth, log mean and
    log peak block intensity, where the peak block sits, the share fallen by a quarter, half and three quarters of the
    storm, 1 / duration, and the reduced depth over the square root of the duration."""
    rows = []
    for s in storms:
        blocks = np.diff(s.F)
        n = blocks.size
        dt_h = s.duration_h / n
        total = s.total_depth
        rows.append([
            np.log(s.duration_h), s.depth_mm / 100.0, s.arf, *s.weights, total / 100.0,
            np.log(total / s.duration_h), np.log(total * blocks.max() / dt_h), (np.argmax(blocks) + 0.5) / n,
            s.F[n // 4], s.F[n // 2], s.F[3 * n // 4], 1.0 / s.duration_h, total / 100.0 / np.sqrt(s.duration_h),
        ])  # fmt: skip
    return np.asarray(rows, np.float64)


# ------------------------------------------------------------------------------------------------ design points


def flow_accumulation(zmin: np.ndarray, mask: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """D8 contributing cells of every cell of a bed (cells processed from high to low), and each cell's steepest
    downhill step (dj, di)."""
    ny, nx = zmin.shape
    z = np.where(mask, zmin, np.inf)
    best = np.zeros((ny, nx))
    step = np.zeros((ny, nx, 2), np.int64)
    for dj in (-1, 0, 1):
        for di in (-1, 0, 1):
            if dj == 0 and di == 0:
                continue
            zn = _shift(z, dj, di)
            with np.errstate(invalid="ignore"):  # inf - inf off the mask: no slope
                slope = (z - zn) / np.hypot(dj, di)
            better = slope > best
            best = np.where(better, slope, best)
            step[better] = (dj, di)
    acc = np.where(mask, 1.0, 0.0)
    order = np.argsort(np.where(mask, zmin, -np.inf), axis=None)[::-1]
    jj, ii = np.unravel_index(order, (ny, nx))
    for j, i in zip(jj, ii, strict=True):
        if not mask[j, i]:
            continue
        dj, di = step[j, i]
        if dj == 0 and di == 0:
            continue
        acc[j + dj, i + di] += acc[j, i]
    return acc, step


def _shift(z: np.ndarray, dj: int, di: int) -> np.ndarray:
    """z[j + dj, i + di] at (j, i), inf past the edge."""
    ny, nx = z.shape
    out = np.full((ny, nx), np.inf)
    out[max(0, -dj) : ny - max(0, dj), max(0, -di) : nx - max(0, di)] = z[max(0, dj) : ny + min(0, dj),
                                                                         max(0, di) : nx + min(0, di)]  # fmt: skip
    return out


def design_lines(grid, zmin: np.ndarray, n: int = 8, half: int = 6, spacing: int = 24, edge: int = 8) -> list:
    """n design lines across the flow at the cells of largest contributing area, at least ``spacing`` cells apart
    and ``edge`` cells from the grid's rim: a line of 2 half + 1 north faces (flow mostly north-south; southward
    positive) or west faces (flow mostly east-west; eastward positive) centred on the cell, as
    (xfaces, xsign, yfaces, ysign, (j, i))."""
    from wadi2d_b200.maxima import faces_across

    acc, step = flow_accumulation(zmin, grid.mask)
    ny, nx = grid.shape
    order = np.argsort(acc, axis=None)[::-1]
    picked: list[tuple[int, int]] = []
    for flat in order:
        j, i = divmod(int(flat), nx)
        if not (edge <= j < ny - edge and edge <= i < nx - edge) or not grid.mask[j, i]:
            continue
        if any(max(abs(j - a), abs(i - b)) < spacing for a, b in picked):
            continue
        picked.append((j, i))
        if len(picked) == n:
            break
    lines = []
    for j, i in picked:
        dj, di = step[j, i]
        if abs(dj) >= abs(di):  # north-south flow: a row of north faces
            sgn = 1.0 if dj >= 0 else -1.0
            xf, xs, yf, ys = faces_across(grid, np.full(2 * half + 1, j + (1 if dj > 0 else 0)),
                                          np.arange(i - half, i + half + 1), axis=0, sign=sgn)  # fmt: skip
        else:
            sgn = 1.0 if di >= 0 else -1.0
            xf, xs, yf, ys = faces_across(grid, np.arange(j - half, j + half + 1),
                                          np.full(2 * half + 1, i + (1 if di > 0 else 0)), axis=1, sign=sgn)  # fmt: skip
        lines.append((xf, xs, yf, ys, (j, i)))
    return lines


# ------------------------------------------------------------------------------------------------ solver runs


@dataclass
class Catchment5:
    """A catchment ready for storm runs: grid, device tables, outfall cells, outfall tally faces, the rained cells
    (reference state indices), and the design lines."""

    grid: object
    tables: object
    boundary: object
    tally: tuple
    rained: np.ndarray
    lines: list
    relief: float = 0.0


def prepare(n: int = 256, dx: float = 10.0, k: int = 4, seed: int = 17, relief: float | None = None,
            device="cuda") -> Catchment5:  # fmt: skip
    """Configuration 5's catchment at n x n cells: a seeded fractal fan (``workloads.catchment``), its tables on the
    device, free outfalls, and 8 design lines on its channels."""
    from wadi2d_b200 import forcing as F
    from wadi2d_b200 import workloads
    from wadi2d_b200.backend import BoundaryCells
    from wadi2d_b200.config import Tables
    from wadi2d_b200.grid import TileGrid
    from wadi2d_b200.state import state_index
    from wadi2d_b200.tables import ArrayBed, build_tables

    relief = relief if relief is not None else 0.03 * n * dx
    c = workloads.catchment(n=n, dx=dx, k=k, seed=seed, relief=relief, device=device)
    grid = TileGrid.from_mask(np.ones((n, n), bool), 0.0, 0.0, dx)
    tables = build_tables(grid, ArrayBed(c.z, dx / k), Tables(), c.manning, device=device)
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
    zmin = np.asarray(tables.zmin)
    lines = design_lines(grid, zmin)
    return Catchment5(grid, tables, bc, (xf, xs, yf, ys), state_index(grid, jj, ii).astype(np.int64), lines, relief)


def solve(cat: Catchment5, storms: list[MixedStorm], recession_h: float = 1.0, batch: int = 256, num=None) -> dict:
    """Every storm through the solver, ``batch`` runs at a time, each to the end of its storm plus ``recession_h``:
    the design lines' peak discharge (m3/s) and the time of the peak (h), (runs x lines) each, and the steps."""
    from wadi2d_b200.batch import Batch
    from wadi2d_b200.config import Numerics

    num = num or Numerics()
    nl = len(cat.lines)
    q = np.zeros((len(storms), nl))
    tp = np.zeros((len(storms), nl))
    steps = np.zeros(len(storms), np.int64)
    # batches of storms of like length: a batch steps until its longest run ends
    by_length = np.argsort([s.duration_h for s in storms], kind="stable")
    for s0 in range(0, len(storms), batch):
        idx = by_length[s0 : s0 + batch]
        part = [storms[i] for i in idx]
        n = len(part)
        B = Batch([cat.grid] * n, [cat.tables] * n, num)
        B.set_boundary([cat.boundary] * n)
        B.set_depth([np.zeros(cat.grid.shape)] * n)
        B.set_tally([cat.tally] * n)
        B.set_lines([[ln[:4] for ln in cat.lines]] * n)
        cells = [B.native_of(r, cat.rained) for r in range(n)]
        t_end = np.array([(s.duration_h + recession_h) * 3600.0 for s in part])
        B.run_windows(t_end, part, window=30.0, cells=cells)
        for r in range(n):
            pk, tt = B.line_peaks(r)
            q[idx[r]], tp[idx[r]] = pk, tt / 3600.0
        steps[idx] = B.nsteps
        del B
    return {"peak_q": q, "t_peak_h": tp, "steps": steps}


def targets(res: dict) -> np.ndarray:
    """The network's 16 outputs a run: log(1 + peak Q) and the time to peak, h, at each of the 8 points."""
    return np.concatenate((np.log1p(res["peak_q"]), res["t_peak_h"]), axis=1)


def screen(x_train, y_train, x_all, top: float = 0.05, point: int = 0, iters: int = 3000, seed: int = 0):
    """Train the network on (x_train, y_train) and rank every candidate by its predicted peak at design point
    ``point``; returns the indices of the top share, largest first, the predictions and the loss history."""
    from wadi2d_b200.surrogate import DIMS, Network, Scaler

    sx, sy = Scaler.fit(x_train), Scaler.fit(y_train)
    nout = y_train.shape[1]
    width = (nout + 15) // 16 * 16  # the network's outputs: the targets, padded with zero columns
    yt = np.zeros((len(y_train), width))
    yt[:, :nout] = sy.to(y_train)
    net = Network(dims=DIMS[:-1] + (width,), seed=seed, lr=1e-3)
    losses = net.fit(sx.to(x_train), yt, iters=iters, batch=min(256, len(x_train)), seed=seed)
    pred = sy.back(net.predict(sx.to(x_all))[:, :nout])
    k = max(1, int(np.ceil(top * len(x_all))))
    order = np.argsort(pred[:, point])[::-1][:k]
    return order, pred, losses
