"""Seeded synthetic inputs for the benchmark configurations and the parity tests.

No dataset is read: every DEM, rain field and hydrograph here is generated from a seed, with the shapes, sizes and
value distributions the configurations name. Pixels are laid out on the padded grid of
``wadi2d_b200.grid.TileGrid.from_mask`` (one cell of margin north and west), pixel (r, c) centred at
``x0 + (c + 0.5) p``, ``y0 - (r + 0.5) p``, as the reference's tests build their beds
(tests/solver/test_subgrid.py:19-22).
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np


def fractal_noise(shape: tuple[int, int], hurst: float, sigma: float, seed: int) -> np.ndarray:
    """Spectral synthesis of a fractional Brownian surface: white noise shaped by |k|^-(H+1), std ``sigma``."""
    rng = np.random.default_rng(seed)
    ny, nx = shape
    white = rng.standard_normal((ny, nx))
    ky = np.fft.fftfreq(ny)[:, None]
    kx = np.fft.rfftfreq(nx)[None, :]
    k = np.sqrt(kx * kx + ky * ky)
    k[0, 0] = 1.0
    amp = k ** (-(hurst + 1.0))
    amp[0, 0] = 0.0
    field = np.fft.irfft2(np.fft.rfft2(white) * amp, s=(ny, nx))
    field -= field.mean()
    std = field.std()
    return field * (sigma / std) if std > 0 else field


@dataclass
class Plain:
    """A single run's inputs on a padded grid: DEM pixels, Manning, rain rate and the outfall cells."""

    ny: int
    nx: int
    dx: float
    k: int
    z: np.ndarray
    manning: float | np.ndarray
    rain_mm_h: float
    rain_s: float
    t_end: float
    cfl: float
    outfall: tuple[np.ndarray, np.ndarray]
    """Grid (row, column) of the free-outfall cells, padded coordinates."""


def v_channel_plane(n: int = 256, dx: float = 10.0, k: int = 5, seed: int = 0) -> Plain:
    """Configuration 1 at any size: n x n cells at ``dx`` with k x k pixels; a plane falling 1 % eastward, a
    V-channel 40 m wide and 1.5 m deep down the centreline, fractal noise (Hurst 0.8, sigma 0.3 m); Manning 0.035;
    50 mm/h of rain for 1 h; a free outfall on the east edge; 2 h at CFL 0.9."""
    pad = 32 * int(np.ceil((n + 2) / 32))
    p = dx / k
    npx = pad * k
    x = (np.arange(npx) + 0.5) * p - dx  # the padded origin lies one cell west of the domain
    y = (np.arange(npx) + 0.5) * p - dx
    X, Y = np.meshgrid(x, y)
    length = n * dx
    z = 100.0 + 0.01 * (length - X)
    yc = 0.5 * n * dx
    z -= 1.5 * np.maximum(0.0, 1.0 - np.abs(Y - yc) / 20.0)
    z += fractal_noise(z.shape, 0.8, 0.3, seed)
    rows = np.arange(1, 1 + n)
    return Plain(
        n, n, dx, k, z, 0.035, 50.0, 3600.0, 7200.0, 0.9, (rows, np.full(n, n, dtype=np.int64)),
    )  # fmt: skip


def rough_dam_break_bed(nx: int, ny: int, k: int, dx: float, seed: int = 3) -> np.ndarray:
    """Smoothed Gaussian relief 30 m about 200 m, the reference's rough dam-break bed
    (tests/solver/test_subgrid.py:95-103), on the padded grid of an ny x nx domain."""
    from scipy.ndimage import gaussian_filter

    rng = np.random.default_rng(seed)
    pny = 32 * int(np.ceil((ny + 2) / 32))
    pnx = 32 * int(np.ceil((nx + 2) / 32))
    return gaussian_filter(rng.normal(0, 1.0, (pny * k + 2, pnx * k + 2)), 5) * 30 + 200.0


@dataclass
class Catchment:
    """Configuration 3's inputs on a padded grid. ``z`` is a float64 tensor of pixels (on the generating device)."""

    n: int
    dx: float
    k: int
    z: object
    manning: float
    outfalls: list
    """(rows, columns) of each free outfall's cells, padded coordinates."""
    rain_mm: np.ndarray
    """(ny, nx) storm depth per cell, mm: a lognormal field on 1 km pixels (0 off the domain)."""
    storm_s: float
    t_end: float
    initial_loss_mm: float
    constant_loss_mm_h: float

    def boundary_cells(self) -> tuple[np.ndarray, np.ndarray]:
        rows = np.concatenate([r for r, _ in self.outfalls])
        cols = np.concatenate([c for _, c in self.outfalls])
        return rows, cols


def _fractal_torch(shape, hurst, gen_seed, device):
    import torch

    g = torch.Generator(device="cpu").manual_seed(int(gen_seed))
    white = torch.randn(shape, generator=g, dtype=torch.float32).to(device)
    ny, nx = shape
    ky = torch.fft.fftfreq(ny, device=device)[:, None]
    kx = torch.fft.rfftfreq(nx, device=device)[None, :]
    kk = torch.sqrt(kx * kx + ky * ky)
    kk[0, 0] = 1.0
    amp = kk ** (-(hurst + 1.0))
    amp[0, 0] = 0.0
    f = torch.fft.irfft2(torch.fft.rfft2(white) * amp, s=(ny, nx))
    f = f - f.mean()
    return (f / f.std()).to(torch.float64)


def catchment(n: int = 4096, dx: float = 30.0, k: int = 4, seed: int = 7, relief: float = 1500.0,
              device=None) -> Catchment:  # fmt: skip
    """Configuration 3: an n x n fractal catchment at ``dx`` (k x k pixels a cell) draining south to an alluvial fan,
    hydrologically conditioned (every cell drains to an outfall), with 5 free outfalls on its rim; a 1 km lognormal
    storm (mean 60 mm, CV 0.5) over a 12 h triangular hyetograph, 24 h of recession (36 h), initial loss 10 mm and
    constant loss 2 mm/h."""
    import torch
    import torch.nn.functional as F

    dev = torch.device(device if device is not None else ("cuda" if torch.cuda.is_available() else "cpu"))
    pad = 32 * int(np.ceil((n + 2) / 32))
    L = n * dx
    c = (torch.arange(pad, device=dev, dtype=torch.float64) - 1 + 0.5) * dx
    Y, X = torch.meshgrid(c, c, indexing="ij")  # y grows south
    xo, yo = 0.5 * L, L
    r = torch.sqrt((X - xo) ** 2 + (Y - yo) ** 2) / L
    base = relief * (0.55 * r**1.2 + 0.12 * torch.abs(X - xo) / L + 0.05 * (1.0 - Y / L))
    smooth = torch.clamp((r - 0.08) / 0.12, 0.0, 1.0)  # the fan near the outlet is smooth
    fan = 45.0 * torch.clamp(1.0 - r / 0.15, min=0.0)
    zc = base + fan + smooth * (0.06 * relief) * _fractal_torch((pad, pad), 0.8, seed, dev)
    domain = torch.zeros((pad, pad), dtype=torch.bool, device=dev)
    domain[1 : 1 + n, 1 : 1 + n] = True
    zc = torch.where(domain, zc, torch.full_like(zc, 1e6))
    # five outfalls on the rim: the main one at the outlet, and the lowest point of four other rim stretches
    zh = zc.cpu().numpy()
    half = 10
    mid = 1 + n // 2
    outfalls = [(np.full(2 * half + 1, n), np.arange(mid - half, mid + half + 1))]
    stretches = [
        ("row", 1, np.arange(1 + n // 8, 1 + 7 * n // 8)),  # north
        ("col", 1, np.arange(1 + n // 8, 1 + 7 * n // 8)),  # west
        ("col", n, np.arange(1 + n // 8, 1 + 7 * n // 8)),  # east
        ("row", n, np.arange(1 + n // 16, 1 + 5 * n // 16)),  # south-west
    ]
    for kind, fixed, span in stretches:
        prof = zh[fixed, span] if kind == "row" else zh[span, fixed]
        m = int(span[np.argmin(prof)])
        seg = np.clip(np.arange(m - 5, m + 6), 1, n)
        outfalls.append((np.full(seg.size, fixed), seg) if kind == "row" else (seg, np.full(seg.size, fixed)))
    sink = torch.zeros_like(domain)
    for rr, cc in outfalls:
        sink[torch.as_tensor(rr, device=dev), torch.as_tensor(cc, device=dev)] = True
    # Planchon-Darboux: the least surface over the ground that drains to a sink, 1 mm a cell of grade
    inf = torch.full_like(zc, float("inf"))
    W = torch.where(sink, zc, inf)
    eps = 1e-3
    for it in range(20 * pad):
        nb = -F.max_pool2d(-W[None, None], 3, stride=1, padding=1)[0, 0]
        Wn = torch.where(domain & ~sink, torch.maximum(zc, torch.minimum(W, nb + eps)), W)
        if it % 64 == 63:
            if torch.equal(Wn, W):
                break
        W = Wn
    # the conditioned surface, its padding repeating the rim; then pixels: bilinear, plus sub-cell relief
    zc = F.pad(W[1 : 1 + n, 1 : 1 + n][None, None], (1, pad - n - 1, 1, pad - n - 1), mode="replicate")[0, 0]
    npx = pad * k
    zp = F.interpolate(zc[None, None], size=(npx, npx), mode="bilinear", align_corners=False)[0, 0]
    zp = zp + 1.5 * _fractal_torch((npx, npx), 0.8, seed + 1, dev)
    # the storm: lognormal depths on 1 km pixels
    rng = np.random.default_rng(3)
    sig = np.sqrt(np.log(1.0 + 0.5**2))
    mu = np.log(60.0) - 0.5 * sig * sig
    nk = int(np.ceil(L / 1000.0))
    field = rng.lognormal(mu, sig, (nk, nk))
    cc = np.clip(((np.arange(pad) - 1 + 0.5) * dx // 1000.0).astype(int), 0, nk - 1)
    rain = field[np.ix_(cc, cc)]
    rain[~domain.cpu().numpy()] = 0.0
    return Catchment(n, dx, k, zp, 0.035, outfalls, rain, 12 * 3600.0, 36 * 3600.0, 10.0, 2.0)


@dataclass(frozen=True)
class EnsembleRun:
    """One run of configuration 4: a seeded fractal fan (``catchment`` at this side, cell size and relief) under a
    uniform storm of its own."""

    side: int
    dx: float
    seed: int
    relief: float
    depth_mm: float
    duration_min: float
    arf: float

    def storm(self):
        from wadi2d_b200.forcing import GivenFactor, UniformStorm

        return UniformStorm(self.depth_mm, self.duration_min, arf=GivenFactor(self.arf))


def ensemble(nruns: int = 64, seed: int = 11, side_min: int = 256, side_max: int = 2048) -> list[EnsembleRun]:
    """Configuration 4: square domains with sides log-uniform in [side_min, side_max] cells at 10-30 m (4 x 4
    pixels a cell), fans with about 3 % of relief over their length, storm durations log-uniform over 1-24 h, depths
    uniform over 20-200 mm, ARF factors uniform over 0.6-1.0."""
    rng = np.random.default_rng(seed)
    out = []
    for r in range(nruns):
        side = int(round(np.exp(rng.uniform(np.log(side_min), np.log(side_max)))))
        dx = float(np.round(rng.uniform(10.0, 30.0), 2))
        dur = float(np.round(np.exp(rng.uniform(np.log(60.0), np.log(1440.0))), 1))
        depth = float(np.round(rng.uniform(20.0, 200.0), 1))
        arf = float(np.round(rng.uniform(0.6, 1.0), 3))
        out.append(EnsembleRun(side, dx, 1000 + r, 0.03 * side * dx, depth, dur, arf))
    return out


@dataclass
class CrestValley:
    """Configuration 2's inputs on a padded grid: DEM pixels, crest faces, Manning per cell, the lumped inflows, the
    reservoir and the downstream outfall."""

    n: int
    dx: float
    k: int
    z: np.ndarray
    crest: object
    """tables.CrestFaces of the breaklines."""
    manning: np.ndarray
    """(ny, nx) Manning n per cell."""
    inflows: list
    """Per inflow: (rows, columns) of its cells, the position of the lowest, hydrograph times (s) and flows (m3/s)."""
    reservoir: tuple
    """(rows, columns) of the reservoir's cells and its start level (m)."""
    outfall: tuple
    """(rows, columns) of the free-outfall cells: the south edge."""
    t_end: float


def crest_valley(n: int = 1024, dx: float = 10.0, k: int = 10, seed: int = 21, relief: float = 120.0,
                 breaklines: int = 40, t_end: float = 6 * 3600.0) -> CrestValley:  # fmt: skip
    """Configuration 2: an n x n fractal valley (Hurst 0.75, ``relief`` m) falling south, carved by 3 seeded
    meandering channels; ``breaklines`` seeded straight breaklines (100-600 m) whose faces carry a crest 0.5-3 m above
    the higher bed beside them; 3 lumped inflows at the channel heads on the north edge (triangular hydrographs, peaks
    50-400 m3/s, times to peak 1-3 h, bases 2.67 times that); a 200 x 50 m reservoir on a channel started 4 m above
    its downstream bed; Manning from seeded Voronoi patches of 0.03-0.06; a free outfall on the south edge."""
    from wadi2d_b200.tables import CrestFaces

    rng = np.random.default_rng(seed)
    pad = 32 * int(np.ceil((n + 2) / 32))
    p = dx / k
    npx = pad * k
    L = n * dx
    c = (np.arange(npx) + 0.5) * p - dx
    X, Y = np.meshgrid(c, c)  # Y grows south
    z = relief * (0.6 * (1.0 - Y / L) + 0.4 * (np.abs(X - 0.5 * L) / L) ** 1.5)
    noise = fractal_noise((npx, npx), 0.75, 1.0, seed)
    z = z + 0.25 * relief * noise / max(float(np.abs(noise).max()), 1e-9)
    # three meandering channels from the north edge to the south edge
    heads = []
    for m in range(3):
        x0 = L * (0.2 + 0.3 * m + rng.uniform(-0.05, 0.05))
        amp, lam, phase = rng.uniform(0.02, 0.06) * L, rng.uniform(0.25, 0.5) * L, rng.uniform(0.0, 2 * np.pi)
        xc = x0 + amp * np.sin(2 * np.pi * Y / lam + phase)
        dist = np.abs(X - xc)
        z = z - np.where(dist < 15.0, 3.0 * (1.0 - dist / 15.0) + 2.0, 2.0 * np.clip(1.0 - (dist - 15.0) / 40.0, 0, 1))
        heads.append(int(np.clip((x0 + amp * np.sin(phase)) // dx + 1, 2, n - 1)))
    zc = z.reshape(pad, k, pad, k)
    cmax = zc.max(axis=(1, 3))
    cmin = zc.min(axis=(1, 3))
    crest = CrestFaces.empty((pad, pad))
    for _ in range(breaklines):
        j0, i0 = rng.integers(2, n - 1), rng.integers(2, n - 1)
        length = rng.uniform(100.0, 600.0) / dx
        ang = rng.uniform(0.0, np.pi)
        j1 = int(np.clip(j0 + length * np.sin(ang), 2, n - 1))
        i1 = int(np.clip(i0 + length * np.cos(ang), 2, n - 1))
        rise = rng.uniform(0.5, 3.0)
        steps = max(abs(j1 - j0), abs(i1 - i0), 1)
        jj = np.round(np.linspace(j0, j1, 2 * steps + 1)).astype(int)
        ii = np.round(np.linspace(i0, i1, 2 * steps + 1)).astype(int)
        for a in range(jj.size - 1):
            ja, ia, jb, ib = jj[a], ii[a], jj[a + 1], ii[a + 1]
            if ib != ia:  # an east-west move crosses the west face of the eastern cell (row ja)
                je, ie = ja, max(ia, ib)
                crest.xz[je, ie] = max(cmax[je, ie], cmax[je, ie - 1]) + rise
            if jb != ja:  # a north-south move crosses the north face of the southern cell (column ib)
                js, is_ = max(ja, jb), ib
                crest.yz[js, is_] = max(cmax[js, is_], cmax[js - 1, is_]) + rise
    # Manning: Voronoi patches
    seeds = rng.uniform(0, pad, (64, 2))
    vals = rng.choice([0.03, 0.04, 0.05, 0.06], 64)
    jg, ig = np.meshgrid(np.arange(pad), np.arange(pad), indexing="ij")
    best = np.full((pad, pad), np.inf)
    manning = np.zeros((pad, pad))
    for s, v in zip(seeds, vals, strict=True):
        d2 = (jg - s[0]) ** 2 + (ig - s[1]) ** 2
        closer = d2 < best
        best[closer] = d2[closer]
        manning[closer] = v
    inflows = []
    for h in heads:
        peak, tp = rng.uniform(50.0, 400.0), rng.uniform(1.0, 3.0) * 3600.0
        rows = np.array([1, 1, 1, 2, 2, 2])
        cols = np.array([h - 1, h, h + 1, h - 1, h, h + 1])
        low = int(np.argmin(cmin[rows, cols]))
        inflows.append((rows, cols, low, np.array([0.0, tp, 2.67 * tp]), np.array([0.0, peak, 0.0])))
    # the reservoir: 20 x 5 cells (200 x 50 m at 10 m) across the middle channel, half-way down
    h = heads[1]
    jr = 1 + n // 2
    rr, cc = np.meshgrid(np.arange(jr - 2, jr + 3), np.arange(h - 10, h + 10), indexing="ij")
    level = float(cmin[jr + 2, h - 10 : h + 10].min()) + 4.0
    rows = np.arange(1, 1 + n)
    return CrestValley(n, dx, k, z, crest, manning, inflows, (rr.ravel(), cc.ravel(), level),
                       (np.full(n, n), rows), t_end)  # fmt: skip
