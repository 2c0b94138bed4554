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
