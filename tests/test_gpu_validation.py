"""Exact solutions on the B200, as the reference's own analytic suite runs them (tests/solver/test_analytic.py:17-70,
wadi2d/validation): the dam break on a wet bed (Stoker 1957) along x and along y, the dam break on a dry bed (Ritter
1892), both on a flat frictionless bed, Thacker's moving shoreline in a parabolic bowl (planar and curved, Thacker
1981), and still water over a seeded rough bed 1,500 m above the datum. The exact states are written here from the
published formulas (as SWASHES gives them, Delestre et al. 2013); the limits are the reference's: depth and discharge
RMSE over the cells wet in either field, the wet extent's F statistic, and the volume."""

from __future__ import annotations

import math

import numpy as np
import pytest
from scipy.optimize import brentq

from wadi2d_b200.config import Numerics, Tables
from wadi2d_b200.grid import TileGrid
from wadi2d_b200.model import Model
from wadi2d_b200.tables import ArrayBed, build_tables

pytestmark = pytest.mark.gpu

G = 9.80665
PAD = 1  # TileGrid.from_mask pads one cell on the low side of each axis
WET = 1e-3  # depth above which a cell counts as wet in the metrics, m
PLAIN = dict(sheet_flow=False, e_wet=1e-5, h_cfl=1e-4, dt_every=1, dt_max=60.0)


def _model(ny: int, nx: int, dx: float, bed_fn, k: int, manning: float, num: dict):
    """A model on an ny x nx grid of cells of side dx, its tables built on the GPU from bed_fn sampled k x k a cell;
    the cell centres' coordinates (x along columns, y along rows)."""
    tg = TileGrid.from_mask(np.ones((ny, nx), bool), 0.0, 0.0, dx)
    pny, pnx = tg.shape
    p = dx / k
    xs, ys = np.meshgrid((np.arange(pnx * k) - PAD * k + 0.5) * p, (np.arange(pny * k) - PAD * k + 0.5) * p)
    tables = build_tables(tg, ArrayBed(bed_fn(xs, ys), p), Tables(), manning)
    xc, yc = np.meshgrid((np.arange(pnx) - PAD + 0.5) * dx, (np.arange(pny) - PAD + 0.5) * dx)
    return Model(tables, Numerics(**num)), tg, xs, ys, xc, yc


def _state(m: Model, ny: int, nx: int, dx: float):
    """Depth and the unit discharges at the cell centres (the mean of a cell's two faces) on the case grid."""
    sl = (slice(PAD, PAD + ny), slice(PAD, PAD + nx))
    qxf, qyf = m.field("qx"), m.field("qy")
    qx = 0.5 * (qxf + np.roll(qxf, -1, axis=1))[sl] / dx
    qy = 0.5 * (qyf + np.roll(qyf, -1, axis=0))[sl] / dx
    return m.field("h")[sl].astype(np.float64), qx.astype(np.float64), qy.astype(np.float64)


def _fan(xi, c):
    """Depth and velocity in a centred rarefaction from still water of celerity c, at xi = (x - x0) / t."""
    return (2.0 * c - xi) ** 2 / (9.0 * G), 2.0 * (xi + c) / 3.0


def _stoker_star(hl: float, hr: float):
    """The plateau between the rarefaction and the shock: the velocity behind the rarefaction (a Riemann invariant)
    equals the velocity behind the shock (Rankine-Hugoniot); its depth, velocity, celerity and the shock speed."""
    cl = math.sqrt(G * hl)

    def gap(h):
        return 2.0 * (cl - math.sqrt(G * h)) - (h - hr) * math.sqrt(G * (h + hr) / (2.0 * h * hr))

    hm = brentq(gap, hr, hl, xtol=1e-13)
    um = 2.0 * (cl - math.sqrt(G * hm))
    return hm, um, math.sqrt(G * hm), hm * um / (hm - hr)


def _dam_exact(s, x0, t, hl, hr):
    """Depth and unit discharge along the profile coordinate s at time t: Stoker for hr > 0, Ritter for hr = 0."""
    cl = math.sqrt(G * hl)
    xi = (s - x0) / t
    fh, fu = _fan(xi, cl)
    if hr > 0.0:
        hm, um, cm, shock = _stoker_star(hl, hr)
        cond = [xi <= -cl, xi <= um - cm, xi <= shock]
        h = np.select(cond, [hl, fh, hm], hr)
        u = np.select(cond, [0.0, fu, um], 0.0)
    else:
        cond = [xi <= -cl, xi <= 2.0 * cl]
        h = np.select(cond, [hl, fh], 0.0)
        u = np.select(cond, [0.0, fu], 0.0)
    return h, h * u


def _dam_break(axis: str, hl: float, hr: float):
    """The dam break of the reference's case (400 cells of 0.5 m along the profile, 8 across, the dam at the middle),
    run to 0.8 of the first wave's arrival at a domain edge; the metrics against the exact state."""
    n_along, dx = 400, 0.5
    ny, nx = (8, n_along) if axis == "x" else (n_along, 8)
    length = n_along * dx
    x0 = 0.5 * length
    cl = math.sqrt(G * hl)
    front = _stoker_star(hl, hr)[3] if hr > 0.0 else 2.0 * cl
    t_end = 0.8 * min(x0 / cl, (length - x0) / front)
    m, tg, _, _, xc, yc = _model(ny, nx, dx, lambda x, y: np.zeros_like(x), 1, 1e-6, PLAIN)
    s_c = xc if axis == "x" else yc
    h0 = np.where(tg.mask, np.where(s_c <= x0, hl, hr), 0.0)
    m.set_depth(h0)
    m.run(t_end)
    h, qx, qy = _state(m, ny, nx, dx)
    sl = (slice(PAD, PAD + ny), slice(PAD, PAD + nx))
    he, qe = _dam_exact(s_c[sl], x0, m.stepper.t, hl, hr)
    qxe, qye = (qe, 0.0 * qe) if axis == "x" else (0.0 * qe, qe)
    wet = (h > WET) | (he > WET)
    depth_rmse = float(np.sqrt(np.mean((h - he)[wet] ** 2)))
    discharge_rmse = float(np.sqrt(np.mean(np.hypot(qx - qxe, qy - qye)[wet] ** 2)))
    union = np.count_nonzero((h > WET) | (he > WET))
    f_stat = np.count_nonzero((h > WET) & (he > WET)) / union
    v0 = float(h0[sl].sum())
    volume = (float(h.sum()) - v0) / v0
    return depth_rmse, discharge_rmse, f_stat, volume


@pytest.mark.parametrize("axis", ["x", "y"])
def test_stoker_dam_break_on_a_wet_bed(axis):
    depth_rmse, discharge_rmse, _, volume = _dam_break(axis, 2.0, 0.5)
    assert depth_rmse < 0.02
    assert discharge_rmse < 0.07
    assert abs(volume) < 1e-6


def test_ritter_dam_break_on_a_dry_bed():
    depth_rmse, _, f_stat, volume = _dam_break("x", 2.0, 0.0)
    assert depth_rmse < 0.01
    assert f_stat > 0.93
    assert abs(volume) < 1e-6


def _rough_bed(amplitude: float, corr: float, seed: int, n_modes: int = 256):
    """A stationary Gaussian random bed by random Fourier features (Rahimi and Recht 2007): n_modes cosines with
    normal wavenumbers of standard deviation 1 / corr and uniform phases; mean 0, standard deviation amplitude."""
    rng = np.random.default_rng(seed)
    kx, ky = rng.normal(0.0, 1.0 / corr, size=(2, n_modes))
    phase = rng.uniform(0.0, 2.0 * math.pi, size=n_modes)

    def bed(x, y):
        total = np.zeros_like(x, dtype=np.float64)
        for a, b, c in zip(kx, ky, phase, strict=True):
            total += np.cos(a * x + b * y + c)
        return amplitude * math.sqrt(2.0 / n_modes) * total

    return bed


@pytest.mark.parametrize("sheet", [False, True])
def test_still_water_stays_still_on_rough_ground_at_altitude(sheet):
    """Still water at 1,500 m over a seeded rough bed (amplitude 0.5 m: about half the bed emerged), 100 x 100 cells
    of 0.1 m with 4 x 4 pixels: after 2 s of settling (the cell-mean start differs from the table's level by the
    interpolation error), 10 s more move nothing and lose no volume."""
    n, dx, k, lift = 100, 0.1, 4, 1500.0
    rough = _rough_bed(0.5, 5.0 * dx, 0)
    m, tg, xs, ys, _, _ = _model(n, n, dx, lambda x, y: rough(x, y) + lift, k, 0.03, dict(sheet_flow=sheet, dt_every=1))
    depth = np.maximum(lift - (rough(xs, ys) + lift), 0.0)
    pny, pnx = tg.shape
    hbar = depth.reshape(pny, k, pnx, k).mean(axis=(1, 3))
    m.set_depth(np.where(tg.mask, hbar, 0.0))
    m.run(2.0)
    v0 = m.volume()
    m.run(12.0)
    h = m.field("h")
    deep = (h > 0.01) & (np.roll(h, 1, axis=1) > 0.01) & (np.roll(h, 1, axis=0) > 0.01)
    assert deep.sum() > 1000
    assert np.abs(m.field("u"))[deep].max() < 1e-2
    assert np.abs(m.field("v"))[deep].max() < 1e-2
    assert abs(m.volume() / v0 - 1.0) < 1e-6


def _thacker(kind: str):
    """Thacker's oscillations in the bowl z = -h0 (1 - r^2 / a^2) (Thacker 1981, with SWASHES' parameters a = 1 m,
    h0 = 0.1 m; the planar surface with eta = 0.5, the curved one with r0 = 0.8), frictionless, on 200 x 200 cells of
    0.02 m with 4 x 4 pixels, started from the exact state averaged over each cell's pixels and run three periods."""
    a, h0, n, dx, k = 1.0, 0.1, 200, 0.02, 4
    xc = yc = 0.5 * n * dx

    def bed(x, y):
        return -h0 * (1.0 - ((x - xc) ** 2 + (y - yc) ** 2) / a**2)

    if kind == "planar":
        eta = 0.5
        omega = math.sqrt(2.0 * G * h0) / a

        def exact(x, y, t):
            ph = omega * t
            surface = eta * h0 / a**2 * (2.0 * (x - xc) * math.cos(ph) + 2.0 * (y - yc) * math.sin(ph) - eta)
            h = np.maximum(surface - bed(x, y), 0.0)
            return h, -eta * omega * math.sin(ph) * h, eta * omega * math.cos(ph) * h
    else:
        r0 = 0.8
        amp = (a * a - r0 * r0) / (a * a + r0 * r0)
        omega = math.sqrt(8.0 * G * h0) / a

        def exact(x, y, t):
            ph = omega * t
            s = math.sqrt(1.0 - amp * amp) / (1.0 - amp * math.cos(ph))
            rate = omega * amp * math.sin(ph) / (2.0 * (1.0 - amp * math.cos(ph)))
            h = np.maximum(h0 * (s - ((x - xc) ** 2 + (y - yc) ** 2) / a**2 * s * s), 0.0)
            return h, h * rate * (x - xc), h * rate * (y - yc)

    m, tg, xs, ys, xcell, ycell = _model(n, n, dx, bed, k, 1e-6, PLAIN)
    pny, pnx = tg.shape
    hp, qxp, qyp = exact(xs, ys, 0.0)

    def mean(f):
        return np.broadcast_to(f, xs.shape).reshape(pny, k, pnx, k).mean(axis=(1, 3))

    hbar, qx, qy = mean(hp), mean(qxp), mean(qyp)
    inside = tg.mask
    m.set_depth(np.where(inside, hbar, 0.0))
    wet = hbar > 1e-9
    m.set_velocity(np.where(wet & inside, qx / np.maximum(hbar, 1e-9), 0.0),
                   np.where(wet & inside, qy / np.maximum(hbar, 1e-9), 0.0))  # fmt: skip
    v0 = m.volume()
    m.run(3.0 * 2.0 * math.pi / omega)
    h, _, _ = _state(m, n, n, dx)
    sl = (slice(PAD, PAD + n), slice(PAD, PAD + n))
    he, _, _ = exact(xcell[sl], ycell[sl], m.stepper.t)
    both = (h > WET) | (he > WET)
    depth_rmse = float(np.sqrt(np.mean((h - he)[both] ** 2)))
    return depth_rmse, m.volume() / v0 - 1.0


@pytest.mark.parametrize("kind, limit", [("planar", 0.0055), ("curved", 0.002)])
def test_thacker_moving_shoreline(kind, limit):
    depth_rmse, volume = _thacker(kind)
    assert depth_rmse < limit
    assert abs(volume) < 5e-5
