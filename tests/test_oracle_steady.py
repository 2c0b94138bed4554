"""MacDonald's steady flows with friction on the oracle, with the reference's setup and limits
(tests/solver/test_steady.py:17-83): subcritical, supercritical, and with a hydraulic jump. No GPU needed.

The exact solutions follow MacDonald et al. 1997 (J. Hydraul. Eng. 123(11)) and the SWASHES set-up (Delestre et al.
2013): a 1,000 m channel, unit discharge 2 m2/s, Manning n = 0.033. The depth profile is prescribed and the bed
follows from steady momentum with Manning friction on a wide channel, d(z + E)/dx = -Sf, integrated from the outlet
(z = 0) upstream. The profiles are written here from those papers:

- subcritical: critical depth times 1 + exp(-16 (x/L - 1/2)^2) / 2;
- supercritical: critical depth times 1 - exp(-36 (x/L - 1/2)^2) / 5;
- jump: the reference's variant of the same set-up. Two linear branches meet at 0.4 L at conjugate depths: 0.7
  times critical depth ahead, with the depth falling 20 % of it per length upstream of the jump, and the sequent
  depth behind, rising 5 % of it per length. The bed is continuous across the jump.

The model is the reference's ``Model`` API on the oracle. It has 200 x 4 cells of 5 m, one pixel a cell, and starts
at the exact state. The inlet holds the exact depth and discharge where the flow there is supercritical; a
subcritical inlet is a discharge source in the first column. The outlet holds the exact depth where the flow there
is subcritical and is free otherwise."""

from __future__ import annotations

import math

import numpy as np
import pytest
from scipy.integrate import quad

from oracle import oracle as O

G, Q, N, L = 9.80665, 2.0, 0.033, 1000.0
DX, NX, NY, PAD = 5.0, 200, 4, 1
HC = (Q * Q / G) ** (1.0 / 3.0)


def friction_slope(h):
    return N * N * Q * Q / h ** (10.0 / 3.0)


def energy(h):
    return h + Q * Q / (2.0 * G * h * h)


def branches(variant: str):
    """(start, end, depth function) of each smooth stretch of the profile, inlet to outlet."""
    if variant == "subcritical":
        return [(0.0, L, lambda s: HC * (1.0 + 0.5 * np.exp(-16.0 * (s / L - 0.5) ** 2)))]
    if variant == "supercritical":
        return [(0.0, L, lambda s: HC * (1.0 - 0.2 * np.exp(-36.0 * (s / L - 0.5) ** 2)))]
    jump = 0.4 * L
    ahead = 0.7 * HC
    behind = 0.5 * ahead * (math.sqrt(1.0 + 8.0 * Q * Q / (G * ahead**3)) - 1.0)  # Belanger's sequent depth
    return [(0.0, jump, lambda s: ahead - 0.2 * ahead / L * (s - jump)),
            (jump, L, lambda s: behind + 0.05 * behind / L * (s - jump))]  # fmt: skip


def exact(variant: str, s: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """Depth and bed at distances s from the inlet; each end branch carries on past the channel's ends."""
    parts = branches(variant)
    # the bed at the end of each branch, marching from the outlet: continuous across the jump
    bed_end = [0.0] * len(parts)
    for k in range(len(parts) - 2, -1, -1):
        a, b, h = parts[k + 1]
        bed_end[k] = bed_end[k + 1] + energy(h(b)) - energy(h(a)) + quad(lambda x: friction_slope(h(x)), a, b)[0]
    s = np.asarray(s, np.float64)
    owner = np.searchsorted([p[1] for p in parts[:-1]], s, side="right")
    depth, bed = np.empty_like(s), np.empty_like(s)
    for idx in np.ndindex(s.shape):
        a, b, h = parts[owner[idx]]
        x = float(s[idx])
        depth[idx] = h(x)
        # z(x) = z(b) + E(h(b)) - E(h(x)) + integral of Sf from x to b
        bed[idx] = bed_end[owner[idx]] + energy(h(b)) - energy(h(x)) + quad(lambda y: friction_slope(h(y)), x, b)[0]
    return depth, bed


def steady(variant: str, t_end: float = 2500.0, on: str = "oracle", arith: str = "exact"):
    """The run of tests/solver/test_steady.py:17-64 on the oracle, or (``on="b200"``) on this package's CUDA path with
    the oracle's tables and the ``arith`` build: (depth, unit discharge) on the channel's cells, and the model."""
    g = O.Grid.from_mask(np.ones((NY, NX), bool), 0.0, 0.0, DX)
    ny, nx = g.shape
    x = (np.arange(nx) - PAD + 0.5) * DX  # cell centres of the padded grid, one pixel a cell
    h_cells, bed_cells = exact(variant, x)
    z = np.broadcast_to(bed_cells, (ny, nx)).copy()
    tables = O.build_tables(g, z, DX, N)
    Boundary = O.Boundary
    if on == "oracle":
        m = O.Model(g, tables, O.Numerics(dt_every=1, e_wet=1e-5))
    else:
        from wadi2d_b200.backend import BoundaryCells as Boundary
        from wadi2d_b200.config import Numerics
        from wadi2d_b200.grid import TileGrid
        from wadi2d_b200.model import Model
        from wadi2d_b200.tables import GridTables

        tg = TileGrid(g.x0, g.y0, g.dx, g.mask)
        m = Model(GridTables.from_dict(tg, tables), Numerics(dt_every=1, e_wet=1e-5, arithmetic=arith))
    h0 = np.broadcast_to(h_cells, (ny, nx))
    m.set_depth(h0)
    m.set_velocity(Q / h0, np.zeros((ny, nx)))
    h_in, h_out = (float(v) for v in exact(variant, np.array([0.5 * DX, L - 0.5 * DX]))[0])
    rows = range(PAD, PAD + NY)
    inlet = [m.cell_state_index(j, PAD) for j in rows]
    first_face = [m.cell_state_index(j, PAD + 1) for j in rows]
    last = [m.cell_state_index(j, PAD + NX - 1) for j in rows]
    before_last = [m.cell_state_index(j, PAD + NX - 2) for j in rows]
    sub_in, sub_out = variant == "subcritical", variant != "supercritical"
    held = [] if sub_in else inlet
    d_out = h_out if sub_out else 0.0
    depths = [h_in] * len(held) + [d_out] * NY
    m.set_boundary(Boundary(np.array(held + last, np.int32), np.array(held + before_last, np.int32),
                            np.array([0] * len(held) + [0 if sub_out else 2] * NY, np.int32),
                            np.array(depths, np.float32), np.array(depths, np.float32)))  # fmt: skip
    if sub_in:
        rate = np.zeros((ny, nx))
        rate[PAD : PAD + NY, PAD] = Q / DX
        m.set_source(rate)
        m.advance(t_end)
    else:
        b = m.backend
        faces = np.array(first_face + inlet)  # the inlet cell's west face too: momentum coming in
        u_in = Q / h_in

        def hold(_):
            b.u[faces] = u_in
            b.mx[faces] = h_in * DX * u_in
            b.qx[faces] = Q * DX

        m.advance(t_end, hold)
    sl = (slice(PAD, PAD + NY), slice(PAD, PAD + NX))
    qxf = m.field("qx")
    qx = 0.5 * (qxf + np.roll(qxf, -1, axis=1))[sl] / DX
    return m.field("h")[sl].astype(np.float64), qx.astype(np.float64), m


LIMITS = [("subcritical", 0.015), ("supercritical", 0.012), ("jump", 0.05)]


@pytest.mark.parametrize(("variant", "limit"), LIMITS)
def test_macdonald(variant, limit):
    h, qx, _ = steady(variant)
    want, _ = exact(variant, (np.arange(NX) + 0.5) * DX)
    err = float(np.sqrt(np.mean((h[1, 2:-2] - want[2:-2]) ** 2)))
    assert err < limit, f"{variant}: depth RMSE {err:.4f} m"
    assert qx[1, 2:-2] == pytest.approx(Q, rel=0.02)
