"""The oracle's face tables against the reference's own known answers for the local hydraulic radius
(tests/tables/test_local_radius.py:100-232; Spada et al. 2015, HESSD 12, 2607, eqs. 14 to 17). No GPU needed.

- On a bed with no relief across the faces, the local radius gives the strips sum.
- On a deep narrow gorge, the conveyance that the x faces of one column carry together equals a direct evaluation of
  Spada et al.'s integrals on the same ground, at 20, 10 and 5 m cells.
- The local radius reads the gorge deeper than the strips sum does, and alike at 20 and 5 m.
- A flat face in a channel deeper than its table still sees the walls.
- A face's line reaches past its ends no further than the bed is long (the reach cap of
  wadi2d/tables/builder.py:261-269, as the GPU builder takes it).

The GPU builder equals the oracle's tables within one float32 ulp (tests/test_gpu_tables.py), so these properties
carry over to it."""

from __future__ import annotations

import numpy as np
import pytest
from scipy.optimize import brentq

from oracle import oracle as O
from wadi2d_b200.config import Tables
from wadi2d_b200.tablebuild import tile_margin

PIXEL, SLOPE, MANNING, Q, BETA = 0.5, 0.01, 0.05, 300.0, 9.0
ACROSS, ALONG = 640, 160  # pixels: 320 m across the gorge, 80 m along it


def gorge_section(t: np.ndarray) -> np.ndarray:
    """Bed height over the thalweg at distance t across: a 12 m floor, walls rising 7 m over 1.5 m, a 10 m ledge at
    5 %, then hills at 50 %."""
    a = np.abs(t)
    return np.select([a < 6.0, a < 7.5, a < 17.5], [0.0 * a, (a - 6.0) * (7.0 / 1.5), 7.0 + 0.05 * (a - 7.5)],
                     7.5 + 0.5 * (a - 17.5))  # fmt: skip


def _across() -> np.ndarray:
    return (np.arange(ACROSS) + 0.5) * PIXEL - 0.5 * ACROSS * PIXEL


def bed_of(section: np.ndarray) -> np.ndarray:
    """Pixels: rows across (y), columns along (x), falling SLOPE along x; rounded through float32 like a DEM."""
    x = (np.arange(ALONG) + 0.5) * PIXEL
    return (100.0 - SLOPE * x[None, :] + section[:, None]).astype(np.float32).astype(np.float64)


def conveyance_from_table(e: float, top: float, tab: np.ndarray) -> float:
    """K = T^(5/3) at depth e over the face invert, T read from the face's table (rows of (area, T) at the depths
    top (r/m)^2, prismatic above top), as the step's face lookup reads it (wadi2d/solver/cpu/kernels.py:62-83)."""
    m = tab.shape[0] - 1
    if e >= top:
        a0, a1 = tab[m - 1, 0], tab[m, 0]
        width = (a1 - a0) / (top * (1.0 - ((m - 1) / m) ** 2))
        area = a1 + width * (e - top)
        t = tab[m, 1] * area / max(a1, 1e-12)
    else:
        r = min(int(np.sqrt(e / top) * m), m - 1)
        e0, e1 = (r / m) ** 2 * top, ((r + 1) / m) ** 2 * top
        f = (e - e0) / (e1 - e0)
        t = tab[r, 1] + f * (tab[r + 1, 1] - tab[r, 1])
    return float(t) ** (5.0 / 3.0)


def column_conveyance(dx: float, local: bool, level_over_bed: float, bed: np.ndarray) -> float:
    """Sum of the conveyances of the x faces of the grid's middle column at a level over the bed there. The grid
    covers the bed, its padding ring one cell before the bed's first pixel (the bed read with edge clipping)."""
    k = round(dx / PIXEL)
    ny, nx = ACROSS // k, ALONG // k
    g = O.Grid.from_mask(np.ones((ny, nx), bool), 0.0, 0.0, dx)
    z = np.pad(bed, ((k, 0), (k, 0)), mode="edge")  # pixel (r, c) of the padded grid is bed[r - k, c - k]
    t = O.build_tables(g, z, PIXEL, MANNING, local_radius=local, beta=BETA)
    ftab, top, fl = g.from_tiles(t["ftabx"]), g.from_tiles(t["efx"]), g.from_tiles(t["flx"])
    i = nx // 2 + 1  # the padded column of the unpadded grid's middle x face
    level = 100.0 - SLOPE * (nx // 2) * dx + level_over_bed
    total = 0.0
    for j in range(1, ny + 1):
        e = level - (fl[j, i] + t["zmin"][j, i - 1])
        if e > 0.0:
            total += conveyance_from_table(float(np.float32(e)), float(top[j, i]), ftab[j, i].astype(np.float64))
    return total


def spada_direct(level_over_bed: float) -> float:
    """Spada et al.'s local-radius conveyance of the gorge's section, evaluated directly at the pixel spacing: for
    each wet pixel, a triangular window of half-width BETA times its depth over the wet stretch it lies in; its radius
    the window-weighted depth over the window-weighted wetted length; K = sum of d R^(2/3) pixel / n."""
    z = gorge_section(_across())
    d = np.clip(level_over_bed - z, 0.0, None)
    wet = d > 0.0
    # wetted length between neighbouring pixel centres: half to each end when both are wet, and when one end is
    # dry, to the wet end the share of the segment under water
    seg = np.hypot(PIXEL, np.diff(z))
    both = wet[:-1] & wet[1:]
    one = wet[:-1] ^ wet[1:]
    per = np.zeros(z.size)
    per[:-1] += np.where(both, 0.5 * seg, 0.0)
    per[1:] += np.where(both, 0.5 * seg, 0.0)
    lo_end = np.where(wet[:-1], np.arange(z.size - 1), np.arange(1, z.size))
    share = np.minimum(d[lo_end] / np.maximum(np.abs(np.diff(z)), 1e-300), 1.0) * seg
    np.add.at(per, lo_end[one], share[one])
    # contiguous wet stretches
    run = np.cumsum(np.concatenate(([1], (~wet[1:] | ~wet[:-1]).astype(int))))
    idx = np.arange(z.size)
    total = 0.0
    for i in np.nonzero(wet)[0]:
        j = idx[(run == run[i]) & wet]
        weight = np.clip(1.0 - np.abs(j - i) / (BETA * d[i] / PIXEL), 0.0, None)
        radius = PIXEL * float(np.sum(d[j] * weight)) / float(np.sum(per[j] * weight))
        total += d[i] * radius ** (2.0 / 3.0) * PIXEL / MANNING
    return total


def test_a_bed_with_no_relief_across_the_faces_gives_the_strips_sum():
    flat = bed_of(np.zeros(ACROSS))
    strips = column_conveyance(20.0, False, 2.0, flat)
    assert column_conveyance(20.0, True, 2.0, flat) == pytest.approx(strips, rel=1e-5)


@pytest.mark.parametrize("dx", [20.0, 10.0, 5.0])
def test_the_gorge_conveyance_is_spada_et_al_s_at_every_cell_size(dx):
    bed = bed_of(gorge_section(_across()))
    for over in (2.0, 4.0, 5.3):
        assert column_conveyance(dx, True, over, bed) == pytest.approx(spada_direct(over), rel=0.01), over


def test_the_gorge_reads_deeper_than_the_strips_sum_and_alike_at_every_size():
    bed = bed_of(gorge_section(_across()))

    def normal_depth(dx, local):
        return brentq(lambda h: column_conveyance(dx, local, h, bed) * SLOPE**0.5 - Q, 1.0, 12.0, xtol=1e-3)

    strips = [normal_depth(dx, False) for dx in (20.0, 5.0)]
    local = [normal_depth(dx, True) for dx in (20.0, 5.0)]
    assert abs(strips[0] - strips[1]) < 0.02 and abs(local[0] - local[1]) < 0.03
    assert local[0] > 1.15 * strips[0], (strips, local)


def test_a_flat_face_in_a_channel_deeper_than_its_table_still_sees_the_walls():
    """A 12 m rectangular channel 20 m deep, at a level 11 m over its bed: above the faces' own (flat) relief the
    table's top reaches the walls in the face's window, so the conveyance stays the walled channel's at 20 m and
    2.5 m cells, well under the strips sum."""
    bed = bed_of(np.where(np.abs(_across()) < 6.0, 0.0, 20.0))
    coarse = column_conveyance(20.0, True, 11.0, bed)
    fine = column_conveyance(2.5, True, 11.0, bed)
    assert fine == pytest.approx(coarse, rel=0.005)
    assert fine < 0.8 * column_conveyance(2.5, False, 11.0, bed)


def test_a_face_line_reaches_no_further_than_the_bed_is_long():
    cfg = Tables()
    asked = int(np.ceil(cfg.local_radius_beta * cfg.face_depth_max / 0.005))  # 5 mm pixels: 28,800
    assert tile_margin(cfg, 0.005, 248) == 248 < asked
    assert tile_margin(cfg, 1.0, 320) == 144  # a bed longer than the reach is read as before
    assert tile_margin(Tables(face_conveyance="strips"), 1.0, 320) == 0
