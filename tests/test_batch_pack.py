"""The batch's host side: shelf packing of uneven runs into one grid of tiles, the tile maps, and the cut neighbour
links that keep one run from waking another's tiles."""

from __future__ import annotations

import numpy as np
import pytest

from wadi2d_b200.batch import pack, shelf_pack
from wadi2d_b200.grid import TileGrid
from wadi2d_b200.layout import TILE


def _grids(sides, seed=0):
    rng = np.random.default_rng(seed)
    out = []
    for n in sides:
        m = rng.random((n, n)) < 0.97
        m[n // 2, :] = True
        out.append(TileGrid.from_mask(m, 0.0, 0.0, float(rng.uniform(10.0, 30.0))))
    return out


def test_shelf_pack_places_every_grid_without_overlap():
    rng = np.random.default_rng(1)
    shapes = [(int(rng.integers(1, 9)), int(rng.integers(1, 9))) for _ in range(40)]
    place, (nty, ntx) = shelf_pack(shapes, 20)
    occ = np.zeros((nty, ntx), np.int32)
    for (h, w), p in zip(shapes, place, strict=True):
        assert p.oi + w <= ntx and p.oj + h <= nty
        occ[p.oj : p.oj + h, p.oi : p.oi + w] += 1
    assert occ.max() == 1
    assert occ.sum() == sum(h * w for h, w in shapes)


def test_shelf_pack_widens_to_the_widest_grid():
    place, (nty, ntx) = shelf_pack([(2, 7), (1, 3)], 4)
    assert ntx == 7 and place[0].oi == 0


@pytest.mark.parametrize("sides", [[30, 100, 62, 5], [200], [33, 33, 33, 33, 33, 33, 33]])
def test_pack_maps_every_run_cell_to_its_packed_cell(sides):
    grids = _grids(sides)
    p = pack(grids)
    assert p.grid.ntiles - 1 == sum(g.ntiles - 1 for g in grids)
    for r, (g, pl, m) in enumerate(zip(grids, p.place, p.map, strict=True)):
        ny, nx = g.shape
        sub = p.grid.mask[pl.oj * TILE : pl.oj * TILE + ny, pl.oi * TILE : pl.oi * TILE + nx]
        assert np.array_equal(sub, g.mask)
        assert np.array_equal(p.grid.tiles[m[1:]], g.tiles[1:] + [pl.oj, pl.oi])
        assert np.all(p.tile_run[m[1:]] == r)
    assert p.tile_run[0] == 0


def test_pack_cuts_neighbour_links_between_runs_only():
    grids = _grids([40, 40, 40, 40])
    p = pack(grids, width=4)
    nbr = p.grid.nbr
    tr = p.tile_run
    linked = nbr[1:] != 0
    assert np.all(tr[nbr[1:]][linked] == np.repeat(tr[1:, None], 8, axis=1)[linked])
    # within a run, the links are the run's own links, mapped
    for g, m in zip(grids, p.map, strict=True):
        assert np.array_equal(nbr[m[1:]], m[g.nbr[1:]])


def test_pack_rejects_a_mask_on_the_grid_edge():
    g = TileGrid(0.0, 0.0, 10.0, np.ones((32, 32), bool))
    with pytest.raises(ValueError):
        pack([g])
