"""Host-side logic of the package against the oracle's restatement of the reference: grid, layout conversions, FP64
level/plan helpers, hbar_at_level. No GPU needed."""

from __future__ import annotations

import numpy as np

from oracle import oracle as O
from wadi2d_b200 import layout, state
from wadi2d_b200.grid import TileGrid
from wadi2d_b200.tables import hbar_at_level


def grids():
    rng = np.random.default_rng(1)
    for shape in ((40, 40), (70, 130), (5, 200)):
        mask = rng.random(shape) > 0.4
        yield TileGrid.from_mask(mask, 100.0, 200.0, 7.5), O.Grid.from_mask(mask, 100.0, 200.0, 7.5)


def test_grid_matches_reference_restatement():
    for g, o in grids():
        assert g.shape == o.shape and g.x0 == o.x0 and g.y0 == o.y0
        assert np.array_equal(g.tiles, o.tiles)
        assert np.array_equal(g.tile_of, o.tile_of)
        assert np.array_equal(g.nbr, o.nbr)


def test_tile_and_state_conversions():
    rng = np.random.default_rng(2)
    for g, o in grids():
        a = rng.random(g.shape).astype(np.float32)
        assert np.array_equal(g.to_tiles(a), o.to_tiles(a))
        assert np.array_equal(g.from_tiles(g.to_tiles(a)), o.from_tiles(o.to_tiles(a)))
        s = state.to_state(g, a)
        assert np.array_equal(s, O.to_state(o, a))
        assert np.array_equal(state.from_state(g, s), O.from_state(o, s))


def test_native_index_of_own_and_halo_entries():
    g, _ = next(grids())
    ny, nx = g.shape
    t = 1
    tj, ti = g.tiles[t]
    k_own = layout.local_index(t, layout.HALO, layout.HALO)
    assert layout.native_of_ref(g.tiles, [k_own], nx)[0] == layout.native_of_cell(tj * 32, ti * 32, nx)
    k_halo = layout.local_index(t, 0, 1)  # two rows north, one column west of the first own cell
    assert layout.native_of_ref(g.tiles, [k_halo], nx)[0] == layout.native_of_cell(tj * 32 - 2, ti * 32 - 1, nx)


def test_fp64_helpers_match_reference_vectors():
    gold = np.load(__import__("pathlib").Path(__file__).resolve().parent / "golden" / "c1_small.npz")
    import cases
    from oracle_api import OracleApi

    _, ctx = cases.c1_small(OracleApi(), t_end=1.0)
    og, tab = ctx["grid"], ctx["tables"]
    g = TileGrid(og.x0, og.y0, og.dx, og.mask)
    hc, dtab = g.from_tiles(tab["hc"]), g.from_tiles(tab["dtab"])
    assert np.array_equal(state.level_of(gold["fp64_hb_in"], hc, dtab), gold["fp64_level"])
    assert np.array_equal(state.plan_of(gold["fp64_hb_in"], hc, dtab), gold["fp64_plan"])
    assert np.array_equal(hbar_at_level(gold["fp64_levels_in"], tab["zmin"], hc, dtab), gold["fp64_hbar"])
