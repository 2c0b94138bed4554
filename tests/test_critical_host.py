"""The critical-duration search's host side on the CPU: the alternating-block hyetographs and the mixed storms built on
them, the candidate set and its descriptors, and the D8 drainage that places the design lines."""

from __future__ import annotations

import numpy as np
import pytest

from wadi2d_b200 import critical as C


@pytest.mark.parametrize("peak_at", [0.0, 0.2, 0.5, 0.8, 1.0])
def test_alternating_block_is_a_percent_graph_with_its_blocks_alternating_about_the_peak(peak_at):
    n = C.N_BLOCKS
    F = C.alternating_block(n=n, peak_at=peak_at)
    assert F.shape == (n + 1,) and F[0] == 0.0 and F[-1] == 1.0
    blocks = np.diff(F)
    assert (blocks >= 0.0).all()
    p = int(round(peak_at * (n - 1)))
    assert blocks[p] == blocks.max()
    # the increments, largest first, go to the peak, then after and before it by turns
    order, lo, hi = [p], p - 1, p + 1
    while len(order) < n:
        if hi < n:
            order.append(hi)
            hi += 1
        if lo >= 0 and len(order) < n:
            order.append(lo)
            lo -= 1
    assert (np.diff(blocks[order]) <= 1e-15).all()
    # the k most intense blocks hold P(k / n) / P(1) of the depth: P(x) = x (x + b)^-c with b = 0.1, c = 0.7
    x = np.arange(1, n + 1) / n
    P = x * (x + 0.1) ** (-0.7)
    np.testing.assert_allclose(np.cumsum(np.sort(blocks)[::-1]), P / P[-1], rtol=1e-12, atol=1e-15)


def test_mixed_storm_cumulative_depth_interpolates_its_percent_graph():
    s = C.MixedStorm(120.0, 6.0, 0.8, np.array([0.1, 0.2, 0.3, 0.4]))
    np.testing.assert_allclose(s.F, s.weights @ C.BASE)
    assert s.total_depth == pytest.approx(96.0)
    n = s.F.size - 1
    edges = np.arange(n + 1) * s.duration_h * 60.0 / n
    np.testing.assert_allclose(s.cumulative_depth(edges), s.total_depth * s.F, rtol=1e-12, atol=1e-12)
    mid = 0.5 * (edges[:-1] + edges[1:])
    np.testing.assert_allclose(s.cumulative_depth(mid), s.total_depth * 0.5 * (s.F[:-1] + s.F[1:]), rtol=1e-12)
    before, after = s.cumulative_depth(np.array([-5.0, 0.0])), s.cumulative_depth(np.array([360.0, 1e6]))
    np.testing.assert_array_equal(before, [0.0, 0.0])
    np.testing.assert_allclose(after, [s.total_depth, s.total_depth])
    t = np.linspace(0.0, 400.0, 997)
    assert (np.diff(s.cumulative_depth(t)) >= -1e-12).all()


def test_cumulative_many_equals_each_storms_own_cumulative_depth():
    storms = C.candidates(12, seed=3)
    stacked = C.MixedStorm.stack(storms)
    t = np.random.default_rng(1).uniform(0.0, 3000.0, size=len(storms))
    many = C.MixedStorm.cumulative_many(stacked, t)
    one = np.array([s.cumulative_depth(np.array([tk]))[0] for s, tk in zip(storms, t, strict=True)])
    np.testing.assert_array_equal(many, one)


def test_candidates_are_seeded_and_keep_their_ranges():
    a, b = C.candidates(200, seed=9), C.candidates(200, seed=9)
    assert [(s.depth_mm, s.duration_h, s.arf) for s in a] == [(s.depth_mm, s.duration_h, s.arf) for s in b]
    assert C.candidates(5, seed=10)[0].depth_mm != a[0].depth_mm
    for s in a:
        assert 0.5 <= s.duration_h <= 48.0 and 20.0 <= s.depth_mm <= 200.0 and 0.6 <= s.arf <= 1.0
        assert s.weights.sum() == pytest.approx(1.0) and (s.weights >= 0.0).all()
    X = C.features(a)
    assert X.shape == (200, 16) and np.isfinite(X).all()
    np.testing.assert_allclose(X[:, 0], np.log([s.duration_h for s in a]))
    assert ((X[:, 11:14] >= 0.0) & (X[:, 11:14] <= 1.0)).all()  # shares fallen by a quarter, half, three quarters
    assert (np.diff(X[:, 11:14], axis=1) >= 0.0).all()


def test_flow_accumulation_on_a_plane_runs_straight_downhill():
    ny, nx = 20, 7
    j = np.arange(ny)[:, None] * np.ones((1, nx))
    z = 100.0 - 0.5 * j  # falling southward
    acc, step = C.flow_accumulation(z, np.ones((ny, nx), bool))
    assert (step[:-1] == (1, 0)).all() and (step[-1] == 0).all()
    np.testing.assert_array_equal(acc, j + 1.0)


def test_flow_accumulation_of_a_valley_reaches_its_outlet_and_the_lines_sit_on_its_floor():
    from wadi2d_b200.grid import TileGrid

    n = 96
    grid = TileGrid.from_mask(np.ones((n, n), bool), 0.0, 0.0, 10.0)
    ny, nx = grid.shape
    jj, ii = np.mgrid[0:ny, 0:nx]
    c = 1 + n // 2
    z = 0.3 * np.abs(ii - c) + 0.02 * (ny - jj)  # a V-valley along column c, falling southward
    acc, step = C.flow_accumulation(z, grid.mask)
    assert acc.max() == grid.mask.sum()  # every active cell drains to one outlet
    oj, oi = np.unravel_index(np.argmax(acc), acc.shape)
    assert oi == c and oj == n  # the valley floor's last active row
    lines = C.design_lines(grid, z, n=3, half=4, spacing=20, edge=8)
    assert len(lines) == 3
    picked = [ln[4] for ln in lines]
    for k, (xf, xs, yf, ys, (pj, pi)) in enumerate(lines):
        assert pi == c  # on the floor, where the contributing area is largest
        assert xf.size == 0 and yf.size == 9 and (ys == 1.0).all()  # north faces across southward flow
        for pj2, pi2 in picked[:k]:
            assert max(abs(pj - pj2), abs(pi - pi2)) >= 20
