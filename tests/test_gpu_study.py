"""The depth-area study on the batch engine: every storm area in one batch gives the same runs, design table and
composite maps as the runs one after another (the reference's order), bit for bit."""

from __future__ import annotations

import numpy as np
import pytest

from wadi2d_b200 import critical as C
from wadi2d_b200 import study as S
from wadi2d_b200.forcing import ArfTable, UniformStorm

pytestmark = pytest.mark.gpu


def test_batched_study_equals_runs_one_after_another():
    cat = C.prepare(n=96, dx=10.0, k=4, seed=3)
    arf = ArfTable(np.array([0.01, 0.1, 1.0, 10.0]), np.array([1.0, 0.95, 0.85, 0.7]))
    storm = UniformStorm(60.0, 40.0, arf=arf)
    areas, cell, line_a = S.bracketing_areas(cat, ratio=2.0, most=4)
    assert len(areas) >= 2
    depths = {round(s.total_depth, 9) for s in S.storms_at(storm, areas)}
    assert len(depths) == len(areas)  # the table tells the runs apart
    names = [f"line{n}" for n in range(len(cat.lines))]
    kw = dict(t_end=3600.0, window=30.0, every=4)
    b = S.run_study(cat, storm, areas, names, list(line_a), cell, batched=True, **kw)
    p = S.run_study(cat, storm, areas, names, list(line_a), cell, batched=False, **kw)
    assert np.array_equal(b.steps, p.steps)
    assert np.array_equal(b.peaks, p.peaks) and np.array_equal(b.times, p.times)
    assert b.table == p.table
    for name in S.COMPOSITE_MAPS:
        assert np.array_equal(b.composite[name], p.composite[name]), name
    # rain falls less deep at larger storm areas, and every line carries water in every run
    assert np.all(b.peaks > 0.0)
    assert len(b.table) == len(cat.lines)
    assert all(r["storm_area_low_km2"] <= r["storm_area_high_km2"] for r in b.table)
