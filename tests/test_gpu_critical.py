"""The critical-duration search on the B200: storms with mixed alternating-block patterns run as one batch give, at
the design lines, the same peak discharges and times, and the same step counts, as each storm run alone (Model.run
through the window driver, lines on the device); the screen trains the network on solver runs and ranks
candidates."""

from __future__ import annotations

import numpy as np
import pytest

from wadi2d_b200 import critical as C

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def catchment():
    return C.prepare(n=64, dx=10.0, k=4, seed=3)


def test_batched_storms_give_each_storm_its_own_peaks(catchment):
    from wadi2d_b200.config import Numerics
    from wadi2d_b200.maxima import Lines, Tally
    from wadi2d_b200.model import Model
    from wadi2d_b200.run import DeviceRain, run_windows

    cat = catchment
    assert len(cat.lines) >= 4
    storms = C.candidates(4, seed=1, hours=(0.3, 0.8), depth=(60.0, 200.0))
    res = C.solve(cat, storms, recession_h=0.25, batch=4)
    assert res["peak_q"].max() > 0.0
    for r, s in enumerate(storms):
        m = Model(cat.tables, Numerics())
        m.set_boundary(cat.boundary)
        m.set_depth(np.zeros(cat.grid.shape))
        tally = Tally(m, *cat.tally)
        lines = Lines(m, [ln[:4] for ln in cat.lines])
        rain = DeviceRain(m, s, cat.rained)
        run_windows(m, (s.duration_h + 0.25) * 3600.0, rain=rain, window=30.0, tally=tally)
        q, t = lines.peaks()
        assert m.stepper.nsteps == res["steps"][r], r
        assert np.array_equal(q, res["peak_q"][r]), r
        assert np.array_equal(t / 3600.0, res["t_peak_h"][r]), r


def test_screen_trains_on_solver_runs_and_ranks(catchment):
    storms = C.candidates(24, seed=2, hours=(0.3, 1.0), depth=(40.0, 200.0))
    res = C.solve(catchment, storms, recession_h=0.25, batch=24)
    x, y = C.features(storms), C.targets(res)
    order, pred, losses = C.screen(x[:16], y[:16], x, top=0.25, iters=400)
    assert len(order) == 6 and len(set(order.tolist())) == 6
    assert losses[-1] < losses[0]
    assert pred.shape == (24, 2 * len(catchment.lines)) and np.all(np.isfinite(pred))
