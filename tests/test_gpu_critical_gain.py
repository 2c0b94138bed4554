"""What the trained network adds to the critical-duration search. On a catchment whose time of concentration is
hours long (96 x 96 cells of 300 m, a fan of 100 m relief: the peak at the main design point comes about 7 h into a
storm), a storm's peak flow follows its depth and its duration together, not its most intense burst: short bursts of
a few tens of millimetres rank first by intensity but peak lower than a longer storm with more depth (on this seeded
set, a 6.2 h storm of 173 mm, 73rd of 160 by peak block intensity). Every candidate goes through the solver (the
exhaustive sweep, as a batch); the network is trained on the solver's results for 64 of them; the critical storm
(largest peak) must be in the network's top 5 % of the candidates and not in the top 5 % by peak block intensity."""

from __future__ import annotations

import numpy as np
import pytest

from wadi2d_b200 import critical as C

pytestmark = pytest.mark.gpu

N, DX, RELIEF, CANDIDATES, TRAIN, STORM_SEED = 96, 300.0, 100.0, 160, 64, 8


def test_network_top_holds_the_critical_storm_the_intensity_ranking_misses():
    cat = C.prepare(n=N, dx=DX, k=4, seed=17, relief=RELIEF)
    storms = C.candidates(CANDIDATES, seed=STORM_SEED)
    x = C.features(storms)
    full = C.solve(cat, storms, recession_h=1.0)
    q = full["peak_q"][:, 0]
    crit = int(np.argmax(q))
    rng = np.random.default_rng(3)
    train = rng.choice(CANDIDATES, size=TRAIN, replace=False)
    assert crit not in set(train.tolist())  # the screen has to find it, not remember it
    y = C.targets({"peak_q": full["peak_q"][train], "t_peak_h": full["t_peak_h"][train]})
    order, pred, losses = C.screen(x[train], y, x, top=0.05, point=0, iters=3000)
    k = len(order)
    by_intensity = np.argsort(x[:, 9])[::-1][:k]
    assert losses[-1] < losses[0]
    assert crit in set(order.tolist()), (crit, order, storms[crit])
    assert crit not in set(by_intensity.tolist())
    # what each screen would report: the largest solver peak among its runs (training runs plus its top share)
    net = max(set(order.tolist()) | set(train.tolist()), key=lambda i: q[i])
    naive = max(set(by_intensity.tolist()) | set(train.tolist()), key=lambda i: q[i])
    assert net == crit
    assert q[naive] < q[crit]
