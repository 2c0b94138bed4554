"""The host forcing against the reference's own loss, storm and ARF arithmetic (golden vectors), and the pieces that
cannot be imported here against their exact definitions."""

from __future__ import annotations

from pathlib import Path

import numpy as np

from wadi2d_b200 import forcing as F
from wadi2d_b200.grid import TileGrid
from wadi2d_b200.state import state_index

GOLDEN = Path(__file__).resolve().parent / "golden" / "forcing.npz"


def test_scs_arf_uniform_match_reference_vectors():
    g = np.load(GOLDEN)
    scs = np.stack([F.ScsCurveNumber(c).cumulative_excess(g["depth"]) for c in g["cn"]])
    assert np.array_equal(scs, g["scs"])
    scs_ia = np.stack([F.ScsCurveNumber(c, 7.5).cumulative_excess(g["depth"]) for c in g["cn"]])
    assert np.array_equal(scs_ia, g["scs_ia"])
    a = np.array([F.ArfTable(g["areas"], g["factors"]).factor(x) for x in g["probe"]])
    b = np.array([F.ArfTable(g["areas"], g["factors"], False).factor(x) for x in g["probe"]])
    assert np.array_equal(a, g["arf_a"]) and np.array_equal(b, g["arf_b"])
    assert np.array_equal(np.array([F.factor_at(F.GivenFactor(0.8), x) for x in g["probe"]]), g["given"])
    uni = F.UniformStorm(85.0, 150.0, 77.7, F.ArfTable(g["areas"], g["factors"])).cumulative_depth(g["minutes"])
    assert np.array_equal(uni, g["uniform"])


def test_injection_integral_is_exact_and_shares_by_depth():
    inj = F.Injection("a", np.arange(3), np.arange(3), 1, np.array([0.0, 3600.0, 9600.0]), np.array([0.0, 200.0, 0.0]),
                      0.01)  # fmt: skip
    assert inj.volume_at(9600.0) == 0.5 * 200.0 * 9600.0
    # on the rising limb q = 200 t / 3600: V(t) = 100 t^2 / 3600
    for t in (0.0, 100.0, 1800.0, 3599.0):
        assert abs(inj.volume_at(t) - 100.0 * t * t / 3600.0) < 1e-9 * max(1.0, inj.volume_at(t))
    assert abs(inj.mean_flow(0.0, 3600.0) - 100.0) < 1e-12
    assert np.array_equal(inj.share(np.zeros(3)), np.array([0.0, 1.0, 0.0]))  # dry: all to the lowest cell
    s = inj.share(np.array([0.0, 0.3, 0.1]))
    assert np.allclose(s, [0.0, 0.75, 0.25]) and abs(s.sum() - 1.0) < 1e-15


def test_initial_constant_loss_takes_the_initial_loss_first_then_the_rate():
    loss = F.InitialConstantLoss(10.0, 2.0)
    assert loss.window_excess(0.0, 10.0, 600.0) == 0.0  # all to the initial loss
    # 10 mm already met, 5 mm in an hour: 2 mm lost
    assert abs(loss.window_excess(10.0, 15.0, 3600.0) - 3.0) < 1e-12
    # half the window meets the initial loss: the constant loss applies to the other half only
    assert abs(loss.window_excess(5.0, 15.0, 3600.0) - (5.0 - 1.0)) < 1e-12
    assert loss.window_excess(12.0, 12.5, 3600.0) == 0.0  # rain below the constant rate


def test_forcing_rate_rain_volume_and_injection():
    cells = np.arange(10, 30)
    storm = F.UniformStorm(60.0, 60.0)
    inj = F.Injection("in", np.array([0, 1]), cells[:2], 0, np.array([0.0, 600.0]), np.array([4.0, 4.0]), 0.01)
    f = F.Forcing(cells, 100.0, storm, injections=[inj], depth_reader=lambda i: np.zeros(2))
    out, rain, inflow = f.rate(0.0, 30.0)
    assert out.dtype == np.float32
    expect = np.float32(60.0 / 3600.0 / 1000.0)
    assert np.all(out[2:] == expect)
    assert rain == float(np.full(20, expect, np.float32).sum(dtype=np.float64)) * 100.0 * 30.0
    assert abs(inflow - 4.0 * 30.0) < 1e-6 * 120.0


def test_open_faces_match_a_direct_count():
    mask = np.ones((6, 7), bool)
    g = TileGrid.from_mask(mask, 0.0, 0.0, 10.0)
    taken = np.zeros(g.shape, bool)
    taken[1:7, 7] = True  # the east column of the domain
    inner = g.mask & ~taken
    (xi, xs), (yi, ys) = F.open_faces(g, inner, taken)
    assert yi.size == 0
    assert np.array_equal(np.sort(xi), np.sort(state_index(g, np.arange(1, 7), np.full(6, 7))))
    assert np.all(xs == 1.0)


def test_injection_matches_reference_vectors():
    g = np.load(GOLDEN)
    bounds = np.concatenate(([0], np.cumsum(g["inj_len"])))
    for n in range(g["inj_len"].size):
        times = g["inj_times"][bounds[n] : bounds[n + 1]]
        flows = g["inj_flows"][bounds[n] : bounds[n + 1]]
        inj = F.Injection("g", np.arange(5), np.arange(5), 2, times, flows, 0.01)
        vol = np.array([inj.volume_at(float(t)) for t in g["inj_t"]])
        assert np.array_equal(vol, g["inj_vol"][n])
        q = np.array([inj.mean_flow(float(a), float(b)) for a, b in g["inj_windows"]])
        assert np.array_equal(q, g["inj_q"][n])
    inj = F.Injection("s", np.arange(5), np.arange(5), 3, g["inj_times"][:3], g["inj_flows"][:3], 0.01)
    shares = np.stack([inj.share(d) for d in g["inj_depths"]])
    assert np.array_equal(shares, g["inj_shares"])
