"""Writes to the state between steps, and the momentum hook, on the B200:

- MacDonald's steady flows (tests/solver/test_steady.py:17-83 of the reference): the supercritical inlet is held by
  writing ``b.u[faces]``, ``b.mx[faces]`` and ``b.qx[faces]`` between steps through the backend's index adapters.
  Depth RMSE within the reference's limits in both builds; the exact build equal to the oracle bit for bit.
- ``Model.set_momentum(FaceKick)`` (wadi2d/solver/momentum.py:18-54, applied before every step as
  wadi2d/solver/stepper.py:111-112 does): a kick on the faces of a channel's inlet column of the V-channel plane,
  against the oracle with the same kick, bit for bit (exact build) and within tolerance (fast build)."""

from __future__ import annotations

import numpy as np
import pytest

import cases
import test_oracle_steady as S
from oracle import oracle as O
from oracle_api import Fp64Api, OracleApi
from product_api import B200Api
from wadi2d_b200.momentum import FaceKick

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("arith", ["exact", "fast"])
@pytest.mark.parametrize(("variant", "limit"), S.LIMITS)
def test_macdonald_on_the_b200(variant, limit, arith):
    h, qx, m = S.steady(variant, on="b200", arith=arith)
    want, _ = S.exact(variant, (np.arange(S.NX) + 0.5) * S.DX)
    err = float(np.sqrt(np.mean((h[1, 2:-2] - want[2:-2]) ** 2)))
    assert err < limit, f"{variant}: depth RMSE {err:.4f} m"
    assert qx[1, 2:-2] == pytest.approx(S.Q, rel=0.02)
    if arith == "exact":
        ho, qo, mo = S.steady(variant)
        assert m.stepper.nsteps == mo.nsteps
        assert np.array_equal(h, ho) and np.array_equal(qx, qo)


def _kicked(api, steps: int = 300, kick: bool = True):
    """The V-channel plane of configuration 1 at 64 x 64 cells with 0.2 m of water, a kick eastward on the x faces of
    column 10 and southward on the y faces of row 20 (rates grow along the face lists), ``steps`` host-loop steps."""
    grid, targs, w = cases.c1_small_inputs(api)
    tables = api.tables(grid, *targs)
    m = api.model(grid, tables, {"cfl": 0.45})
    h = np.where(grid.mask, 0.2, 0.0)
    m.set_depth(h)
    xf = np.array([m.cell_state_index(j, 10) for j in range(5, 60)], np.int64)
    yf = np.array([m.cell_state_index(20, i) for i in range(5, 60)], np.int64)
    if kick:
        m.set_momentum(FaceKick.build(xf, np.linspace(0.5, 3.0, xf.size), yf, np.linspace(-1.0, 1.0, yf.size)))

    class Stop(Exception):
        pass

    def cb(st):
        if st.nsteps >= steps:
            raise Stop

    try:
        m.advance(1e9, cb)
    except Stop:
        pass
    return m, grid


@pytest.mark.parametrize("arith, steps", [("exact", 300), ("fast", 100)])
def test_face_kick_against_the_oracle(arith, steps):
    """The exact build equals the oracle bit for bit after 300 kicked steps. The kick drives fronts across the plane,
    a transient in which float32 rounding differences grow: after 100 steps the reference's own float32 step (the
    oracle) is 1.7e-3 m of depth from the FP64 run of the same steps. So the fast build is measured the same way: its
    distance from the FP64 run of its own steps, field by field, may be at most twice the exact step's."""
    api_o = OracleApi()
    mo, go = _kicked(api_o, steps)
    api_b = B200Api(arith=arith)
    mb, gb = _kicked(api_b, steps)
    assert mb.stepper.nsteps == mo.nsteps == steps
    if arith == "exact":
        for name in ("h", "d", "u", "v", "mx", "my", "qx", "qy"):
            assert np.array_equal(mb.field(name), O.from_state(go, mo.backend.get_field(name))), name
    else:
        m64o, _ = _kicked(Fp64Api(list(mo.dts)), steps)
        m64b, _ = _kicked(Fp64Api(list(api_b.dts)), steps)
        for name in ("h", "d", "u", "v", "qx", "qy"):
            exact_err = np.abs(mo.field(name).astype(np.float64) - m64o.field(name)).max()
            fast_err = np.abs(mb.field(name).astype(np.float64) - m64b.field(name)).max()
            scale = np.abs(m64o.field(name)).max()
            assert fast_err <= 2.0 * exact_err + 1e-6 * scale, (name, fast_err, exact_err)
    # the kick reaches the faces: without it the same run ends elsewhere
    m0, _ = _kicked(B200Api(arith=arith), steps, kick=False)
    assert not np.array_equal(mb.field("qx"), m0.field("qx"))
    assert not np.array_equal(mb.field("qy"), m0.field("qy"))
