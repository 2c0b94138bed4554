"""The face momenta formed from the state (the face pass reads the last step's mean depths and the face velocities
instead of stored momenta, and writes none) against reads and writes of the state between steps.

Reading the velocities or momenta between steps (the Field adapters, get_field, w2b_sync_momentum) puts the momenta
in their arrays and makes the next step start from them; that must not change a run by a bit, whether the reads fall
between the device loop's windows or between the host loop's steps, and asking twice must change nothing."""

from __future__ import annotations

import numpy as np
import pytest

from oracle import oracle as O
from wadi2d_b200 import workloads
from wadi2d_b200.config import Numerics
from wadi2d_b200.grid import TileGrid
from wadi2d_b200.model import Model
from wadi2d_b200.tables import GridTables

pytestmark = pytest.mark.gpu

FIELDS = ("h", "d", "u", "v", "mx", "my", "qx", "qy", "res")


def _models(arith: str, count: int = 2):
    """Configuration 1 at 64 x 64 with a wet start under rain, every tile stepped."""
    w = workloads.v_channel_plane(n=64, dx=10.0, k=5, seed=0)
    og = O.Grid.from_mask(np.ones((64, 64), bool), 0.0, 0.0, w.dx)
    tab = O.build_tables(og, w.z, w.dx / w.k, w.manning)
    g = TileGrid.from_mask(np.ones((64, 64), bool), 0.0, 0.0, w.dx)
    out = []
    for _ in range(count):
        m = Model(GridTables.from_dict(g, tab), Numerics(arithmetic=arith))
        m.stepper.adaptive_active = False
        m.set_depth(np.where(g.mask, 0.05, 0.0))
        rate = np.zeros(g.shape)
        rate[1 : 1 + w.ny, 1 : w.nx] = w.rain_mm_h / 3.6e6
        m.set_source(rate)
        out.append(m)
    return g, out


def _peek(m, idx) -> None:
    """Read the velocities and momenta every way a caller can."""
    b = m.backend
    b.u[idx], b.mx[idx], b.v[idx], b.my[idx]
    b.get_field("mx")
    b.sync_momentum()
    b.sync_momentum()


@pytest.mark.parametrize("arith", ["exact", "fast"])
def test_reads_between_windows_leave_the_device_loop_unchanged(arith):
    g, (a, b) = _models(arith)
    idx = np.arange(1296, g.ntiles * 1296, 97)
    for k in range(1, 7):
        a.run(20.0 * k)
        b.run(20.0 * k)
        _peek(b, idx)
    assert a.stepper.nsteps == b.stepper.nsteps > 20
    for name in FIELDS:
        assert np.array_equal(a.field(name), b.field(name)), name


@pytest.mark.parametrize("arith", ["exact", "fast"])
def test_reads_between_host_steps_leave_the_host_loop_unchanged(arith):
    g, (a, b) = _models(arith)
    idx = np.arange(1296, g.ntiles * 1296, 89)
    seen = []

    def peek(st):
        _peek(b, idx)
        seen.append(st.nsteps)

    a.advance(30.0)
    b.advance(30.0, peek)
    assert a.stepper.nsteps == b.stepper.nsteps == len(seen) > 10
    for name in FIELDS:
        assert np.array_equal(a.field(name), b.field(name)), name


def test_written_velocity_keeps_the_momentum_the_step_starts_from():
    """A velocity written between steps does not change the momentum the next step starts from (it is the last
    step's, as in the reference, where u and mx are separate arrays): writing u and writing it back is no change."""
    g, (a, b) = _models("exact")
    a.run(40.0)
    b.run(40.0)
    u = b.backend.get_field("u")
    b.backend.set_field("u", u * 1.5)
    b.backend.set_field("u", u)
    a.run(80.0)
    b.run(80.0)
    for name in FIELDS:
        assert np.array_equal(a.field(name), b.field(name)), name
