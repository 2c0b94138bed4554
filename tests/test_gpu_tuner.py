"""The device loop's launch tuner (w2b_loop_tuning / w2b_loop_config): a run whose first graph launches rotate through
the candidate launch schedules gives the same bits as the run under the default schedule fixed, and the tuner settles
on one of its candidates; the face pass's strip forms (16 and 8 rows of a tile at a time) give its tile form's bits."""

from __future__ import annotations

import numpy as np
import pytest

import cases
from product_api import B200Api

pytestmark = pytest.mark.gpu


class LoopApi(B200Api):
    """The case API with the device loop, tuning (``tune``) or under the occupancy-given default fixed (the face pass
    in its tile form, or with ``strips`` in its strip form)."""

    def __init__(self, tune: bool, strips: int = 0, arith: str = "exact") -> None:
        super().__init__(device_loop=True, arith=arith)
        self.tune, self.strips = tune, strips
        self.m = None

    def model(self, grid, tables, numerics):
        m = super().model(grid, tables, numerics)
        cfg = m.backend.loop_config()
        assert cfg["tuning"] == 1  # a new handle tunes
        if not self.tune:
            faces = cfg[f"strips{self.strips}_occupancy"] if self.strips else cfg["faces_occupancy"]
            m.backend.set_loop(False, faces, cfg["update_occupancy"], 16, strips=self.strips)
        self.m = m
        return m


def test_tuned_run_equals_the_default_schedule_bit_for_bit():
    tuned, fixed = LoopApi(True), LoopApi(False)
    a, ctx = cases.c1_small(tuned, t_end=1500.0)
    b, _ = cases.c1_small(fixed, t_end=1500.0)
    assert int(a["nsteps"]) > 300  # enough graph launches for every candidate's samples
    for key in a:
        assert np.array_equal(np.asarray(a[key]), np.asarray(b[key])), key
    cfg = tuned.m.backend.loop_config()
    assert cfg["tuning"] == 0
    occ = cfg[f"strips{cfg['strips']}_occupancy"] if cfg["strips"] else cfg["faces_occupancy"]
    assert 1 <= cfg["faces_per_sm"] <= occ
    assert 1 <= cfg["update_per_sm"] <= cfg["update_occupancy"]
    assert cfg["steps_per_graph"] in (8, 16, 32)
    fcfg = fixed.m.backend.loop_config()
    assert fcfg["tuning"] == 0 and fcfg["steps_per_graph"] == 16


def test_fixed_schedule_is_checked():
    api = LoopApi(False)
    cases.c1_small(api, t_end=30.0)
    b = api.m.backend
    cfg = b.loop_config()
    from wadi2d_b200 import _lib

    for bad in ((0, 1, 16), (cfg["faces_occupancy"] + 1, 1, 16), (1, cfg["update_occupancy"] + 1, 16), (1, 1, 65)):
        with pytest.raises(_lib.W2BError):
            b.set_loop(False, *bad)
    b.set_loop(False, 1, 1, 4)
    assert b.loop_config()["steps_per_graph"] == 4


@pytest.mark.parametrize("rows", [16, 8])
@pytest.mark.parametrize("arith", ["exact", "fast"])
def test_strip_form_equals_the_tile_form_bit_for_bit(arith, rows):
    tiles, strips = LoopApi(False, 0, arith), LoopApi(False, rows, arith)
    a, _ = cases.c1_small(tiles, t_end=900.0)
    b, _ = cases.c1_small(strips, t_end=900.0)
    assert strips.m.backend.loop_config()["strips"] == rows and tiles.m.backend.loop_config()["strips"] == 0
    for key in a:
        assert np.array_equal(np.asarray(a[key]), np.asarray(b[key])), key
