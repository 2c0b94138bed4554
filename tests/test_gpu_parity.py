"""The CUDA path against the reference's own outputs (the golden cases) and against the oracle.

Tolerances: the wet set and the active tiles identical; depth within 1e-5 m absolute; unit discharge and velocity
within 1e-4 relative of the field's scale. The arithmetic is the reference CPU twin's statement
for statement, so the step count and every dt are expected to match exactly, and they are asserted so.
"""

from __future__ import annotations

import numpy as np
import pytest

import cases
from product_api import B200Api
from wadi2d_b200.state import from_state

GOLDEN = __import__("pathlib").Path(__file__).resolve().parent / "golden"
pytestmark = pytest.mark.gpu

H_ABS = 1e-5
REL = 1e-4


def _compare(grid, arrays, gold):
    assert int(arrays["nsteps"]) == int(gold["nsteps"])
    assert float(arrays["t"]) == pytest.approx(float(gold["t"]), abs=1e-9)
    assert float(arrays["dt_next"]) == float(gold["dt_next"])
    assert np.array_equal(np.sort(arrays["active"]), np.sort(gold["active"]))
    own = lambda a: from_state(grid, a)  # noqa: E731
    h, hg = own(arrays["state_h"]), own(gold["state_h"])
    assert np.array_equal(h > 0, hg > 0), "wet set differs"
    assert np.abs(h - hg).max() <= H_ABS
    assert np.abs(own(arrays["state_d"]) - own(gold["state_d"])).max() <= H_ABS
    for name in ("u", "v", "mx", "my", "qx", "qy", "res", "om"):
        a, b = own(arrays[f"state_{name}"]), own(gold[f"state_{name}"])
        scale = max(float(np.abs(b).max()), 1e-6)
        assert np.abs(a - b).max() <= REL * scale, name
    wet_t = np.asarray(arrays["wet"])[np.sort(gold["active"])]
    assert np.array_equal(wet_t, np.asarray(gold["wet"])[np.sort(gold["active"])])
    for key in gold.files:
        if key.startswith("max_"):
            a, b = own(arrays[key]), own(gold[key])
            scale = max(float(np.abs(b).max()), 1e-6)
            assert np.abs(a - b).max() <= REL * scale, key
    if "tally" in gold.files:
        assert float(arrays["tally"]) == pytest.approx(float(gold["tally"]), rel=1e-7)


@pytest.mark.parametrize("name", list(cases.CASES))
def test_host_loop_matches_reference(name):
    gold = np.load(GOLDEN / f"{name}.npz")
    api = B200Api()
    arrays, ctx = cases.CASES[name](api)
    assert np.array_equal(np.asarray(api.dts), gold["dts"]), "dt sequence differs"
    _compare(ctx["grid"], arrays, gold)


def test_host_loop_bit_exact_on_c1():
    """With the reference's tables, the float32 step reproduces the reference's bits."""
    gold = np.load(GOLDEN / "c1_small.npz")
    arrays, ctx = cases.c1_small(B200Api())
    g = ctx["grid"]
    for name in ("h", "d", "u", "v", "mx", "my", "qx", "qy", "res", "om"):
        assert np.array_equal(from_state(g, arrays[f"state_{name}"]), from_state(g, gold[f"state_{name}"])), name


@pytest.mark.parametrize("name", list(cases.CASES))
def test_device_loop_matches_reference(name):
    """The graph-captured device loop (dt rule, sleeping tiles, envelope, tally on the device) gives the host loop's
    result."""
    gold = np.load(GOLDEN / f"{name}.npz")
    arrays, ctx = cases.CASES[name](B200Api(device_loop=True))
    _compare(ctx["grid"], arrays, gold)
