"""The step's fast build (``Numerics.arithmetic = "fast"``: FMA contraction and the hardware's approximate division,
square root and cube root in the face pass) against the FP64 run and against the reference's golden outputs, with
the step's accuracy bounds. The exact build is pinned to the reference's bits (test_gpu_parity.py); the fast build is
pinned by the bounds: the wet set and the crest-blocked faces identical, depth within 1e-4 relative or 1e-5 m, unit
discharge within 1e-4 of its field's scale."""

from __future__ import annotations

import numpy as np
import pytest

import cases
import fp64_check as F
from product_api import B200Api
from wadi2d_b200.state import from_state

GOLDEN = __import__("pathlib").Path(__file__).resolve().parent / "golden"
pytestmark = pytest.mark.gpu

H_ABS = 1e-5
REL = 1e-4


def test_fast_configuration1_within_the_accuracy_bounds_of_the_fp64_run():
    s32, dts = F.snapshots(B200Api(arith="fast"), (200,), n=256)
    s64 = F.fp64_snapshots(dts, (200,), n=256)
    r = F.compare(s32[200], s64[200])
    assert r["wet_set_identical"]
    assert r["depth_within"]
    assert r["discharge_within"], (r["fields"]["qx"], r["fields"]["qy"])
    assert r["tally_rel"] < 1e-6
    for name, e in r["fields"].items():
        assert e["rel_to_scale"] < 1e-4, (name, e)


def test_fast_crest_case_blocked_faces_match_the_fp64_run():
    s32, dts = F.snapshots(B200Api(arith="fast"), (100,), case="crest")
    s64 = F.fp64_snapshots(dts, (100,), case="crest")
    r = F.compare(s32[100], s64[100], F.crest_faces())
    assert r["crest_blocked"] > 0
    assert r["crest_blocked_identical"]
    assert r["wet_set_identical"] and r["depth_within"] and r["discharge_within"]


@pytest.mark.parametrize("loop", [False, True], ids=["host_loop", "device_loop"])
@pytest.mark.parametrize("name", list(cases.CASES))
def test_fast_build_within_tolerance_of_the_reference(name, loop):
    """The golden cases through the fast build: the same end time, the step count within one step, the wet set
    identical, depth within 1e-5 m, the other fields and the envelope within 1e-4 of their scale."""
    gold = np.load(GOLDEN / f"{name}.npz")
    arrays, ctx = cases.CASES[name](B200Api(arith="fast", device_loop=loop))
    grid = ctx["grid"]
    assert abs(int(arrays["nsteps"]) - int(gold["nsteps"])) <= 1
    assert float(arrays["t"]) == pytest.approx(float(gold["t"]), abs=1e-6)
    own = lambda a: from_state(grid, a)  # noqa: E731
    h, hg = own(arrays["state_h"]), own(gold["state_h"])
    assert np.array_equal(h > 0, hg > 0), "wet set differs"
    assert np.abs(h - hg).max() <= H_ABS
    assert np.abs(own(arrays["state_d"]) - own(gold["state_d"])).max() <= H_ABS
    for key in ("u", "v", "mx", "my", "qx", "qy"):
        a, b = own(arrays[f"state_{key}"]), own(gold[f"state_{key}"])
        assert np.abs(a - b).max() <= REL * max(float(np.abs(b).max()), 1e-6), key
    for key in gold.files:
        if key.startswith("max_"):
            a, b = own(arrays[key]), own(gold[key])
            assert np.abs(a - b).max() <= REL * max(float(np.abs(b).max()), 1e-6), key
    if "tally" in gold.files:
        assert float(arrays["tally"]) == pytest.approx(float(gold["tally"]), rel=1e-5)


def test_fast_build_differs_from_the_exact_build():
    """The switch reaches the kernels: the fast build's fields are not the exact build's bits (and both are within
    the bounds above)."""
    a, ctx = cases.c1_small(B200Api(arith="exact"))
    b, _ = cases.c1_small(B200Api(arith="fast"))
    g = ctx["grid"]
    assert not np.array_equal(from_state(g, a["state_qx"]), from_state(g, b["state_qx"]))
