"""The CUDA path against the FP64 run (oracle/fp64.py), with the step's accuracy bounds: configuration 1 at its full
size (256 x 256 cells, 5 x 5 pixels) after 200 steps, and the crest case after 100 steps. The FP64 run replays the
CUDA run's own dt sequence, so the two differ only by arithmetic precision."""

from __future__ import annotations

import pytest

import fp64_check as F
from product_api import B200Api

pytestmark = pytest.mark.gpu


def test_configuration1_within_the_accuracy_bounds_of_the_fp64_run():
    s32, dts = F.snapshots(B200Api(), (200,), n=256)
    s64 = F.fp64_snapshots(dts, (200,), n=256)
    r = F.compare(s32[200], s64[200])
    assert r["wet_set_identical"]
    assert r["depth_within"]
    assert r["discharge_within"], (r["fields"]["qx"], r["fields"]["qy"])
    assert r["tally_rel"] < 1e-6
    for name, e in r["fields"].items():
        assert e["rel_to_scale"] < 1e-4, (name, e)


def test_crest_case_blocked_faces_match_the_fp64_run():
    s32, dts = F.snapshots(B200Api(), (100,), case="crest")
    s64 = F.fp64_snapshots(dts, (100,), case="crest")
    r = F.compare(s32[100], s64[100], F.crest_faces())
    assert r["crest_blocked"] > 0
    assert r["crest_blocked_identical"]
    assert r["wet_set_identical"] and r["depth_within"] and r["discharge_within"]
