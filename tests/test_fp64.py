"""The FP64 run (oracle/fp64.py) against the float32 oracle, on the CPU: configuration 1 at 64 x 64 after 100 and
200 steps. The float32 oracle equals the reference bit for bit (tests/test_oracle_golden.py) and the CUDA path equals
the oracle (tests/test_gpu_parity.py); tests/test_gpu_fp64.py measures the CUDA path against the FP64 run directly."""

from __future__ import annotations

import numpy as np

import fp64_check as F
from oracle import fp64
from oracle_api import OracleApi

MARKS = (100, 200)


def test_float32_oracle_within_the_accuracy_bounds_of_the_fp64_run():
    s32, dts = F.snapshots(OracleApi(), MARKS, n=64)
    s64 = F.fp64_snapshots(dts, MARKS, n=64)
    for k in MARKS:
        r = F.compare(s32[k], s64[k])
        assert r["wet_set_identical"], k
        assert r["depth_within"], k
        assert r["discharge_within"], (k, r["fields"]["qx"], r["fields"]["qy"])
        assert r["tally_rel"] < 1e-6, k
        for name, e in r["fields"].items():
            assert e["rel_to_scale"] < 1e-4, (k, name, e)


def test_fp64_run_is_double_and_replays_the_given_steps():
    s32, dts = F.snapshots(OracleApi(), (20,), n=64)
    s64 = F.fp64_snapshots(dts, (20,), n=64)
    assert set(s64) == {20}
    # the two runs differ, but only by rounding
    assert not np.array_equal(s32[20]["h"], s64[20]["h"])
    assert fp64.field_errors(s32[20]["h"], s64[20]["h"])["rel_to_scale"] < 1e-5


def test_crest_case_blocked_faces_match_the_fp64_run():
    s32, dts = F.snapshots(OracleApi(), (100,), case="crest")
    s64 = F.fp64_snapshots(dts, (100,), case="crest")
    r = F.compare(s32[100], s64[100], F.crest_faces())
    assert r["crest_faces"] > 0 and r["crest_blocked"] > 0
    assert r["crest_blocked_identical"]
    assert r["wet_set_identical"] and r["depth_within"]
