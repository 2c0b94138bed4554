"""The oracle against the reference's own outputs: every table array, state array, step size, envelope entry and
tally bit for bit on the golden cases (tests/golden/make_golden.py ran the reference to make them)."""

from __future__ import annotations

import hashlib
import json
from pathlib import Path

import numpy as np
import pytest

import cases
from oracle import oracle as O
from oracle_api import OracleApi

GOLDEN = Path(__file__).resolve().parent / "golden"


def digest(a: np.ndarray) -> str:
    a = np.ascontiguousarray(a)
    return hashlib.sha256(a.dtype.str.encode() + str(a.shape).encode() + a.tobytes()).hexdigest()


@pytest.fixture(scope="module")
def runs():
    O.threads(0)
    out = {}
    for name, case in cases.CASES.items():
        api = OracleApi()
        arrays, ctx = case(api)
        arrays["dts"] = np.asarray(api.dts, np.float64)
        out[name] = (arrays, ctx)
    return out


@pytest.mark.parametrize("name", list(cases.CASES))
def test_inputs_and_tables_bit_exact(runs, name):
    meta = json.loads((GOLDEN / f"{name}.json").read_text())
    arrays, ctx = runs[name]
    assert digest(ctx["z"]) == meta["inputs"]["z"], "the seeded generator drifted"
    bad = [n for n, d in meta["tables"].items() if digest(ctx["tables"][n]) != d]
    assert not bad, f"tables differ from the reference: {bad}"


@pytest.mark.parametrize("name", list(cases.CASES))
def test_state_bit_exact(runs, name):
    gold = np.load(GOLDEN / f"{name}.npz")
    arrays, _ = runs[name]
    assert int(arrays["nsteps"]) == int(gold["nsteps"])
    assert np.array_equal(arrays["dts"], gold["dts"])
    assert float(arrays["t"]) == float(gold["t"]) and float(arrays["dt_next"]) == float(gold["dt_next"])
    for key in gold.files:
        if key.startswith(("state_", "max_")) or key in ("wet", "active"):
            assert np.array_equal(arrays[key], gold[key]), key
    if "tally" in gold.files:
        assert float(arrays["tally"]) == float(gold["tally"])


def test_fp64_helpers_bit_exact(runs):
    gold = np.load(GOLDEN / "c1_small.npz")
    _, ctx = runs["c1_small"]
    g, tab = ctx["grid"], ctx["tables"]
    hc, dtab = g.from_tiles(tab["hc"]), g.from_tiles(tab["dtab"])
    assert np.array_equal(O.level_of(gold["fp64_hb_in"], hc, dtab), gold["fp64_level"])
    assert np.array_equal(O.plan_of(gold["fp64_hb_in"], hc, dtab), gold["fp64_plan"])
    assert np.array_equal(O.hbar_at_level(gold["fp64_levels_in"], tab["zmin"], hc, dtab), gold["fp64_hbar"])
