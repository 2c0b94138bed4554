"""The GPU table builder against the reference's tables (pinned through the oracle, bit for bit to the reference):
every array within one float32 ulp, and the step on GPU-built tables within the step's accuracy tolerances of the
reference's run. CUDA's double cbrt and pow may round the last bit of a double differently from glibc's; a float32
table entry then differs by at most one ulp, and only rarely."""

from __future__ import annotations

import numpy as np
import pytest

import cases
from oracle_api import OracleApi
from product_api import B200Api
from test_gpu_parity import GOLDEN, _compare

pytestmark = pytest.mark.gpu

FIELDS = ("hc", "dtab", "flx", "frx", "glx", "grx", "efx", "cwx", "ftabx", "fly", "fry", "gly", "gry", "efy", "cwy",
          "ftaby", "zcx", "zcy", "zmin", "zbar")  # fmt: skip


def ulps(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """Distance in units in the last place (float32 by bit pattern; float64 by spacing)."""
    if b.dtype == np.float64:
        return np.abs(a - b) / np.maximum(np.spacing(np.abs(b)), 1e-300)
    ia = np.asarray(a, np.float32).view(np.int32).astype(np.int64)
    ib = np.asarray(b, np.float32).view(np.int32).astype(np.int64)
    return np.abs(ia - ib)


@pytest.mark.parametrize("name", list(cases.CASES))
def test_gpu_tables_match_reference_tables(name):
    og, targs, _ = cases.TABLE_INPUTS[name](OracleApi())
    ref = OracleApi().tables(og, *targs)
    api = B200Api(table_source="gpu")
    g, targs_g, _ = cases.TABLE_INPUTS[name](api)
    got = api.tables(g, *targs_g)
    for f in FIELDS:
        a, b = getattr(got, f), ref[f]
        assert a.shape == b.shape, f
        u = ulps(a, b)
        assert u.max() <= 1, (f, float(u.max()))
        assert np.count_nonzero(u) <= max(2, a.size // 100000), (f, int(np.count_nonzero(u)))


@pytest.mark.parametrize("name", list(cases.CASES))
def test_step_on_gpu_tables_matches_reference(name):
    gold = np.load(GOLDEN / f"{name}.npz")
    arrays, ctx = cases.CASES[name](B200Api(table_source="gpu", device_loop=True))
    _compare(ctx["grid"], arrays, gold)
