"""The step's float cube root against the reference's formulation (the cube root rounded through double, as Numba's
float32 np.cbrt is formed) on every positive finite float: they must agree bit for bit."""

from __future__ import annotations

import pytest

pytestmark = pytest.mark.gpu


def test_cbrt_matches_double_rounded_cube_root_on_every_positive_float():
    import torch

    from wadi2d_b200 import _lib

    out = torch.zeros(5, dtype=torch.int64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    first, last = 0x00000001, 0x7F7FFFFF  # the smallest subnormal to the largest finite float
    _lib.call("w2b_selftest_cbrt", first, last - first + 1, out.data_ptr(), stream)
    torch.cuda.synchronize()
    res = out.cpu().tolist()
    assert res[0] == 0, f"{res[0]} mismatches, e.g. bit patterns {[hex(v) for v in res[1:1 + min(res[0], 4)]]}"
