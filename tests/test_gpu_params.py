"""Replacing a handle's kernel constants (w2b_set_params) and reading its cell size (w2b_cell_size): the constants a
handle is made with read back, a replacement takes effect, and other constants set halfway through a run and the
first ones put back give the run that was never changed, bit for bit (the device loop captures its graphs again)."""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

import cases
from product_api import B200Api
from wadi2d_b200 import _lib

pytestmark = pytest.mark.gpu


def _cell_size(backend) -> float:
    dx = ctypes.c_float()
    _lib.call("w2b_cell_size", backend.handle, ctypes.byref(dx))
    return dx.value


class ParamsApi(B200Api):
    """The case API with the device loop, each run advanced to half its end and then to its end; ``swap`` sets other
    constants at the half and puts the first ones back."""

    def __init__(self, swap: bool) -> None:
        super().__init__(device_loop=True)
        self.swap = swap

    def model(self, grid, tables, numerics):
        m = super().model(grid, tables, numerics)
        b = m.backend
        first = b._params
        assert _cell_size(b) == np.float32(first.dx)
        advance = m.advance

        def halves(t_end, on_step=None):
            advance(0.5 * t_end, on_step)
            if self.swap:
                other = _lib.Params.from_buffer_copy(first)
                other.dx = 2.0 * first.dx
                other.g = 1.5 * first.g
                _lib.call("w2b_set_params", b.handle, ctypes.byref(other))
                assert _cell_size(b) == np.float32(2.0 * first.dx)
                _lib.call("w2b_set_params", b.handle, ctypes.byref(first))
                assert _cell_size(b) == np.float32(first.dx)
            return advance(t_end, on_step)

        m.advance = halves
        return m


def test_constants_put_back_give_the_unchanged_run():
    a, _ = cases.c1_small(ParamsApi(True), t_end=300.0)
    b, _ = cases.c1_small(ParamsApi(False), t_end=300.0)
    assert int(a["nsteps"]) > 0
    for key in a:
        assert np.array_equal(np.asarray(a[key]), np.asarray(b[key])), key


def test_replaced_constants_take_effect():
    """Gravity halved: the same run takes other steps (the wave speed, hence the step, depends on g)."""

    class Halved(B200Api):
        def __init__(self) -> None:
            super().__init__(device_loop=True)

        def model(self, grid, tables, numerics):
            m = super().model(grid, tables, numerics)
            p = _lib.Params.from_buffer_copy(m.backend._params)
            p.g = 0.5 * p.g
            _lib.call("w2b_set_params", m.backend.handle, ctypes.byref(p))
            return m

    a, _ = cases.c1_small(Halved(), t_end=300.0)
    b, _ = cases.c1_small(ParamsApi(False), t_end=300.0)
    assert any(not np.array_equal(np.asarray(a[k]), np.asarray(b[k])) for k in a)
