"""``momentum.FaceKick`` on the CPU: repeated faces merged by an FP64 sum then rounded to float32, and ``apply`` as one
float32 indexed add an axis (m += float32(dt) * rate), checked on a stand-in backend of numpy arrays. With
WADI2D_REFERENCE naming the reference's source tree, the same kicks are built and applied by the reference's own
FaceKick (wadi2d/solver/momentum.py:18-54) and compared bit for bit."""

from __future__ import annotations

import importlib
import os
import sys
from types import SimpleNamespace

import numpy as np
import pytest

from wadi2d_b200.momentum import FaceKick

REF = os.environ.get("WADI2D_REFERENCE")


def _cases():
    rng = np.random.default_rng(7)
    fx = rng.integers(0, 50, size=40)  # repeats likely
    fy = rng.integers(0, 50, size=25)
    yield fx, rng.standard_normal(40).astype(np.float32), fy, rng.standard_normal(25).astype(np.float32)
    yield fx, 0.37, np.zeros(0, np.int64), np.zeros(0, np.float32)  # one rate for every face; no y faces
    yield np.array([3, 3, 3]), np.array([1e-3, 1e3, -1e3], np.float32), np.array([9]), np.array([2.5], np.float32)


def _backend(n=64, seed=0):
    rng = np.random.default_rng(seed)
    return SimpleNamespace(mx=rng.standard_normal(n).astype(np.float32), my=rng.standard_normal(n).astype(np.float32))


def test_build_merges_repeated_faces_by_an_fp64_sum():
    fx, rx, fy, ry = next(_cases())
    k = FaceKick.build(fx, rx, fy, ry)
    for faces, rate, kf, kr in ((fx, rx, k.faces_x, k.rate_x), (fy, ry, k.faces_y, k.rate_y)):
        assert kf.dtype == np.int64 and kr.dtype == np.float32
        np.testing.assert_array_equal(kf, np.unique(faces))
        want = [np.float32(sum(float(r) for f, r in zip(faces, rate, strict=True) if f == u)) for u in kf]
        np.testing.assert_array_equal(kr, np.array(want, np.float32))


def test_apply_adds_dt_times_rate_in_float32_once_a_face():
    fx, rx, fy, ry = next(_cases())
    k = FaceKick.build(fx, rx, fy, ry)
    b = _backend()
    mx0, my0 = b.mx.copy(), b.my.copy()
    k.apply(b, 0.75)
    want_x, want_y = mx0.copy(), my0.copy()
    want_x[k.faces_x] = mx0[k.faces_x] + np.float32(0.75) * k.rate_x
    want_y[k.faces_y] = my0[k.faces_y] + np.float32(0.75) * k.rate_y
    np.testing.assert_array_equal(b.mx, want_x)
    np.testing.assert_array_equal(b.my, want_y)
    assert k.on(b) is k  # the B200 backend takes host index arrays


@pytest.mark.skipif(not REF, reason="WADI2D_REFERENCE (the reference source tree) is not set")
def test_build_and_apply_equal_the_references_face_kick(monkeypatch):
    monkeypatch.syspath_prepend(REF)
    for name in [n for n in sys.modules if n == "wadi2d" or n.startswith("wadi2d.")]:
        monkeypatch.delitem(sys.modules, name)
    theirs = importlib.import_module("wadi2d.solver.momentum").FaceKick
    try:
        for fx, rx, fy, ry in _cases():
            mine, ref = FaceKick.build(fx, rx, fy, ry), theirs.build(fx, rx, fy, ry)
            for a in ("faces_x", "rate_x", "faces_y", "rate_y"):
                x, y = getattr(mine, a), getattr(ref, a)
                assert x.dtype == y.dtype, a
                np.testing.assert_array_equal(x, y)
            b1, b2 = _backend(seed=1), _backend(seed=1)
            mine.apply(b1, 0.3)
            ref.apply(b2, 0.3)
            np.testing.assert_array_equal(b1.mx, b2.mx)
            np.testing.assert_array_equal(b1.my, b2.my)
    finally:
        for name in [n for n in sys.modules if n == "wadi2d" or n.startswith("wadi2d.")]:
            del sys.modules[name]
