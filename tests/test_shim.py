"""The drop-in shim on a stand-in Wadi2D package (no reference needed): backend selection is routed, the monitor's
envelope and tally classes are swapped only for B200 models, and uninstall restores the originals."""

from __future__ import annotations

import sys
import types

import pytest


@pytest.fixture
def fake_wadi2d(monkeypatch):
    calls = []

    def select_backend(name, tables, num):
        calls.append(name)
        return ("reference", name)

    pkg = types.ModuleType("wadi2d")
    solver = types.ModuleType("wadi2d.solver")
    model = types.ModuleType("wadi2d.solver.model")
    model.select_backend = select_backend
    engine = types.ModuleType("wadi2d.engine")
    monitor = types.ModuleType("wadi2d.engine.monitor")

    class RefMaxima:
        def __init__(self, m, *a):
            self.kind = "reference"

    monitor.Maxima = RefMaxima
    monitor.Tally = RefMaxima
    limiter_log = types.ModuleType("wadi2d.engine.step_limiter")
    limiter_log.step_limiter = lambda m, tables=None: "reference reading"
    for name, mod in (("wadi2d", pkg), ("wadi2d.solver", solver), ("wadi2d.solver.model", model),
                      ("wadi2d.engine", engine), ("wadi2d.engine.monitor", monitor),
                      ("wadi2d.engine.step_limiter", limiter_log)):  # fmt: skip
        monkeypatch.setitem(sys.modules, name, mod)
    return model, monitor, calls, limiter_log


def test_install_routes_and_uninstall_restores(fake_wadi2d, monkeypatch):
    from wadi2d_b200 import shim

    model, monitor, calls, limiter_log = fake_wadi2d
    original = model.select_backend
    original_limiter = limiter_log.step_limiter
    monkeypatch.setattr(shim, "_b200_available", lambda: False)
    shim.install()
    try:
        assert model.select_backend("cpu", None, None) == ("reference", "cpu")
        assert model.select_backend("auto", None, None) == ("reference", "auto")  # no B200: the reference's choice
        m = types.SimpleNamespace(backend=object())
        assert monitor.Maxima(m).kind == "reference"  # a reference model keeps the reference's envelope
        assert limiter_log.step_limiter(m) == "reference reading"  # and the reference's limiter reading
        assert limiter_log.step_limiter is not original_limiter
        from wadi2d_b200.backend import NumericsRecord

        num = NumericsRecord(9.80665, 10.0, 1e-4, 0.01, 25.0, 8.0, 0.02, True, True, True)
        with pytest.raises(RuntimeError):
            model.select_backend("b200", None, num)  # asked for explicitly, fails loudly without a device
    finally:
        shim.uninstall()
    assert model.select_backend is original
    assert limiter_log.step_limiter is original_limiter
    assert calls == ["cpu", "auto"]
