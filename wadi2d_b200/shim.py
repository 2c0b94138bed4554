"""Install the B200 backend into an importable Wadi2D (the reference package), without editing it.

``install()`` wraps ``wadi2d.solver.model.select_backend`` (which ``Model`` imported by name from
wadi2d/solver/backend.py:58-75) so that ``"b200"``, and ``"auto"``/``"gpu"`` when a CUDA device is present, return a
``B200Backend``; it replaces ``wadi2d.engine.monitor.Maxima`` and ``Tally`` (wadi2d/engine/maxima.py:103-192) with
this package's device versions when the model's backend is a B200 one; and it routes the run monitor's step-limiter
reading (``step_limiter`` as wadi2d/engine/step_limiter.py:15 imported it) to ``wadi2d_b200.limiter`` for B200
models. ``uninstall()`` restores the originals.
"""

from __future__ import annotations

import importlib

_saved: dict = {}


def _b200_available() -> bool:
    try:
        import torch

        return bool(torch.cuda.is_available())
    except Exception:
        return False


def install(auto: bool = True) -> None:
    """Route backend selection and the run monitor's envelope/tally through this package."""
    from wadi2d_b200.backend import B200Backend, NumericsRecord
    from wadi2d_b200.maxima import Maxima as B200Maxima
    from wadi2d_b200.maxima import Tally as B200Tally

    model = importlib.import_module("wadi2d.solver.model")
    if "select_backend" not in _saved:
        _saved["select_backend"] = model.select_backend
    original = _saved["select_backend"]

    def select_backend(name, tables, num):
        if name == "b200" or (auto and name in ("auto", "gpu") and _b200_available()):
            fields = {f: getattr(num, f) for f in NumericsRecord.__dataclass_fields__ if hasattr(num, f)}
            return B200Backend(tables, NumericsRecord(**fields))
        return original(name, tables, num)

    model.select_backend = select_backend
    try:
        monitor = importlib.import_module("wadi2d.engine.monitor")
    except Exception:  # the run driver's optional dependencies may be absent
        return
    for name, mine in (("Maxima", B200Maxima), ("Tally", B200Tally)):
        if name not in _saved:
            _saved[name] = getattr(monitor, name)
        theirs = _saved[name]

        def make(theirs=theirs, mine=mine):
            def factory(model_, *args, **kwargs):
                if isinstance(getattr(model_, "backend", None), B200Backend):
                    return mine(model_, *args, **kwargs)
                return theirs(model_, *args, **kwargs)

            return factory

        setattr(monitor, name, make())
    try:
        logmod = importlib.import_module("wadi2d.engine.step_limiter")
    except Exception:  # the limiter log's optional dependencies may be absent
        return
    if "step_limiter" not in _saved:
        _saved["step_limiter"] = logmod.step_limiter
    theirs = _saved["step_limiter"]

    def step_limiter(model_, tables=None):
        if isinstance(getattr(model_, "backend", None), B200Backend):
            from wadi2d_b200.limiter import step_limiter as mine

            return mine(model_, tables)
        return theirs(model_, tables)

    logmod.step_limiter = step_limiter


def uninstall() -> None:
    if "select_backend" in _saved:
        importlib.import_module("wadi2d.solver.model").select_backend = _saved.pop("select_backend")
    try:
        monitor = importlib.import_module("wadi2d.engine.monitor")
    except Exception:
        return
    for name in ("Maxima", "Tally"):
        if name in _saved:
            setattr(monitor, name, _saved.pop(name))
    try:
        logmod = importlib.import_module("wadi2d.engine.step_limiter")
    except Exception:
        return
    if "step_limiter" in _saved:
        logmod.step_limiter = _saved.pop("step_limiter")
