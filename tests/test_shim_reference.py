"""The drop-in shim against the reference package itself, on the CPU: ``shim.install()`` reaches the reference's own
hook points, and every backend member the reference's Model and Stepper use exists on ``B200Backend``.

It needs the reference's Python source tree, named by the environment variable WADI2D_REFERENCE (the same variable
the golden generators read); without it the test is skipped. No backend is built (that needs a GPU): the checks are
of names, signatures and the routing itself."""

from __future__ import annotations

import importlib
import inspect
import os
import re
import sys
from pathlib import Path

import pytest

REF = os.environ.get("WADI2D_REFERENCE")
pytestmark = pytest.mark.skipif(not REF, reason="WADI2D_REFERENCE (the reference source tree) is not set")


@pytest.fixture
def reference(monkeypatch):
    """The reference's modules imported from its tree, and forgotten afterwards."""
    monkeypatch.syspath_prepend(REF)
    for name in [n for n in sys.modules if n == "wadi2d" or n.startswith("wadi2d.")]:
        monkeypatch.delitem(sys.modules, name)
    yield importlib.import_module("wadi2d.solver.model")
    from wadi2d_b200 import shim

    shim.uninstall()
    for name in [n for n in sys.modules if n == "wadi2d" or n.startswith("wadi2d.")]:
        del sys.modules[name]


def test_install_routes_the_references_backend_choice_and_uninstall_restores_it(reference):
    from wadi2d_b200 import shim

    model = reference
    original = model.select_backend
    # Model looks select_backend up as a module global at construction (wadi2d/solver/model.py:38), so replacing the
    # module's name routes every new Model
    assert "select_backend" in model.Model.__init__.__code__.co_names
    shim.install(auto=False)
    assert model.select_backend is not original
    assert list(inspect.signature(model.select_backend).parameters) == ["name", "tables", "num"]
    shim.uninstall()
    assert model.select_backend is original


def test_the_monitor_and_the_limiter_log_hooks_match_the_references_signatures(reference):
    from wadi2d_b200 import shim
    from wadi2d_b200.maxima import Maxima, Tally

    theirs = importlib.import_module("wadi2d.engine.maxima")
    for name, mine in (("Maxima", Maxima), ("Tally", Tally)):
        want = list(inspect.signature(getattr(theirs, name).__init__).parameters)[1:]
        got = list(inspect.signature(mine.__init__).parameters)[1:]
        assert len(got) >= len(want), (name, want, got)  # ours take the reference's arguments by position
    limiter = importlib.import_module("wadi2d.solver.limiter")
    assert list(inspect.signature(limiter.step_limiter).parameters) == ["model", "tables"]
    try:
        monitor = importlib.import_module("wadi2d.engine.monitor")
    except ImportError:  # the run driver's optional readers (rasterio, h5py) are absent: the shim skips it too
        monitor = None
    shim.install(auto=False)
    if monitor is not None:
        assert monitor.Maxima is not theirs.Maxima and monitor.Tally is not theirs.Tally
    shim.uninstall()
    if monitor is not None:
        assert monitor.Maxima is theirs.Maxima and monitor.Tally is theirs.Tally


def test_b200_backend_has_every_member_the_references_model_and_stepper_use(reference):
    from wadi2d_b200.backend import STATE, B200Backend, NumericsRecord

    used = set()
    for mod in ("wadi2d/solver/model.py", "wadi2d/solver/stepper.py"):
        src = (Path(REF) / mod).read_text()
        used |= set(re.findall(r"(?:self\.backend|backend|\bb)\.(\w+)", src))
    optional = {"cp"}  # looked up with hasattr: a backend without CuPy takes the host path
    assigned = set(re.findall(r"self\.(\w+)\s*=", inspect.getsource(B200Backend)))  # instance attributes
    missing = sorted(n for n in used - optional if not hasattr(B200Backend, n) and n not in set(STATE) | assigned)
    assert not missing, missing
    # the shim builds this package's NumericsRecord from the reference's: every field it needs is one of theirs
    ref_record = importlib.import_module("wadi2d.solver.backend").NumericsRecord
    assert set(NumericsRecord.__dataclass_fields__) - {"level_fp64", "arith"} <= set(ref_record.__dataclass_fields__)
