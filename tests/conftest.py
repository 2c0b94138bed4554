"""pytest configuration: the ``gpu`` marker, and the repository root on the import path."""

from __future__ import annotations

import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]
for p in (str(ROOT), str(ROOT / "tests" / "golden")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (a B200); runs the sm_100a path")
    config.addinivalue_line("markers", "slow: takes more than a few seconds")
