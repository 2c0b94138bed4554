"""The exact-solution cases of tests/test_gpu_validation.py with their numbers (test infrastructure; run on a machine
with a B200, from the repository root: ``python tests/validation_report.py``): one JSON line a case."""

from __future__ import annotations

import json
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
sys.path[:0] = [str(HERE.parent), str(HERE)]

import test_gpu_validation as V  # noqa: E402


def main() -> None:
    for axis in ("x", "y"):
        d, q, f, v = V._dam_break(axis, 2.0, 0.5)
        print(json.dumps({"case": f"Stoker dam break along {axis}", "depth_rmse": d, "depth_limit": 0.02,
                          "discharge_rmse": q, "discharge_limit": 0.07, "volume_error": v, "volume_limit": 1e-6}))
    d, q, f, v = V._dam_break("x", 2.0, 0.0)
    print(json.dumps({"case": "Ritter dam break", "depth_rmse": d, "depth_limit": 0.01, "f_statistic": f,
                      "f_limit": 0.93, "volume_error": v, "volume_limit": 1e-6}))
    for kind, limit in (("planar", 0.0055), ("curved", 0.002)):
        d, v = V._thacker(kind)
        print(json.dumps({"case": f"Thacker {kind}", "depth_rmse": d, "depth_limit": limit, "volume_error": v,
                          "volume_limit": 5e-5}))


if __name__ == "__main__":
    main()
