"""Golden vectors of the reference's loss, storm and ARF arithmetic (the parts of its forcing that import without
its GIS dependencies). Run where the reference tree is importable:

    WADI2D_REFERENCE=/root/reference PYTHONDONTWRITEBYTECODE=1 python tests/golden/make_golden_forcing.py

It writes tests/golden/forcing.npz: SCS cumulative excess over curve numbers x depths (with and without a given
initial abstraction), ARF table factors over areas (both ends' rules), and uniform-storm cumulative depths."""

from __future__ import annotations

import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, os.environ.get("WADI2D_REFERENCE", "/root/reference"))

from wadi2d.hydrology.losses import ScsCurveNumber  # noqa: E402
from wadi2d.storm.arf import ArfTable, GivenFactor, factor_at  # noqa: E402
from wadi2d.storm.uniform import UniformStorm  # noqa: E402


def main() -> None:
    cn = np.array([45.0, 60.0, 72.5, 80.0, 88.0, 95.0, 99.0])
    depth = np.concatenate(([0.0, 1e-3, 0.5], np.linspace(0.0, 400.0, 57)[1:]))
    scs = np.stack([ScsCurveNumber(curve_number=c).cumulative_excess(depth) for c in cn])
    scs_ia = np.stack([ScsCurveNumber(curve_number=c, initial_abstraction_mm=7.5).cumulative_excess(depth) for c in cn])
    areas = np.array([1.0, 10.0, 50.0, 100.0, 500.0, 2000.0])
    factors = np.array([0.99, 0.95, 0.9, 0.86, 0.78, 0.7])
    probe = np.array([0.2, 1.0, 3.3, 10.0, 77.7, 100.0, 1234.5, 2000.0, 5000.0])
    arf_a = np.array([ArfTable(areas, factors).factor(a) for a in probe])
    arf_b = np.array([ArfTable(areas, factors, reduces_below_table=False).factor(a) for a in probe])
    given = np.array([factor_at(GivenFactor(0.8), a) for a in probe])
    minutes = np.linspace(-10.0, 200.0, 43)
    uni = UniformStorm(85.0, 150.0, 77.7, ArfTable(areas, factors)).cumulative_depth(minutes)
    np.savez_compressed(HERE / "forcing.npz", cn=cn, depth=depth, scs=scs, scs_ia=scs_ia, areas=areas,
                        factors=factors, probe=probe, arf_a=arf_a, arf_b=arf_b, given=given, minutes=minutes,
                        uniform=uni)  # fmt: skip
    print("forcing.npz written")


if __name__ == "__main__":
    main()
