"""Make the golden vectors of the depth-area study's host arithmetic: run the reference's own functions on seeded
inputs.

Run in a container that holds the reference source tree (read-only is fine):

    WADI2D_REFERENCE=<the reference source tree> python tests/golden/make_golden_study.py

The reference's study module (wadi2d/arf.py) imports its I/O stack (rasterio, h5py and the products) at the top, which
this image does not have, so the script reads the module's source, takes the definitions of its pure numpy helpers
(``bracket_areas``, ``storm_areas``, ``run_name``, ``interpolate_peak``, ``_row``, ``interpolated_row``,
``log_area_weights``, ``composite_map``) and executes those alone, with numpy; ``storm_areas`` reads its job settings
from stand-in records with the same attribute names. It writes ``study.npz`` (inputs and outputs) and
``study.json`` (the interpolated design rows and the run names). Nothing on the GPU side reads the reference.
"""

from __future__ import annotations

import ast
import json
import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
if not os.environ.get("WADI2D_REFERENCE"):
    sys.exit("set WADI2D_REFERENCE to the reference source tree")
REF = Path(os.environ["WADI2D_REFERENCE"])
WANTED = ("bracket_areas", "storm_areas", "run_name", "interpolate_peak", "_row", "interpolated_row",
          "log_area_weights", "composite_map")  # fmt: skip


def reference_helpers() -> dict:
    src = (REF / "wadi2d" / "arf.py").read_text()
    tree = ast.parse(src)
    keep = [node for node in tree.body if isinstance(node, ast.FunctionDef) and node.name in WANTED]
    missing = set(WANTED) - {node.name for node in keep}
    if missing:
        raise SystemExit(f"not found in wadi2d/arf.py: {sorted(missing)}")
    module = ast.Module(body=keep, type_ignores=[])
    ns: dict = {"np": np, "__name__": "reference_arf_helpers"}
    exec(compile(module, str(REF / "wadi2d" / "arf.py"), "exec"), ns)  # noqa: S102 - the reference's own helpers
    return ns


def main() -> None:
    R = reference_helpers()
    rng = np.random.default_rng(31)
    out: dict[str, np.ndarray] = {}
    meta: dict[str, object] = {}

    # bracket_areas: (wanted, ratio, most)
    bracket_cases = [
        ([3.0, 40.0, 12.5], 2.0, 8),
        ([5.0, 5.0], 2.0, 8),
        ([1.0, 1000.0], 1.5, 6),
        ([0.7, 2.1], 3.0, 10),
        ([12.0, 13.0, 250.0, 90.0], 1.8, 12),
    ]
    meta["bracket"] = [
        {"wanted": w, "ratio": r, "most": m, "areas": [float(x) for x in R["bracket_areas"](w, r, m)]}
        for w, r, m in bracket_cases
    ]
    meta["run_names"] = {str(a): R["run_name"](a) for a in (0.5, 12.25, 1234.5678, 10.0)}

    # ArfTable.step_areas (wadi2d/storm/arf.py imports numpy only, so it is imported as it stands)
    sys.path.insert(0, str(REF))
    from wadi2d.storm.arf import ArfTable

    step_tables = [
        ([1.0, 10.0, 100.0, 1000.0], [1.0, 0.9, 0.75, 0.6], True),
        ([5.0, 20.0, 80.0], [0.95, 0.7, 0.8], True),  # a factor that rises again
        ([5.0, 20.0, 80.0], [0.9, 0.8, 0.6], False),  # the full depth below the table
    ]
    step_cases = [(0, 2.0, 500.0, 0.05), (0, 30.0, 40.0, 0.05), (0, 7.0, 7.0, 0.05), (1, 1.0, 200.0, 0.03),
                  (2, 1.0, 200.0, 0.04), (2, 10.0, 60.0, 0.5), (0, 0.5, 3000.0, 0.02)]  # fmt: skip
    meta["step_tables"] = step_tables
    meta["step_areas"] = [
        {"table": t, "low": lo, "high": hi, "step": st,
         "areas": ArfTable(np.array(step_tables[t][0]), np.array(step_tables[t][1]), step_tables[t][2]).step_areas(
             lo, hi, st)}
        for t, lo, hi, st in step_cases
    ]  # fmt: skip

    # storm_areas: the job's arf settings and design lines as stand-in records
    from types import SimpleNamespace as NS

    def cfg(lines, **arf):
        base = dict(areas_km2=[], n_areas=6, area_min_km2=10.0, area_max_km2=600.0, bracket=False, by_arf_step=False,
                    bracket_ratio=2.0, bracket_max=6, exact_points=False, arf_step_max=0.05)  # fmt: skip
        base.update(arf)
        outs = NS(lines=[NS(drainage_area_km2=a) for a in lines])
        return NS(arf=NS(**base), outputs=outs)

    area_cases = [
        ([3.3, None, 41.0], {}),
        ([3.3, 41.0], {"areas_km2": [5.0, 2.0, 5.00001, 80.0]}),
        ([3.3, 41.0], {"n_areas": 4, "area_min_km2": 0.1, "area_max_km2": 30.0}),
        ([3.3, None, 41.0, 12.0], {"bracket": True, "bracket_ratio": 1.7, "bracket_max": 9}),
        ([3.3, 41.0], {"bracket": True, "exact_points": True}),
        ([0.25, 0.2], {"n_areas": 6, "area_min_km2": 0.1, "area_max_km2": 30.0, "exact_points": True}),
    ]
    meta["storm_areas"] = [
        {"lines": lines, "arf": arf, "areas": [float(x) for x in R["storm_areas"](cfg(lines, **arf))]}
        for lines, arf in area_cases
    ]
    # by_arf_step: the module's arf_step_areas reads the job's storm table; here it reads the first step table
    step_table = ArfTable(np.array(step_tables[0][0]), np.array(step_tables[0][1]), step_tables[0][2])
    R["arf_step_areas"] = lambda job, low, high: step_table.step_areas(low, high, job.arf.arf_step_max)
    arf_step_cases = [
        ([3.3, None, 41.0], {"by_arf_step": True}),
        ([3.3, 410.0, 12.0], {"by_arf_step": True, "arf_step_max": 0.02, "exact_points": True}),
        ([3.3, 41.0], {"by_arf_step": True, "bracket": True}),  # the bracket rule comes first
    ]
    meta["storm_areas_by_step"] = [
        {"lines": lines, "arf": arf, "areas": [float(x) for x in R["storm_areas"](cfg(lines, **arf))]}
        for lines, arf in arf_step_cases
    ]

    # interpolate_peak and interpolated_row
    areas = np.geomspace(1.0, 300.0, 7)
    peaks = rng.uniform(5.0, 500.0, 7)
    peaks[2] = 0.0  # a dry run
    times = rng.uniform(1800.0, 20000.0, 7)
    queries = np.array([0.5, 1.0, 2.2, 5.0, 17.0, 80.0, 300.0, 900.0])
    out["ip_areas"], out["ip_peaks"], out["ip_times"], out["ip_queries"] = areas, peaks, times, queries
    out["ip_result"] = np.array([R["interpolate_peak"](areas, peaks, float(q)) for q in queries])
    out["ip_dry"] = np.array([R["interpolate_peak"](areas, np.zeros(7), 3.0)])
    meta["rows"] = [
        R["interpolated_row"](f"P{n}", float(q), areas, peaks, times, "storm-centred", "design line, 2D runs either side")
        for n, q in enumerate(queries)
    ]

    # log_area_weights and composite_map
    cell_area = np.exp(rng.uniform(np.log(0.3), np.log(600.0), (24, 32)))
    low, high, w = R["log_area_weights"](areas, cell_area)
    out["lw_cell_area"], out["lw_low"], out["lw_high"], out["lw_w"] = cell_area, low, high, w
    maps = [rng.uniform(0.0, 3.0, (24, 32)) for _ in range(areas.size)]
    out["cm_maps"] = np.stack(maps)
    out["cm_result"] = R["composite_map"](maps, areas, cell_area)
    out["cm_single"] = R["composite_map"](maps[:1], areas[:1], cell_area)

    np.savez_compressed(HERE / "study.npz", **out)
    (HERE / "study.json").write_text(json.dumps(meta, indent=1))
    print("wrote study.npz, study.json")


if __name__ == "__main__":
    main()
