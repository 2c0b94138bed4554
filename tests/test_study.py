"""The depth-area study's readings against the reference's own functions (tests/golden/make_golden_study.py ran
wadi2d/arf.py's helpers on these inputs): storm areas, run names, interpolated peaks and design rows, log-area weights
and composite maps."""

from __future__ import annotations

import json
from pathlib import Path

import numpy as np
import pytest

from wadi2d_b200 import study as S

GOLD = Path(__file__).resolve().parent / "golden"


@pytest.fixture(scope="module")
def gold():
    return np.load(GOLD / "study.npz"), json.loads((GOLD / "study.json").read_text())


def test_bracket_areas_and_run_names(gold):
    _, meta = gold
    for case in meta["bracket"]:
        assert S.bracket_areas(case["wanted"], case["ratio"], case["most"]) == case["areas"]
    for area, name in meta["run_names"].items():
        assert S.run_name(float(area)) == name


def test_interpolated_peaks_and_rows(gold):
    g, meta = gold
    got = np.array([S.interpolate_peak(g["ip_areas"], g["ip_peaks"], float(q)) for q in g["ip_queries"]])
    assert np.array_equal(got, g["ip_result"])
    assert S.interpolate_peak(g["ip_areas"], np.zeros(7), 3.0) == float(g["ip_dry"][0])
    for n, (q, row) in enumerate(zip(g["ip_queries"], meta["rows"], strict=True)):
        mine = S.interpolated_row(f"P{n}", float(q), g["ip_areas"], g["ip_peaks"], g["ip_times"], "storm-centred",
                                  S.READ_LINE)  # fmt: skip
        assert mine == row
        assert list(mine) == list(row)  # the CSV's column order


def test_design_table_reads_each_line(gold):
    g, meta = gold
    peaks = np.stack([g["ip_peaks"], g["ip_peaks"] * 7.0, g["ip_peaks"] * 2.0], axis=1)  # a column a line
    times = np.stack([g["ip_times"]] * 3, axis=1)
    rows = S.design_table(["P2", "skip", "P2b"], [2.2, None, 2.2], g["ip_areas"], peaks, times, "storm-centred")
    assert [r["design_point"] for r in rows] == ["P2", "P2b"]
    assert rows[0] == meta["rows"][2]
    assert rows[1]["design_peak_m3s"] == pytest.approx(2.0 * rows[0]["design_peak_m3s"], rel=1e-12)


def test_log_area_weights_and_composites(gold):
    g, _ = gold
    low, high, w = S.log_area_weights(g["ip_areas"], g["lw_cell_area"])
    assert np.array_equal(low, g["lw_low"]) and np.array_equal(high, g["lw_high"])
    assert np.array_equal(w, g["lw_w"])
    maps = list(g["cm_maps"])
    assert np.array_equal(S.composite_map(maps, g["ip_areas"], g["lw_cell_area"]), g["cm_result"])
    assert np.array_equal(S.composite_map(maps[:1], g["ip_areas"][:1], g["lw_cell_area"]), g["cm_single"])


def test_composites_from_envelopes_with_a_depth_floor():
    rng = np.random.default_rng(2)
    envs = [{k: rng.uniform(0.0, 1.0, (4, 5)) for k in ("depth", "speed", "hazard")} for _ in range(3)]
    areas = [1.0, 4.0, 16.0]
    cell = np.full((4, 5), 2.0)
    out = S.composite_maps(envs, areas, cell, depth_floor=0.5)
    w = np.log(2.0) / np.log(4.0)
    for name, field in S.ENVELOPE_OF_MAP.items():
        a = np.where(envs[0]["depth"] < 0.5, 0.0, envs[0][field])
        b = np.where(envs[1]["depth"] < 0.5, 0.0, envs[1][field])
        assert np.allclose(out[name], (1 - w) * a + w * b, rtol=0, atol=1e-15)


def test_storm_areas(gold):
    _, meta = gold
    for case in meta["storm_areas"]:
        assert S.storm_areas(case["lines"], **case["arf"]) == case["areas"], case
    with pytest.raises(ValueError):
        S.storm_areas([None], bracket=True)


def test_arf_step_areas_and_the_by_step_placement(gold):
    from wadi2d_b200.forcing import ArfTable

    _, meta = gold
    tables = [ArfTable(np.array(a), np.array(f), r) for a, f, r in meta["step_tables"]]
    for case in meta["step_areas"]:
        assert tables[case["table"]].step_areas(case["low"], case["high"], case["step"]) == case["areas"], case
    with pytest.raises(ValueError):
        tables[0].step_areas(1.0, 2.0, 0.0)
    for case in meta["storm_areas_by_step"]:
        assert S.storm_areas(case["lines"], table=tables[0], **case["arf"]) == case["areas"], case
    with pytest.raises(ValueError):
        S.storm_areas([3.0, 9.0], by_arf_step=True)  # no table to place the areas by


def test_a_study_refuses_storms_that_make_identical_runs():
    from wadi2d_b200.forcing import ArfTable, GivenFactor, UniformStorm

    table = ArfTable(np.array([1.0, 10.0, 100.0]), np.array([1.0, 0.9, 0.7]))
    S.check_study(UniformStorm(50.0, 60.0, arf=table), [2.0, 20.0])
    for storm in (UniformStorm(50.0, 60.0), UniformStorm(50.0, 60.0, arf=GivenFactor(0.8))):
        with pytest.raises(ValueError):
            S.check_study(storm, [2.0, 20.0])
    flat = ArfTable(np.array([1.0, 10.0]), np.array([0.8, 0.8]))
    with pytest.raises(ValueError):
        S.check_study(UniformStorm(50.0, 60.0, arf=flat), [2.0, 5.0])
    S.check_study(UniformStorm(50.0, 60.0, arf=flat), [2.0])  # one area: one run


def test_study_outputs_in_the_reference_layout(tmp_path, gold):
    import csv

    g, meta = gold
    rows = [meta["rows"][2], meta["rows"][4]]
    res = S.StudyResult([1.0, 3.0], np.zeros((2, 2)), np.zeros((2, 2)), rows,
                        {"max_depth": np.ones((3, 4)), "max_speed": np.zeros((3, 4)), "hazard": np.zeros((3, 4))},
                        np.array([5, 6]), 0.0)  # fmt: skip
    paths = S.write_study(tmp_path / "study1", res, "storm-centred")
    with open(paths["table"], newline="", encoding="utf-8") as f:
        back = list(csv.DictReader(f))
    assert list(back[0]) == list(rows[0])
    assert [float(r["design_peak_m3s"]) for r in back] == [r["design_peak_m3s"] for r in rows]
    study = __import__("json").loads(paths["study"].read_text())
    assert study["areas_km2"] == [1.0, 3.0] and study["arf_table_type"] == "storm-centred" and study["table"] == rows
    assert np.array_equal(np.load(paths["max_depth"]), np.ones((3, 4)))
    S.write_table(tmp_path / "empty.csv", [])
    assert (tmp_path / "empty.csv").read_text() == "design_point\n"
