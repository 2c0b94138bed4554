"""The run-folder writers' layout on CPU (wadi2d/io/results.py:1-99, wadi2d/io/checkpoint.py:53-61): a results file
written and read back, dataset paths and attributes as the reference names them, appending keeps what was there, and
a checkpoint's job hash."""

from __future__ import annotations

import numpy as np

from wadi2d_b200.grid import TileGrid
from wadi2d_b200.runfolder import CHECKPOINT_FORMAT, FORMAT_VERSION, Results, Store, checkpoint_job, read_results


def test_results_round_trip_and_append(tmp_path):
    g = TileGrid.from_mask(np.ones((40, 50), bool), 1000.0, 2000.0, 10.0)
    rng = np.random.default_rng(0)
    maps = {"depth": rng.random(g.shape), "mean_depth": rng.random(g.shape), "speed": rng.random(g.shape)}
    r = Results(tmp_path / "results.h5", g, "LOCAL_CS", '{"run": 1}')
    r.snapshot(600.4, maps)
    r.maxima({"depth": maps["depth"] * 2})
    r.series("lines", "Main channel / km 3", np.array([0.0, 60.0]), {"discharge_m3s": np.array([0.0, 12.5])})
    r.attributes({"status": "finished", "steps": 1234, "relative_error": 1e-9})
    r.close()
    r = Results(tmp_path / "results.h5", g, append=True)  # a resumed run appends
    r.snapshot(1200.0, {"depth": maps["depth"] + 1})
    r.close()
    f = read_results(tmp_path / "results.h5")
    assert f.attr("", "format_version") == FORMAT_VERSION
    assert f.attr("", "config") == '{"run": 1}'
    assert (f.attr("", "x0"), f.attr("", "y0"), f.attr("", "dx")) == (g.x0, g.y0, g.dx)
    assert np.array_equal(f.get("mask"), g.mask)
    assert f.children("maps") == ["t000000600", "t000001200"]
    assert f.attr("maps/t000000600", "t_s") == 600.4
    for k, a in maps.items():
        assert np.array_equal(f.get(f"maps/t000000600/{k}"), a.astype(np.float32))
    assert np.array_equal(f.get("maps/t000001200/depth"), (maps["depth"] + 1).astype(np.float32))
    assert np.array_equal(f.get("maxima/depth"), (maps["depth"] * 2).astype(np.float32))
    grp = "series/lines/Main_channel_km_3"
    assert f.attr(grp, "name") == "Main channel / km 3"
    assert np.array_equal(f.get(f"{grp}/discharge_m3s"), [0.0, 12.5]) and np.array_equal(f.get(f"{grp}/t_s"), [0, 60])
    assert f.attr("", "status") == "finished" and f.attr("", "steps") == 1234


def test_checkpoint_job_reads_the_hash_or_none(tmp_path):
    s = Store(tmp_path / "c.h5", "w")
    s.set_attr("", "format", CHECKPOINT_FORMAT)
    s.set_attr("", "job_hash", "abc123")
    s.close()
    assert checkpoint_job(tmp_path / "c.h5") == "abc123"
    s = Store(tmp_path / "old.h5", "w")
    s.set_attr("", "format", "1")
    s.close()
    assert checkpoint_job(tmp_path / "old.h5") is None
    (tmp_path / "bad.h5").write_bytes(b"not a checkpoint")
    assert checkpoint_job(tmp_path / "bad.h5") is None
    assert checkpoint_job(tmp_path / "missing.h5") is None
