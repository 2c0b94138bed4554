"""``bench.py --impl reference``: the reference's CPU step (the oracle, on every host thread) on a bounded sample of the
workload, printed as one JSON line with the keys the arm's contract names; ranks other than 0 exit 0 without work."""

from __future__ import annotations

import json
import os
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]
CMD = [sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--n", "256", "--steps", "3", "--warmup", "3"]


def _run(rank: str | None) -> subprocess.CompletedProcess:
    env = {k: v for k, v in os.environ.items() if k != "RANK"}
    if rank is not None:
        env["RANK"] = rank
    return subprocess.run(CMD, cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)


def test_reference_arm_prints_one_line_with_the_contract_keys():
    out = _run(None)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.strip()]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["metric"] == "cell-steps/s" and d["unit"] == "cell-steps/s" and d["higher_is_better"] is True
    assert d["value"] > 0 and d["steps"] == 3 and d["warmup"] == 3 and d["n_gpus"] == 1
    cb = d["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == d["value"] and cb["sample"]
    # the block is the grid's middle, a tile short of its side on a grid this small: 8 x 8 tiles, the outer ring
    # of cells inactive
    assert cb["sample"].startswith("8x8 tiles (64516 cells)")
    assert d["e2e"] == {"value": d["value"], "unit": "cell-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert d["config"]["workload"].startswith("configuration 3, 256x256 cells")


def test_reference_arm_other_ranks_exit_without_work():
    out = _run("1")
    assert out.returncode == 0, out.stderr[-2000:]
    assert out.stdout.strip() == ""
