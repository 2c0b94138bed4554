"""The CUDA path's error against the FP64 run, field by field, as configuration 1 (256 x 256 cells) steps on: one
JSON line per step count, then the crest case's line (test infrastructure; run on a machine with a B200, from the
repository root: ``python tests/fp64_report.py``)."""

from __future__ import annotations

import json
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
sys.path[:0] = [str(HERE.parent), str(HERE), str(HERE / "golden")]

import fp64_check as F  # noqa: E402
from product_api import B200Api  # noqa: E402

MARKS = (50, 100, 200, 400, 800, 1600, 3200)


def _line(case: str, k: int, r: dict) -> str:
    rel = {name: float(f"{e['rel_to_scale']:.3g}") for name, e in r["fields"].items()}
    absd = {name: float(f"{e['max_abs']:.3g}") for name, e in r["fields"].items()}
    checks = {key: r[key] for key in r if key != "fields"}
    return json.dumps({"case": case, "steps": k, **checks, "rel_to_scale": rel, "max_abs": absd})


def main() -> None:
    s32, dts = F.snapshots(B200Api(), MARKS, n=256)
    s64 = F.fp64_snapshots(dts, MARKS, n=256)
    for k in MARKS:
        print(_line("configuration 1, 256 x 256", k, F.compare(s32[k], s64[k])), flush=True)
    c32, cdts = F.snapshots(B200Api(), (100,), case="crest")
    c64 = F.fp64_snapshots(cdts, (100,), case="crest")
    print(_line("crest case", 100, F.compare(c32[100], c64[100], F.crest_faces())), flush=True)


if __name__ == "__main__":
    main()
