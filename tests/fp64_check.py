"""Float32 results against the FP64 run (test infrastructure: the tests and ``tests/fp64_report.py`` use it).

``snapshots`` drives a case of tests/golden/cases.py through any case API and keeps every field (and, where the case
records them, the envelope and the outfall volume) at chosen step counts: configuration 1 (``c1_small``: rain on a
V-channel plane, free outfall, CFL 0.9, sleeping tiles, the envelope every 4 steps) or the crest case (``crest``:
crest caps, walls, fixed-stage and follow boundaries). ``compare`` measures a float32 run's snapshot against the FP64
run's (oracle/fp64.py, replaying the float32 run's own dt sequence) with the step's accuracy bounds: the wet set and
the crest-blocked faces identical, depth within 1e-4 relative or 1e-5 m, and unit discharge within 1e-4 of its
field's scale.
"""

from __future__ import annotations

import numpy as np

import cases
from oracle import fp64
from oracle import oracle as O

FIELDS = ("h", "d", "u", "v", "mx", "my", "qx", "qy", "om")
DEPTH_REL, DEPTH_ABS, Q_REL = 1e-4, 1e-5, 1e-4


class _Stop(Exception):
    pass


def _own(grid, a):
    if isinstance(grid, O.Grid):
        return O.from_state(grid, a)
    from wadi2d_b200.state import from_state

    return from_state(grid, a)


def snapshots(api, marks, n: int = 256, case: str = "c1") -> tuple[dict, list]:
    """The case (configuration 1 at n x n, or the crest case) stepped to the largest of ``marks``; the fields
    (cell-grid arrays, float64), the envelope and the outfall volume at each mark, and the run's dt sequence."""
    marks = sorted(int(m) for m in marks)
    api._maxima = api._tally = None
    store: dict[int, dict] = {}
    make = api.model

    def model(*a, **k):
        m = make(*a, **k)
        advance = m.advance

        def stepped(t_end, on_step=None):
            def cb(st):
                if on_step is not None:
                    on_step(st)
                if st.nsteps in marks:
                    g = m.grid
                    snap = {f: _own(g, m.backend.get_field(f)).astype(np.float64) for f in FIELDS}
                    if api._maxima is not None:
                        for name, a in api._maxima.raw().items():
                            snap["max_" + name] = _own(g, a).astype(np.float64)
                    if api._tally is not None:
                        snap["tally"] = float(api._tally.volume())
                    store[st.nsteps] = snap
                    if st.nsteps == marks[-1]:
                        raise _Stop

            return advance(t_end, cb)

        m.advance = stepped
        return m

    api.model = model
    try:
        if case == "c1":
            cases.c1_small(api, t_end=1e7, n=n)
        else:
            cases.crest(api, t_end=1e7)
    except _Stop:
        pass
    return store, list(api.dts)


def crest_faces() -> tuple[np.ndarray, np.ndarray]:
    """The crest case's crest faces (nonzero crest coefficient) on the cell grid, x and y, from the oracle's tables."""
    from oracle_api import OracleApi

    api = OracleApi()
    grid, z, crest, npix, (nx, ny, k, dx) = cases.crest_inputs(api)
    t = api.tables(grid, z, dx / k, 0.04, True, crest, npix)
    return grid.from_tiles(t["cwx"]) != 0, grid.from_tiles(t["cwy"]) != 0


def compare(s32: dict, s64: dict, crest: tuple | None = None) -> dict:
    """The float32 snapshot against the FP64 one: per-field errors and the accuracy checks (with ``crest``, the
    crest faces' masks, also the set of crest faces that carry no discharge)."""
    out = {"fields": {}}
    for key in s32:
        if key == "tally":
            continue
        out["fields"][key] = fp64.field_errors(s32[key], s64[key])
    h32, h64 = s32["h"], s64["h"]
    diff = np.abs(h32 - h64)
    out["wet_set_identical"] = bool(np.array_equal(h32 > 0, h64 > 0))
    out["depth_within"] = bool(np.all((diff <= DEPTH_ABS) | (diff <= DEPTH_REL * np.abs(h64))))
    out["discharge_within"] = all(out["fields"][q]["rel_to_scale"] <= Q_REL for q in ("qx", "qy"))
    if "tally" in s32:
        out["tally_rel"] = abs(s32["tally"] - s64["tally"]) / max(abs(s64["tally"]), 1e-30)
    if crest is not None:
        cx, cy = crest
        out["crest_faces"] = int(cx.sum() + cy.sum())
        out["crest_blocked"] = int(((s64["qx"] == 0) & cx).sum() + ((s64["qy"] == 0) & cy).sum())
        out["crest_blocked_identical"] = bool(
            np.array_equal((s32["qx"] == 0) & cx, (s64["qx"] == 0) & cx)
            and np.array_equal((s32["qy"] == 0) & cy, (s64["qy"] == 0) & cy)
        )
    return out


def fp64_snapshots(dts, marks, n: int = 256, case: str = "c1") -> dict:
    """The FP64 run of the case through ``dts`` (a float32 run's steps), at the same marks."""
    from oracle_api import Fp64Api

    store, _ = snapshots(Fp64Api(dts[: max(marks)]), marks, n, case)
    return store
