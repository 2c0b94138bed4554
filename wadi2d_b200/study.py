"""The depth-area (ARF) study on the batch engine: one run per storm area, all of them advanced together.

The reference runs a study's storm areas one after another through ``run_job`` (wadi2d/arf.py:346-372, ``_study``)
and then reads them: each design line's peak between the two runs that bracket its drainage area, ln Q linear in
ln A (``design_table``, arf.py:157-168), and per cell the same reading of the runs' max-depth, max-speed and hazard
maps against an accumulation raster (``composite_maps``, arf.py:300-316). Here the runs share one grid and one set
of device tables and go into one ``Batch``: each run is the same storm with its storm area set to one of the study's
areas (the ARF table read there), its own clock, envelope and design lines, and each run steps exactly as it would
alone. The readings below keep the reference's names, arguments and results (pinned by ``tests/test_study.py``
against the reference's own functions), and ``write_study`` writes ``design_points.csv`` and ``study.json`` as the
reference does; the job file, the GeoTIFF maps and the progress file around them are the reference's run driver and
stay there.
"""

from __future__ import annotations

import dataclasses
from dataclasses import dataclass, field

import numpy as np

COMPOSITE_MAPS = ("max_depth", "max_speed", "hazard")
ENVELOPE_OF_MAP = {"max_depth": "depth", "max_speed": "speed", "hazard": "hazard"}
"""Each composite's per-run map and the envelope field it is (wadi2d/products/cell_maps.py:79-89)."""
READ_LINE = "design line, 2D runs either side"


# ------------------------------------------------------------------------------------------------ storm areas


def bracket_areas(wanted, ratio: float, most: int) -> list[float]:
    """Storm areas spanning the wanted ones (wadi2d/arf.py:79-86): log-spaced from the smallest to the largest, as
    few as keep neighbours within ``ratio`` of each other but at least two and at most ``most``; a single area when
    the wanted areas are all the same."""
    lo, hi = float(min(wanted)), float(max(wanted))
    if hi <= lo * (1.0 + 1e-9):
        return [lo]
    gaps = int(np.ceil(np.log(hi / lo) / np.log(ratio) - 1e-9))
    return list(np.geomspace(lo, hi, min(max(gaps + 1, 2), most)))


def storm_areas(lines_km2=(), areas_km2=(), n_areas: int = 6, area_min_km2: float = 10.0,
                area_max_km2: float = 600.0, bracket: bool = False, bracket_ratio: float = 2.0, bracket_max: int = 6,
                exact_points: bool = False, by_arf_step: bool = False, arf_step_max: float = 0.05,
                table=None) -> list[float]:  # fmt: skip
    """A study's storm areas (wadi2d/arf.py:89-115, its ``arf`` settings as arguments, the defaults the reference's):
    ``areas_km2`` as given, else ``n_areas`` log-spaced from ``area_min_km2`` to ``area_max_km2``; or, with
    ``bracket``, areas bracketing the design lines' drainage areas ``lines_km2``; or, with ``by_arf_step``, areas
    over the lines' span placed so that the storm's area-reduction ``table`` (a ``forcing.ArfTable``) changes by at
    most ``arf_step_max`` between neighbours; with ``exact_points`` the lines' own areas too. Rounded to 1e-4 km2,
    sorted, each once."""
    lines = [float(a) for a in lines_km2 if a is not None]
    if bracket or by_arf_step:
        if not lines:
            rule = "arf.bracket" if bracket else "arf.by_arf_step"
            raise ValueError(f"{rule} needs a design line with a drainage area")
        if bracket:
            base = bracket_areas(lines, bracket_ratio, bracket_max)
        else:
            if table is None or not hasattr(table, "step_areas"):
                raise ValueError("arf.by_arf_step needs the storm's area-reduction table: the areas are placed by it")
            base = table.step_areas(min(lines), max(lines), arf_step_max)
    else:
        base = list(areas_km2) or list(np.geomspace(area_min_km2, area_max_km2, n_areas))
    if exact_points:
        base += lines
    return sorted({round(float(x), 4) for x in base})


def run_name(area: float) -> str:
    """A run folder's name for a storm area (wadi2d/arf.py:118-119): km2 with three decimals, the point as 'p'."""
    return ("A%010.3fkm2" % area).replace(".", "p")


# ------------------------------------------------------------------------------------------------ readings


def interpolate_peak(areas, peaks, area: float) -> float:
    """A peak at drainage area ``area`` from the runs' peaks (wadi2d/arf.py:122-128): ln Q linear in ln A over the
    runs that carried water, the end values held beyond them; 0 when no run did."""
    areas, peaks = np.asarray(areas, np.float64), np.asarray(peaks, np.float64)
    wet = peaks > 0.0
    if not np.any(wet):
        return 0.0
    return float(np.exp(np.interp(np.log(area), np.log(areas[wet]), np.log(peaks[wet]))))


def _design_row(name, area, a_low, a_high, q_low, q_high, q, t, kind, read_as) -> dict[str, object]:
    """One row of design_points.csv, in the reference's column order (wadi2d/arf.py:131-143)."""
    return {
        "design_point": name,
        "drainage_area_km2": area,
        "storm_area_low_km2": float(a_low),
        "storm_area_high_km2": float(a_high),
        "peak_low_m3s": float(q_low),
        "peak_high_m3s": float(q_high),
        "design_peak_m3s": float(q),
        "time_of_peak_s": float(t),
        "arf_table_type": kind,
        "read_as": read_as,
    }


def interpolated_row(name: str, area: float, grid_a, peaks, times, kind: str, read_as: str) -> dict[str, object]:
    """The row of a point at drainage area ``area`` read from the runs either side of it (wadi2d/arf.py:145-154);
    the time of the peak is the run nearer in ln A."""
    grid_a = np.asarray(grid_a, np.float64)
    peaks, times = np.asarray(peaks, np.float64), np.asarray(times, np.float64)
    last = grid_a.size - 1
    hi = min(max(int(np.searchsorted(grid_a, area)), 0), last)
    lo = max(hi - 1, 0)
    near = lo if abs(np.log(area / grid_a[lo])) <= abs(np.log(area / grid_a[hi])) else hi
    q = interpolate_peak(grid_a, peaks, area)
    return _design_row(name, area, grid_a[lo], grid_a[hi], peaks[lo], peaks[hi], q, times[near], kind, read_as)


def design_table(names, line_areas, areas, peaks, times, kind: str = "unspecified") -> list[dict[str, object]]:
    """One row per design line with a drainage area (wadi2d/arf.py:157-168). ``peaks``, ``times``: (runs x lines),
    the runs in the order of ``areas``; a line whose area is None gets no row."""
    peaks, times = np.asarray(peaks, np.float64), np.asarray(times, np.float64)
    rows = []
    for n, (name, area) in enumerate(zip(names, line_areas, strict=True)):
        if area is None:
            continue
        rows.append(interpolated_row(name, float(area), areas, peaks[:, n], times[:, n], kind, READ_LINE))
    return rows


def log_area_weights(areas, area):
    """The runs bracketing ``area`` (one value or one per cell) and the larger run's weight, linear in ln A
    (wadi2d/arf.py:275-286): ``(low, high, w)``, read as ``(1 - w) * low + w * high``; beyond the runs the end run
    holds (weight 0 or 1). ``areas`` rise and hold two at least."""
    areas = np.asarray(areas, np.float64)
    ln_runs = np.log(areas)
    ln_at = np.log(np.clip(area, areas[0], areas[-1]))
    high = np.clip(np.searchsorted(ln_runs, ln_at), 1, ln_runs.size - 1)
    low = high - 1
    return low, high, (ln_at - ln_runs[low]) / (ln_runs[high] - ln_runs[low])


def composite_map(maps, areas, cell_area) -> np.ndarray:
    """Per cell, the runs' maps read at the cell's drainage area (wadi2d/arf.py:289-297): the two runs that bracket it,
    linear in ln A; beyond them the end run. One run: its map."""
    areas = np.asarray(areas, np.float64)
    if areas.size == 1:
        return np.array(maps[0], dtype=np.float64)
    low, high, w = log_area_weights(areas, cell_area)
    stack = np.stack([np.asarray(m, np.float64) for m in maps])
    j, i = np.indices(np.shape(cell_area), sparse=True)
    return (1.0 - w) * stack[low, j, i] + w * stack[high, j, i]


def composite_maps(envelopes: list[dict], areas, cell_area, depth_floor: float | None = None) -> dict[str, np.ndarray]:
    """The study's composites (wadi2d/arf.py:300-316) from each run's envelope. With ``depth_floor``, a cell whose max
    depth stays under it reads 0 in every map, as the reference reads a floored (no-data) cell of a run's map
    (wadi2d/products/cell_maps.py:96-107, arf.py:311)."""
    out = {}
    for name in COMPOSITE_MAPS:
        maps = []
        for env in envelopes:
            m = np.asarray(env[ENVELOPE_OF_MAP[name]], np.float64)
            if depth_floor is not None:
                m = np.where(np.asarray(env["depth"]) < depth_floor, 0.0, m)
            maps.append(m)
        out[name] = composite_map(maps, areas, cell_area)
    return out


# ------------------------------------------------------------------------------------------------ the runs


@dataclass
class StudyResult:
    areas_km2: list[float]
    peaks: np.ndarray  # (runs x lines) peak |Q|, m3/s
    times: np.ndarray  # (runs x lines) time of the peak, s
    table: list[dict[str, object]]
    composite: dict[str, np.ndarray]
    steps: np.ndarray
    seconds: float
    envelopes: list[dict] = field(default_factory=list)


def check_study(storm, areas) -> None:
    """A study needs a storm with an area-reduction table that tells its runs apart (wadi2d/arf.py:319-349,
    :374-383): a single given factor, no table, or the same depth at every storm area would make every run the same
    run. Raises ValueError."""
    from wadi2d_b200.forcing import ArfTable, GivenFactor

    arf = getattr(storm, "arf", None)
    if isinstance(arf, GivenFactor):
        raise ValueError("a depth-area study reads the area-reduction table at each storm area; a given factor is one "
                         "factor at every area, so every run would be the same run")  # fmt: skip
    if not isinstance(arf, ArfTable):
        raise ValueError("a depth-area study needs the storm's area-reduction table: without it every run is the same")
    depths = {round(s.total_depth, 9) for s in storms_at(storm, areas)}
    if len(areas) > 1 and len(depths) == 1:
        raise ValueError(f"the area-reduction table gives one factor at all the storm areas {list(areas)}: the runs "
                         "would be identical")  # fmt: skip


def storms_at(storm, areas) -> list:
    """The study's storm at each storm area: the same storm with ``storm_area_km2`` set (its ARF table read there)."""
    return [dataclasses.replace(storm, storm_area_km2=float(a)) for a in areas]


def solve_runs(cat, storms: list, t_end: float, window: float = 30.0, every: int = 4, num=None,
               batched: bool = True) -> tuple:  # fmt: skip
    """The storms on the catchment from dry ground to ``t_end``: each run's design-line peaks and their times (runs x
    lines), its steps and its envelope, and the CUDA-event seconds around the runs. ``batched``: all runs in one batch
    (the B200 form), else one plain run after another (the reference's order)."""
    import torch

    from wadi2d_b200.config import Numerics

    num = num or Numerics()
    n, nl = len(storms), len(cat.lines)
    peaks, times = np.zeros((n, nl)), np.zeros((n, nl))
    steps = np.zeros(n, np.int64)
    envelopes: list[dict] = []
    lines = [ln[:4] for ln in cat.lines]
    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if batched:
        from wadi2d_b200.batch import Batch

        B = Batch([cat.grid] * n, [cat.tables] * n, num)
        B.set_boundary([cat.boundary] * n)
        B.set_depth([np.zeros(cat.grid.shape)] * n)
        B.set_tally([cat.tally] * n)
        B.set_lines([lines] * n)
        B.reset_envelope()
        cells = [B.native_of(r, cat.rained) for r in range(n)]
        torch.cuda.synchronize()
        e0.record(stream)
        B.run_windows(np.full(n, float(t_end)), storms, window=window, max_every=every, cells=cells)
        e1.record(stream)
        torch.cuda.synchronize()
        for r in range(n):
            peaks[r], times[r] = B.line_peaks(r)
            envelopes.append(B.envelope(r))
        steps[:] = B.nsteps
        del B
    else:
        from wadi2d_b200.maxima import Lines, Maxima, Tally
        from wadi2d_b200.model import Model
        from wadi2d_b200.run import DeviceRain, run_windows

        torch.cuda.synchronize()
        e0.record(stream)
        for r in range(n):
            m = Model(cat.tables, num)
            m.set_boundary(cat.boundary)
            m.set_depth(np.zeros(cat.grid.shape))
            tally = Tally(m, *cat.tally)
            maxima = Maxima(m, 0.1, 0.05, every=every)
            lines_r = Lines(m, lines)
            rain = DeviceRain(m, storms[r], cat.rained)
            run_windows(m, float(t_end), rain=rain, window=window, maxima=maxima, tally=tally)
            peaks[r], times[r] = lines_r.peaks()
            envelopes.append(maxima.fields())
            steps[r] = m.stepper.nsteps
            del m, tally, maxima, lines_r, rain
        e1.record(stream)
        torch.cuda.synchronize()
    return peaks, times, steps, envelopes, e0.elapsed_time(e1) / 1e3


def run_study(cat, storm, areas, line_names, line_areas, cell_area, t_end: float, window: float = 30.0,
              every: int = 4, num=None, batched: bool = True, kind: str = "unspecified",
              depth_floor: float | None = None) -> StudyResult:  # fmt: skip
    """Every storm area of the study through the solver from dry ground to ``t_end``, then the design table and the
    composites. ``cat``: the catchment (``critical.Catchment5``: grid, device tables, outfalls, outfall tally, rained
    cells, design lines). ``batched``: all runs in one batch (the B200 form), else one plain run after another (the
    reference's order). Seconds are CUDA-event time around the runs."""
    areas = [float(a) for a in areas]
    check_study(storm, areas)
    peaks, times, steps, envelopes, seconds = solve_runs(cat, storms_at(storm, areas), t_end, window, every, num,
                                                         batched)  # fmt: skip
    table = design_table(line_names, line_areas, areas, peaks, times, kind)
    composite = composite_maps(envelopes, areas, cell_area, depth_floor)
    return StudyResult(areas, peaks, times, table, composite, steps, seconds, envelopes)


def run_study_sharded(cat, storm, areas, line_names, line_areas, cell_area, t_end: float, window: float = 30.0,
                      every: int = 4, num=None, kind: str = "unspecified", depth_floor: float | None = None,
                      world: int | None = None, rank: int | None = None, group=None,
                      solve=None) -> StudyResult | None:  # fmt: skip
    """The study over the ranks of a process group, one GPU a rank: the storm areas are split by ``sweep.partition``
    (every run has the same catchment and end time, so the cost is equal), each rank solves its share as one batch,
    and one gather (``sweep.gather_results``) brings every run's peaks, times, steps and envelope to rank 0, which
    reads the design table and the composites. Returns the StudyResult on rank 0 (``seconds``: the slowest rank's),
    None elsewhere. ``solve`` stands in for ``solve_runs`` (same arguments and results)."""
    from wadi2d_b200.sweep import gather_results, partition

    if world is None or rank is None:
        import torch.distributed as dist

        world, rank = dist.get_world_size(group), dist.get_rank(group)
    areas = [float(a) for a in areas]
    check_study(storm, areas)
    storms = storms_at(storm, areas)
    mine = partition([1.0] * len(areas), world)[rank]
    local: dict = {}
    if mine:
        p, t, st, env, sec = (solve or solve_runs)(cat, [storms[i] for i in mine], t_end, window, every, num, True)
        local = {i: (p[k], t[k], int(st[k]), env[k], sec) for k, i in enumerate(mine)}
    merged = gather_results(local, world, rank, group)
    if merged is None:
        return None
    if sorted(merged) != list(range(len(areas))):
        raise ValueError("a storm area came back from no rank")
    rec = [merged[i] for i in range(len(areas))]
    peaks = np.stack([np.asarray(r[0], np.float64) for r in rec])
    times = np.stack([np.asarray(r[1], np.float64) for r in rec])
    steps = np.array([r[2] for r in rec], np.int64)
    envelopes = [r[3] for r in rec]
    table = design_table(line_names, line_areas, areas, peaks, times, kind)
    composite = composite_maps(envelopes, areas, cell_area, depth_floor)
    return StudyResult(areas, peaks, times, table, composite, steps, max(r[4] for r in rec), envelopes)


def drainage_km2(cat) -> tuple[np.ndarray, np.ndarray]:
    """Each cell's D8 drainage area, km2 (the study's accumulation raster), and each design line's (at its centre
    cell)."""
    from wadi2d_b200.critical import flow_accumulation

    acc, _ = flow_accumulation(np.asarray(cat.tables.zmin), cat.grid.mask)
    cell = acc * float(cat.grid.dx) ** 2 / 1e6
    return cell, np.array([cell[j, i] for *_, (j, i) in cat.lines])


def write_table(path, rows: list[dict[str, object]]) -> None:
    """``design_points.csv`` (wadi2d/arf.py:186-195): a header of the rows' keys and a line a row; with no rows, the
    header ``design_point`` alone."""
    import csv
    from pathlib import Path

    path = Path(path)
    path.parent.mkdir(parents=True, exist_ok=True)
    with path.open("w", newline="", encoding="utf-8") as f:
        if not rows:
            f.write("design_point\n")
            return
        writer = csv.DictWriter(f, fieldnames=list(rows[0]))
        writer.writeheader()
        writer.writerows(rows)


def write_study(folder, res: StudyResult, kind: str = "unspecified") -> dict:
    """A study's outputs into ``folder`` as the reference lays them out (wadi2d/arf.py:383-395): ``design_points.csv``,
    ``study.json`` (storm areas, the table's type, the rows, no on-grid elements) and one composite per quantity under
    ``composite/``, as ``.npy`` arrays on the cell grid (the reference writes GeoTIFF through rasterio, which this
    package does not carry). Returns the paths."""
    import json
    from pathlib import Path

    folder = Path(folder)
    folder.mkdir(parents=True, exist_ok=True)
    write_table(folder / "design_points.csv", res.table)
    study = {"areas_km2": res.areas_km2, "arf_table_type": kind, "table": res.table, "on_grid": []}
    (folder / "study.json").write_text(json.dumps(study, indent=2), encoding="utf-8")
    out = {"table": folder / "design_points.csv", "study": folder / "study.json"}
    (folder / "composite").mkdir(exist_ok=True)
    for name, data in res.composite.items():
        out[name] = folder / "composite" / f"{name}.npy"
        np.save(out[name], np.asarray(data, np.float64))
    return out


def bracketing_areas(cat, ratio: float = 2.0, most: int = 6) -> tuple[list[float], np.ndarray, np.ndarray]:
    """The study's storm areas bracketing the design lines' drainage areas (``arf.bracket``), with the cells' and the
    lines' drainage areas."""
    cell, line_a = drainage_km2(cat)
    return storm_areas(list(line_a), bracket=True, bracket_ratio=ratio, bracket_max=most), cell, line_a
