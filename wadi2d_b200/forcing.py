"""Sources and boundaries of a run, on the host in FP64: what the step's ``src`` vector and the balance books hold.

Restated from the reference (each piece cites it): the SCS curve-number loss (wadi2d/hydrology/losses.py:47-77),
area-reduction factors (wadi2d/storm/arf.py:13-98), the uniform storm (wadi2d/storm/uniform.py:17-39), lumped inflow
injections (wadi2d/forcing.py:427-477), the window rate of the net source (wadi2d/forcing.py:646-695), the faces
between the interior and the boundary cells (wadi2d/forcing.py:334-356) and the water balance
(wadi2d/engine/monitor.py:36-80, :197-218).

Added for configuration 3, with no counterpart on the reference's grid cells (its grid cells take only the SCS loss
or none, wadi2d/hydrology/losses.py:37-77): a triangular hyetograph and an initial-and-constant loss, both defined
here in FP64 and checked against the oracle-free restatement in tests/test_forcing.py.
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

MM_PER_M = 1000.0
SECONDS_PER_MINUTE = 60.0
MM_PER_INCH = 25.4
ZERO_WATER = 1e-9


# ---------------------------------------------------------------------------------------------------- losses


@dataclass(frozen=True)
class ScsCurveNumber:
    """SCS curve number (wadi2d/hydrology/losses.py:47-77); ``curve_number`` may be an array of classes."""

    curve_number: float | np.ndarray
    initial_abstraction_mm: float | None = None

    @property
    def retention_mm(self):
        return (1000.0 / np.asarray(self.curve_number, np.float64) - 10.0) * MM_PER_INCH

    @property
    def abstraction_mm(self):
        if self.initial_abstraction_mm is None:
            return 0.2 * self.retention_mm
        return self.initial_abstraction_mm

    def cumulative_excess(self, cumulative_mm):
        """Pe(P) = (P - Ia)^2 / (P - Ia + S), zero up to Ia."""
        effective = np.maximum(cumulative_mm - self.abstraction_mm, 0.0)
        return effective**2 / (effective + self.retention_mm)


@dataclass(frozen=True)
class InitialConstantLoss:
    """Initial loss ``initial_mm``, then ``constant_mm_h`` of the rain intensity (configuration 3).

    Per source window [t0, t1] with rain p = P(t1) - P(t0): what is left of the initial loss takes the rain first;
    the constant loss applies over the part of the window after the initial loss is met, the rain taken as steady
    within the window; excess = max(p - ia_left - fc (t1 - t_met), 0), t_met the moment the initial loss is met."""

    initial_mm: float = 10.0
    constant_mm_h: float = 2.0

    def window_excess(self, p0, p1, dt_s: float):
        """Excess depth (mm) of a window from the cumulative rain at its start and end."""
        p0 = np.asarray(p0, np.float64)
        p = np.asarray(p1, np.float64) - p0
        left = np.maximum(self.initial_mm - p0, 0.0)
        after = np.maximum(p - left, 0.0)
        share = np.where(p > 0.0, after / np.where(p > 0.0, p, 1.0), 0.0)  # the part of the window past the loss
        return np.maximum(after - self.constant_mm_h * share * dt_s / 3600.0, 0.0)


# ---------------------------------------------------------------------------------------------------- storms


@dataclass(frozen=True)
class ArfTable:
    """A (storm area, factor) table read by linear interpolation in area (wadi2d/storm/arf.py:13-40)."""

    areas_km2: np.ndarray
    factors: np.ndarray
    reduces_below_table: bool = True

    def factor(self, area_km2: float) -> float:
        if area_km2 < self.areas_km2[0] and not self.reduces_below_table:
            return 1.0
        return float(np.interp(area_km2, self.areas_km2, self.factors))

    def step_areas(self, low_km2: float, high_km2: float, largest_change: float) -> list[float]:
        """Storm areas from ``low_km2`` to ``high_km2``, both in, with the factor (as ``factor`` reads it) changing by
        at most ``largest_change`` between neighbours, in as few areas as that allows (wadi2d/storm/arf.py:39-67). The
        factor's whole path over the span, its rises and falls both counted, is cut into equal steps, and each cut is
        placed by linear interpolation along the path between the table's areas."""
        if not largest_change > 0.0:
            raise ValueError("the largest change of the area-reduction factor must be above zero")
        lo, hi = float(low_km2), float(high_km2)
        if hi <= lo * (1.0 + 1e-9):
            return [lo]
        knots = sorted({lo, hi, *(float(a) for a in self.areas_km2 if lo < a < hi)})
        vals = [self.factor(a) for a in knots]
        first = float(self.areas_km2[0])
        if not self.reduces_below_table and lo < first < hi:  # the full depth holds up to just below the table
            at = knots.index(first)
            knots.insert(at, first)
            vals.insert(at, 1.0)
        path = np.concatenate(([0.0], np.cumsum(np.abs(np.diff(vals)))))
        n = max(1, int(np.ceil(path[-1] / largest_change - 1e-9)))
        out = [lo]
        for target in path[-1] * np.arange(1, n) / n:
            k = min(max(int(np.searchsorted(path, target, side="left")), 1), len(knots) - 1)
            seg = path[k] - path[k - 1]
            share = (target - path[k - 1]) / seg if seg > 0 else 1.0
            out.append(float(knots[k - 1] + share * (knots[k] - knots[k - 1])))
        out.append(hi)
        return sorted(set(out))


@dataclass(frozen=True)
class GivenFactor:
    value: float

    def factor(self, _area_km2=None) -> float:
        return self.value


def factor_at(arf, area_km2) -> float:
    """wadi2d/storm/arf.py:89-98."""
    if arf is None:
        return 1.0
    if isinstance(arf, GivenFactor):
        return arf.value
    if area_km2 is None:
        return 1.0
    return arf.factor(area_km2)


@dataclass(frozen=True)
class UniformStorm:
    """``depth_mm`` at a constant rate over ``duration_minutes``, reduced by the ARF (wadi2d/storm/uniform.py)."""

    depth_mm: float
    duration_minutes: float
    storm_area_km2: float | None = None
    arf: ArfTable | GivenFactor | None = None

    @property
    def total_depth(self) -> float:
        return self.depth_mm * factor_at(self.arf, self.storm_area_km2)

    def fraction(self, minutes) -> np.ndarray:
        return np.clip(np.asarray(minutes, dtype=np.float64) / self.duration_minutes, 0.0, 1.0)

    def cumulative_depth(self, minutes) -> np.ndarray:
        return self.total_depth * self.fraction(minutes)


@dataclass(frozen=True)
class TriangularStorm:
    """Configuration 3's hyetograph: intensity rising linearly to a peak at half the storm and falling back."""

    depth_mm: float
    duration_minutes: float
    factor: float = 1.0

    @property
    def total_depth(self) -> float:
        return self.depth_mm * self.factor

    def fraction(self, minutes) -> np.ndarray:
        x = np.clip(np.asarray(minutes, dtype=np.float64) / self.duration_minutes, 0.0, 1.0)
        return np.where(x <= 0.5, 2.0 * x * x, 1.0 - 2.0 * (1.0 - x) ** 2)

    def cumulative_depth(self, minutes) -> np.ndarray:
        return self.total_depth * self.fraction(minutes)


# ---------------------------------------------------------------------------------------------------- inflows


@dataclass
class Injection:
    """A hydrograph, linear between its table times, and the cells that take it (wadi2d/forcing.py:427-477).
    ``cells`` are positions in the source vector; ``index`` their reference state indices."""

    name: str
    cells: np.ndarray
    index: np.ndarray
    lowest: int
    times: np.ndarray
    flows: np.ndarray
    min_depth: float
    window: float = 0.0
    volume: np.ndarray = field(init=False)

    def __post_init__(self) -> None:
        self.times = np.asarray(self.times, np.float64)
        self.flows = np.asarray(self.flows, np.float64)
        if np.any(np.diff(self.times) <= 0.0):
            raise ValueError(f"inflow {self.name}: table times must increase")
        seg = np.diff(self.times) * (self.flows[1:] + self.flows[:-1]) / 2.0  # the trapezoid sum in scipy's order
        self.volume = np.concatenate(([0.0], np.cumsum(seg)))

    def volume_at(self, t: float) -> float:
        """The exact integral of the piecewise-linear flow up to t."""
        times = self.times
        if t <= times[0]:
            return 0.0
        if t >= times[-1]:
            return float(self.volume[-1])
        k = int(np.searchsorted(times, t, side="right")) - 1
        flow = self.flows[k] + (self.flows[k + 1] - self.flows[k]) * (t - times[k]) / (times[k + 1] - times[k])
        return float(self.volume[k] + 0.5 * (self.flows[k] + flow) * (t - times[k]))

    def mean_flow(self, t0: float, t1: float) -> float:
        return (self.volume_at(t1) - self.volume_at(t0)) / (t1 - t0)

    def share(self, depth: np.ndarray) -> np.ndarray:
        """Weights over the cells: by depth over ``min_depth``; all to the lowest cell while every cell is dry."""
        wet = depth >= self.min_depth
        if not wet.any():
            out = np.zeros(depth.size)
            out[self.lowest] = 1.0
            return out
        weights = np.where(wet, depth, 0.0).astype(np.float64)
        return weights / weights.sum()


# ---------------------------------------------------------------------------------------------------- the window rate


class Forcing:
    """The net source rate over the interior cells, per source window (wadi2d/forcing.py:479-551, :646-695).

    ``cells``: reference state indices of the interior cells; ``storm`` any object with ``cumulative_depth(minutes)``
    (or None); ``depth_factor`` an optional per-cell depth multiplier (a storm depth grid, ``storm.depth_grid``);
    ``loss`` a ScsCurveNumber (``class_of`` per cell, -1 = no loss), an InitialConstantLoss, or None; ``rained`` a
    mask of the cells that take rain (lumped subbasins take none); ``injections`` the lumped inflows.
    """

    def __init__(self, cells, area: float, storm=None, depth_factor=None, loss=None, class_of=None, rained=None,
                 injections=(), depth_reader=None) -> None:  # fmt: skip
        self.state = np.asarray(cells, np.int64)
        self.area = float(area)
        self.storm = storm
        self.depths = None if depth_factor is None else np.asarray(depth_factor, np.float64)
        self.loss = loss
        n = self.state.size
        self.class_of = np.full(n, -1, np.int64) if class_of is None else np.asarray(class_of, np.int64)
        self.rained = np.ones(n, bool) if rained is None else np.asarray(rained, bool)
        self.injections = list(injections)
        self.depth_reader = depth_reader

    def _cumulative_rain(self, t: float) -> np.ndarray:
        depth = float(np.asarray(self.storm.cumulative_depth(np.array([t / SECONDS_PER_MINUTE])))[0])
        if self.depths is not None:
            return depth * self.depths
        return np.full(self.state.size, depth)

    def _excess_mm(self, t: float) -> np.ndarray:
        """Cumulative excess at t, per cell (wadi2d/forcing.py:646-665)."""
        rain = self._cumulative_rain(t)
        if isinstance(self.loss, ScsCurveNumber):
            has = self.class_of >= 0
            out = rain.copy()
            with np.errstate(divide="ignore", invalid="ignore"):
                cls = ScsCurveNumber(np.asarray(self.loss.curve_number)[self.class_of[has]],
                                     self.loss.initial_abstraction_mm)  # fmt: skip
                out[has] = np.nan_to_num(cls.cumulative_excess(rain[has]))
            return out
        return rain

    def rate(self, t0: float, t1: float) -> tuple[np.ndarray, float, float]:
        """Mean net rate over [t0, t1] per interior cell (m/s, float32), rain and inflow volumes of the window."""
        step = t1 - t0
        out = np.zeros(self.state.size, np.float32)
        rain = 0.0
        if self.storm is not None:
            if isinstance(self.loss, InitialConstantLoss):
                excess = self.loss.window_excess(self._cumulative_rain(t0), self._cumulative_rain(t1), step)
                excess = excess / (MM_PER_M * step)
            else:
                excess = (self._excess_mm(t1) - self._excess_mm(t0)) / (MM_PER_M * step)
            out[:] = excess * self.rained
            rain = float(out.sum(dtype=np.float64)) * self.area * step
        inflow = 0.0
        for inj in self.injections:
            inj.window = 0.0
            q = inj.mean_flow(t0, t1)
            if q <= 0.0:
                continue
            depth = self.depth_reader(inj) if self.depth_reader is not None else np.zeros(inj.cells.size)
            added = q * inj.share(np.asarray(depth)) / self.area
            out[inj.cells] += added.astype(np.float32)
            inj.window = float(np.float32(added).sum(dtype=np.float64)) * self.area * step
            inflow += inj.window
        return out, rain, inflow


# ---------------------------------------------------------------------------------------------------- boundaries


def open_faces(grid, inner: np.ndarray, taken: np.ndarray) -> list[tuple[np.ndarray, np.ndarray]]:
    """The x and y faces between ``inner`` and ``taken`` cells, with the sign of a flow into ``taken``, as reference
    state indices (wadi2d/forcing.py:334-356)."""
    from wadi2d_b200.state import state_index

    faces = []
    for axis in (1, 0):
        out_low = inner & np.roll(taken, -1, axis=axis)
        j, i = np.nonzero(out_low)
        if axis == 1:
            i = i + 1
        else:
            j = j + 1
        into = inner & np.roll(taken, 1, axis=axis)
        ja, ia = np.nonzero(into)
        index = np.concatenate((state_index(grid, j, i), state_index(grid, ja, ia))).astype(np.int64)
        sign = np.concatenate((np.ones(j.size), -np.ones(ja.size)))
        faces.append((index, sign))
    return faces


# ---------------------------------------------------------------------------------------------------- balance


@dataclass
class Balance:
    """Water accounts of the interior cells, m3 (wadi2d/engine/monitor.py:36-80)."""

    rain: float = 0.0
    inflow: float = 0.0
    outflow: float = 0.0
    storage0: float = 0.0
    storage: float = 0.0
    transmission: float = 0.0

    @property
    def error(self) -> float:
        return self.rain + self.inflow - self.transmission - self.outflow - (self.storage - self.storage0)

    @property
    def relative(self) -> float:
        """Error over the water that entered the model."""
        scale = max(self.rain + self.inflow + max(-self.outflow, 0.0) + self.storage0, ZERO_WATER)
        return self.error / scale


def storage(model, index: np.ndarray) -> float:
    """Water in the interior cells, the rounding residual of each cell included (wadi2d/engine/monitor.py:214-218):
    sum of h + res over the cells, FP64, times the cell area."""
    b = model.backend
    h = np.asarray(b.h[index], np.float64)
    res = np.asarray(b.res[index], np.float64)
    return float((h + res).sum()) * model.grid.dx**2
