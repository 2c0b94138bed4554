"""The run driver's window loop (wadi2d/run.py:1712-1740) on the B200 backend: per source window the net source is
set, the model advances to the window's end on the device (envelope and FP64 outfall tally inside the loop), and the
books are kept as the reference's monitor keeps them (wadi2d/engine/monitor.py:36-80, :197-218).

Rain comes either from the host (``forcing.Forcing.rate``, the reference's form: a float32 rate per interior cell
uploaded each window) or from the device (``DeviceRain``: the same rate formed on the GPU from per-cell storm depth
multipliers, which removes the per-window upload). Lumped inflows likewise: on the host (``Forcing`` with
injections, the cells' levels read back from the device each window) or on the device (``DeviceInflow``: each
hydrograph's window flow shared by the levels read in place, no read-back and no upload). A host that knows its next
window's rates ahead can upload them while the current window steps (``SourceStager``).
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from wadi2d_b200 import _lib
from wadi2d_b200.forcing import Balance, InitialConstantLoss, ScsCurveNumber
from wadi2d_b200.layout import native_of_ref

SECONDS_PER_MINUTE = 60.0


class DeviceRain:
    """A storm over a set of cells, rated on the device each window (w2b_rain_window).

    ``cells``: reference state indices of the rained cells; ``multiplier``: per-cell factor on the storm's cumulative
    depth (a depth grid; 1 for uniform rain); ``loss``: ScsCurveNumber (per-cell curve numbers), InitialConstantLoss,
    or None."""

    def __init__(self, model, storm, cells, multiplier=None, loss=None, curve_number=None) -> None:
        b = model.backend
        torch = b.torch
        self.model, self.storm = model, storm
        dev = b.device
        n = int(np.asarray(cells).size)
        native = native_of_ref(model.grid.tiles, cells, model.grid.shape[1]).astype(np.int32)
        self.cells = torch.as_tensor(native, device=dev)
        mult = np.ones(n) if multiplier is None else np.asarray(multiplier, np.float64)
        self.depth = torch.as_tensor(mult, dtype=torch.float64, device=dev)
        self.partial = torch.zeros(_lib.PARTIALS, dtype=torch.float64, device=dev)
        self.volume = torch.zeros(1, dtype=torch.float64, device=dev)
        self.s = self.ia = None
        kind, fc = 0, 0.0
        if isinstance(loss, ScsCurveNumber):
            cn = np.broadcast_to(np.asarray(curve_number if curve_number is not None else loss.curve_number,
                                            np.float64), (n,))  # fmt: skip
            scs = ScsCurveNumber(cn, loss.initial_abstraction_mm)
            self.s = torch.as_tensor(np.broadcast_to(scs.retention_mm, (n,)).copy(), device=dev)
            self.ia = torch.as_tensor(np.broadcast_to(scs.abstraction_mm, (n,)).astype(np.float64).copy(), device=dev)
            kind = 1
        elif isinstance(loss, InitialConstantLoss):
            self.ia = torch.full((n,), float(loss.initial_mm), dtype=torch.float64, device=dev)
            fc, kind = float(loss.constant_mm_h), 2
        self.tiles = np.unique(np.asarray(cells, np.int64) // 1296)
        self.rain = _lib.Rain(n, self.cells.data_ptr(), self.depth.data_ptr(), kind,
                              None if self.s is None else self.s.data_ptr(),
                              None if self.ia is None else self.ia.data_ptr(), fc, self.partial.data_ptr())  # fmt: skip

    def window(self, t0: float, t1: float) -> float:
        """Write the window's rates into src; return its rain volume, m3."""
        f0 = float(np.asarray(self.storm.cumulative_depth(np.array([t0 / SECONDS_PER_MINUTE])))[0])
        f1 = float(np.asarray(self.storm.cumulative_depth(np.array([t1 / SECONDS_PER_MINUTE])))[0])
        b = self.model.backend
        _lib.call("w2b_rain_window", b.handle, ctypes.byref(self.rain), f0, f1, float(t0), float(t1),
                  self.volume.data_ptr(), b._stream())  # fmt: skip
        return float(self.volume.item())


class DeviceInflow:
    """Lumped inflows rated on the device each window (w2b_inflow_window): each injection's mean flow over the
    window (the exact integral of its piecewise-linear hydrograph, ``forcing.Injection.mean_flow``, on the host) is
    shared over its cells by their level, read in place on the device, as ``forcing.Forcing.rate`` shares it on the
    host (wadi2d/forcing.py:684-694, :468-476). ``rained``: reference state indices of the cells whose source the
    window's ``DeviceRain`` writes (the inflow is added on top of their rain), or None. The window volumes are kept on
    the device; ``total()`` reads their sum once."""

    def __init__(self, model, injections, area: float, rained=None) -> None:
        b = model.backend
        torch = b.torch
        self.model, self.injections = model, list(injections)
        n = len(self.injections)
        if n > _lib.INFLOWS_MAX:
            raise ValueError(f"{n} inflows: at most {_lib.INFLOWS_MAX} a call")
        index = [np.asarray(inj.index, np.int64) for inj in self.injections]
        self.start = np.concatenate(([0], np.cumsum([i.size for i in index]))).astype(np.int32)
        allidx = np.concatenate(index) if n else np.zeros(0, np.int64)
        native = native_of_ref(model.grid.tiles, allidx, model.grid.shape[1]).astype(np.int32)
        flags = np.zeros(allidx.size, np.uint8) if rained is None else np.isin(allidx, rained).astype(np.uint8)
        self.cells = torch.as_tensor(native, device=b.device)
        self.rained = torch.as_tensor(flags, device=b.device)
        self.lowest = np.array([inj.lowest for inj in self.injections], np.int32)
        self.min_depth = np.array([inj.min_depth for inj in self.injections], np.float64)
        self.volume = torch.zeros(n + 1, dtype=torch.float64, device=b.device)
        self.tiles = [np.unique(i // 1296) for i in index]
        self.arg = _lib.Inflow(n, self.start.ctypes.data, self.lowest.ctypes.data, self.min_depth.ctypes.data,
                               self.cells.data_ptr(), self.rained.data_ptr(), float(area),
                               self.volume.data_ptr())  # fmt: skip

    def window(self, t0: float, t1: float) -> np.ndarray:
        """Add the window's inflow rates to src on the device; return the tiles of the injections that flow in it."""
        q = np.array([inj.mean_flow(t0, t1) for inj in self.injections], np.float64)
        b = self.model.backend
        _lib.call("w2b_inflow_window", b.handle, ctypes.byref(self.arg), q.ctypes.data, float(t0), float(t1),
                  b._stream())  # fmt: skip
        flowing = [self.tiles[i] for i in range(len(q)) if q[i] > 0.0]
        return np.concatenate(flowing) if flowing else np.zeros(0, np.int64)

    def total(self) -> float:
        """The inflow volume of every window so far, m3 (FP64, summed as the host form sums it)."""
        return float(self.volume[len(self.injections)].item())


class DeviceStorage:
    """FP64 storage (h + res) over a set of cells, on the device (w2b_storage)."""

    def __init__(self, model, cells) -> None:
        b = model.backend
        torch = b.torch
        self.model = model
        native = native_of_ref(model.grid.tiles, cells, model.grid.shape[1]).astype(np.int32)
        self.cells = torch.as_tensor(native, device=b.device)
        self.partial = torch.zeros(_lib.PARTIALS, dtype=torch.float64, device=b.device)
        self.out = torch.zeros(1, dtype=torch.float64, device=b.device)

    def launch(self) -> None:
        """The storage into ``out`` (a device FP64 scalar), on the current stream, without waiting for it."""
        b = self.model.backend
        _lib.call("w2b_storage", b.handle, int(self.cells.numel()), self.cells.data_ptr(), self.partial.data_ptr(),
                  self.out.data_ptr(), b._stream())  # fmt: skip

    def __call__(self) -> float:
        self.launch()
        return float(self.out.item())


class MonitorReads:
    """What the run driver's monitor reads after each window (wadi2d/engine/monitor.py:197-218, :229-232), in one
    round trip: each design line's discharge, the outfall volume and the FP64 storage are queued on the current stream
    into one pinned buffer and read after a single synchronisation, where reading them one by one waits on the device
    once each. The figures are the same as ``Lines.discharge``, ``Tally.volume`` and ``DeviceStorage`` give."""

    def __init__(self, model, lines=None, tally=None, storage=None) -> None:
        b = model.backend
        self.b, self.torch = b, b.torch
        self.lines, self.tally, self.storage = lines, tally, storage
        self.nl = 0 if lines is None else int(lines.n)
        self.buf = self.torch.zeros(self.nl + 2, dtype=self.torch.float64, device=b.device)
        self.host = self.torch.zeros(self.nl + 2, dtype=self.torch.float64).pin_memory()

    def __call__(self) -> tuple[np.ndarray, float, float]:
        """(each line's discharge m3/s, the outfall volume m3, the storage m3); 0 for what was not given."""
        nl, buf = self.nl, self.buf
        if nl:
            buf[:nl].copy_(self.lines.discharge_device())
        if self.tally is not None and self.tally.n:
            buf[nl].copy_(self.tally.total.sum())
        if self.storage is not None:
            self.storage.launch()
            buf[nl + 1].copy_(self.storage.out[0])
        self.host.copy_(buf, non_blocking=True)
        self.torch.cuda.current_stream(self.b.device).synchronize()
        h = self.host.numpy()
        outflow = 0.0 if self.tally is None else (self.tally.held + float(h[nl]) if self.tally.n else self.tally.held)
        return h[:nl].copy(), outflow, float(h[nl + 1])


class SourceStager:
    """Double-buffered upload of the source field, for a host whose next window's rates are known before the current
    window has stepped (rain read from a radar or forecast grid, a precomputed storm): ``stage`` copies the next
    window's rates, NATIVE layout, from pinned host memory into a device buffer on a side stream and returns at once;
    ``commit`` (at the window's start) makes the step's stream wait for that copy and puts the rates in place with a
    device-to-device copy (w2b_set_field, about 20 us for 16.8 M cells). The host-to-device copy thus overlaps the
    stepping of the window before. The host buffer must not change until the next ``commit`` has returned."""

    def __init__(self, model) -> None:
        b = model.backend
        self.b, self.torch = b, b.torch
        self.buf = self.torch.empty(b.native("src").numel(), dtype=self.torch.float32, device=b.device)
        self.side = self.torch.cuda.Stream(device=b.device)
        self.ready = self.torch.cuda.Event()
        self.pending = False

    def stage(self, rates) -> int:
        """Start the copy of ``rates`` (a pinned host tensor of the NATIVE field's size); returns its bytes."""
        if rates.numel() != self.buf.numel() or rates.dtype != self.torch.float32:
            raise ValueError(f"stage: {rates.numel()} {rates.dtype} values for {self.buf.numel()} float32")
        if self.pending:
            raise RuntimeError("stage: the rates staged before have not been committed")
        cur = self.torch.cuda.current_stream(self.b.device)
        self.side.wait_stream(cur)  # the buffer's last commit has been copied out
        with self.torch.cuda.stream(self.side):
            self.buf.copy_(rates, non_blocking=True)
        self.ready.record(self.side)
        self.pending = True
        return rates.numel() * 4

    def commit(self) -> None:
        """The staged rates into the source field, ordered on the current stream after their upload."""
        if not self.pending:
            raise RuntimeError("commit: nothing staged")
        cur = self.torch.cuda.current_stream(self.b.device)
        cur.wait_event(self.ready)
        _lib.call("w2b_set_field", self.b.handle, _lib.FIELD_ID["src"], self.buf.data_ptr(), _lib.LAYOUT_NATIVE, 0,
                  cur.cuda_stream)  # fmt: skip
        self.pending = False


@dataclass
class RunSummary:
    t: float
    steps: int
    windows: int
    balance: Balance


def run_windows(model, t_end: float, rain=None, host_forcing=None, window: float = 30.0, maxima=None, tally=None,
                storage=None, on_window=None, inflow=None) -> RunSummary:  # fmt: skip
    """Advance ``model`` to ``t_end`` window by window; rain from ``rain`` (DeviceRain) and lumped inflows from
    ``inflow`` (DeviceInflow), or both from ``host_forcing`` (forcing.Forcing, whose ``state`` are the interior
    cells)."""
    bal = Balance()
    if storage is not None:
        bal.storage0 = bal.storage = storage()
    t = model.stepper.t
    n0 = model.stepper.nsteps
    windows = 0
    while t < t_end - 1e-9:
        t1 = min(t + window, t_end)
        if rain is not None or inflow is not None:
            falling = False
            if rain is not None:
                bal.rain += rain.window(t, t1)
                falling = rain.storm.cumulative_depth(np.array([t1 / 60.0]))[0] > rain.storm.cumulative_depth(
                    np.array([t / 60.0]))[0]
            flowing = inflow.window(t, t1) if inflow is not None else None
            st = model.stepper
            # as set_source_cells does: tiles that take a source stay active while it runs (an injection's tiles
            # whole, a superset of its cells with a nonzero rate: a dry tile stepped is left as it was)
            st.keep_active[:] = False
            if falling:
                st.keep_active[rain.tiles] = True
            if flowing is not None and flowing.size:
                st.keep_active[flowing] = True
            st.keep_active[model.boundary_tiles] = True
            if st.adaptive_active:
                st.rebuild_active(retain=True)
            st.refresh_due = True
        elif host_forcing is not None:
            rate, r, q = host_forcing.rate(t, t1)
            model.set_source_cells(host_forcing.state, rate)
            bal.rain += r
            bal.inflow += q
        model.run(t1, maxima=maxima, tally=tally)
        t = model.stepper.t
        windows += 1
        if on_window is not None:
            on_window(t, bal)
    if inflow is not None:
        bal.inflow = inflow.total()
    if tally is not None:
        bal.outflow = tally.volume()
    if storage is not None:
        bal.storage = storage()
    return RunSummary(t, model.stepper.nsteps - n0, windows, bal)
