"""Golden vectors of the reference's loss, storm and ARF arithmetic (the parts of its forcing that import without
its GIS dependencies). Run where the reference tree is importable:

    WADI2D_REFERENCE=<the reference source tree> PYTHONDONTWRITEBYTECODE=1 python tests/golden/make_golden_forcing.py

It writes tests/golden/forcing.npz: SCS cumulative excess over curve numbers x depths (with and without a given
initial abstraction), ARF table factors over areas (both ends' rules), uniform-storm cumulative depths, and the
lumped-inflow injections' exact volume integrals, window mean flows and depth shares (wadi2d/forcing.py:427-477).
The reference's forcing module imports GIS packages that this container lacks (shapely, rasterio, ...); the
injection arithmetic uses none of them, so they are stubbed for the import."""

from __future__ import annotations

import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
if not os.environ.get("WADI2D_REFERENCE"):
    sys.exit("set WADI2D_REFERENCE to the reference source tree")
sys.path.insert(0, os.environ["WADI2D_REFERENCE"])


class _Stub:
    """A stand-in module for a missing GIS package, so that the reference's forcing module imports."""

    MISSING = ("shapely", "rasterio", "h5py", "pyproj", "fiona", "contourpy", "openpyxl", "hecdss", "cupy")

    def find_spec(self, name, path, target=None):
        import importlib.machinery

        if name.split(".")[0] in self.MISSING:
            return importlib.machinery.ModuleSpec(name, self, is_package=True)
        return None

    def create_module(self, spec):
        from unittest import mock

        m = mock.MagicMock(name=spec.name)
        m.__path__ = []
        m.__spec__ = spec
        return m

    def exec_module(self, module):
        pass


sys.meta_path.insert(0, _Stub())

from wadi2d.forcing import Injection  # noqa: E402
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
    # injections: a triangular hydrograph, a multi-point one with a plateau, and one starting late
    hydro = [
        (np.array([0.0, 3600.0, 9600.0]), np.array([0.0, 200.0, 0.0])),
        (np.array([0.0, 600.0, 1800.0, 2400.0, 7200.0, 10000.0]), np.array([5.0, 80.0, 80.0, 350.0, 40.0, 0.0])),
        (np.array([1200.0, 4000.0, 4001.0, 20000.0]), np.array([0.0, 55.5, 120.25, 0.0])),
    ]
    inj_t = np.concatenate(([-5.0, 0.0, 1e-3], np.linspace(0.0, 21000.0, 701)[1:], [3600.0, 4000.5, 9599.999]))
    windows = np.stack([np.arange(0.0, 21000.0, 30.0), np.arange(30.0, 21030.0, 30.0)], axis=1)
    inj_vol, inj_q = [], []
    for times, flows in hydro:
        inj = Injection("g", np.arange(5), np.arange(5), 2, times, flows, 0.01)
        inj_vol.append([inj.volume_at(float(t)) for t in inj_t])
        inj_q.append([inj.mean_flow(float(a), float(b)) for a, b in windows])
    rng = np.random.default_rng(12)
    depths = np.concatenate((np.zeros((1, 5)), np.full((1, 5), 0.005), rng.random((30, 5)) * 0.05,
                             np.where(rng.random((10, 5)) < 0.5, 0.0, rng.random((10, 5)))))  # fmt: skip
    inj = Injection("s", np.arange(5), np.arange(5), 3, hydro[0][0], hydro[0][1], 0.01)
    shares = np.stack([inj.share(d) for d in depths])
    np.savez_compressed(HERE / "forcing.npz", cn=cn, depth=depth, scs=scs, scs_ia=scs_ia, areas=areas,
                        factors=factors, probe=probe, arf_a=arf_a, arf_b=arf_b, given=given, minutes=minutes,
                        uniform=uni, inj_t=inj_t, inj_windows=windows, inj_vol=np.array(inj_vol),
                        inj_q=np.array(inj_q), inj_depths=depths, inj_shares=shares,
                        inj_len=np.array([h[0].size for h in hydro]),
                        inj_times=np.concatenate([h[0] for h in hydro]),
                        inj_flows=np.concatenate([h[1] for h in hydro]))  # fmt: skip
    print("forcing.npz written")


if __name__ == "__main__":
    main()
