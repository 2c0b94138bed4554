"""The C-ABI library loads and exports every entry point include/wadi_b200.h declares; the host-only entry points
(layout and index conversion) agree with the Python layout helpers. No GPU needed."""

from __future__ import annotations

import ctypes
import re
from pathlib import Path

import numpy as np

from wadi2d_b200 import _lib, build, layout
from wadi2d_b200.grid import TileGrid

HEADERS = sorted((Path(__file__).resolve().parents[1] / "include").glob("*.h"))


def declared() -> list[str]:
    names = []
    for h in HEADERS:
        names += re.findall(r"^\s*(?:int32_t|int64_t)\s+(w2b_\w+)\s*\(", h.read_text(), flags=re.M)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    build.build()
    lib = _lib.lib()
    names = declared()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_every_declared_entry_point_is_bound_and_no_other():
    assert set(_lib._SIGNATURES) == set(declared())


def test_layout_and_index_conversion_match_python():
    rng = np.random.default_rng(0)
    mask = rng.random((70, 90)) > 0.3
    g = TileGrid.from_mask(mask, 0.0, 0.0, 10.0)
    desc = _lib.GridDesc(g.shape[0], g.shape[1], g.ntiles, 16)
    lay = _lib.Layout()
    assert _lib.lib().w2b_layout(ctypes.byref(desc), ctypes.byref(lay)) == 0
    assert lay.px == layout.native_pitch(g.shape[1])
    assert lay.ncells == layout.native_size(*g.shape)
    ref = rng.integers(layout.STRIDE2, g.ntiles * layout.STRIDE2, 5000).astype(np.int64)
    out = np.zeros_like(ref)
    tiles = np.ascontiguousarray(g.tiles, np.int32)
    st = _lib.lib().w2b_ref_to_native(ctypes.byref(desc), tiles.ctypes.data, ref.size, ref.ctypes.data,
                                      out.ctypes.data)  # fmt: skip
    assert st == 0
    assert np.array_equal(out, layout.native_of_ref(g.tiles, ref, g.shape[1]))


def test_bad_arguments_are_refused_without_a_gpu():
    bad = _lib.GridDesc(33, 64, 2, 16)
    assert _lib.lib().w2b_layout(ctypes.byref(bad), ctypes.byref(_lib.Layout())) == _lib.EINVAL
    g = _lib.GridDesc(64, 64, 2, 16)
    tiles = np.array([[-1, -1], [0, 0]], np.int32)
    ref = np.array([5], np.int64)  # an entry of the void tile
    out = np.zeros(1, np.int64)
    assert _lib.lib().w2b_ref_to_native(ctypes.byref(g), tiles.ctypes.data, 1, ref.ctypes.data, out.ctypes.data) == -1


def test_every_entry_point_refuses_null_arguments_without_a_gpu():
    """Every entry point checks its handle and pointers before it touches the device: called with null pointers and
    zero sizes, each returns W2B_EINVAL (the sizing queries return their sizes)."""
    sizes = {"w2b_version", "w2b_run_table_bytes", "w2b_table_workspace_doubles"}
    L = _lib.lib()
    for name, args in _lib._SIGNATURES.items():
        if name in sizes:
            continue
        zeros = [0.0 if a in (ctypes.c_float, ctypes.c_double) else (0 if a in (ctypes.c_int32, ctypes.c_int64,
                 ctypes.c_uint32) else None) for a in args]  # fmt: skip
        assert getattr(L, name)(*zeros) == _lib.EINVAL, name
    assert L.w2b_version() == 3
    assert L.w2b_run_table_bytes(0) == 0


def test_table_build_refuses_a_bad_margin_without_a_gpu():
    """With the local radius on, a negative margin or one beyond W2B_TABLE_MARGIN_MAX is refused before any device
    work, by both table-build entry points."""
    from wadi2d_b200.tablebuild import TableIn, TableOut

    L = _lib.lib()
    fake = 256  # never dereferenced: the arguments are checked first
    for margin in (-1, (1 << 20) + 1, -(1 << 30)):
        tin = TableIn(fake, 64, 64, 0, 0, None, fake, None, None, None, None, None, None, None, None, fake, fake, 2, 32,
                      32, 2, 16, 1, margin, 1.0, 8.0, 16.0, 9.0, 0.05)  # fmt: skip
        out = TableOut(*([None] * 22), fake, 128)
        assert L.w2b_build_tables(ctypes.byref(tin), ctypes.byref(out), None) == _lib.EINVAL, margin
        assert L.w2b_build_tables_noalloc(ctypes.byref(tin), ctypes.byref(out), None) == _lib.EINVAL, margin
