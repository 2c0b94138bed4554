"""The table build for callers that cannot allocate device memory (w2b_build_tables_noalloc).

Such a caller (a host program whose device memory belongs to a pool or caching allocator it does not control, or an
FFI binding with no allocator of its own) passes inputs and outputs but no scratch; the entry point uses the
library's own fixed 32 MiB device array instead. Here it is called twice in a row through the C-ABI, and each result
must equal, bit for bit, the tables of the entry point that takes the caller's scratch. Two face-line lengths:
configuration 1's (149 pixels), whose local-radius workspace fits in shared memory, and one of 3,005 pixels (a
margin of 1,500 pixels), beyond the 2,843 pixels shared memory holds, so the face-table kernel works in the static
array itself. This file is collected last, so a run that stops at its first failure has already run every other
test; it also passes alone in a fresh process.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

import cases
from oracle_api import OracleApi

pytestmark = pytest.mark.gpu


def _marshal(torch, dev, grid, z, pixel, manning, local, margin):
    """Device inputs and zeroed outputs of one table build, as the C-ABI structures want them."""
    from wadi2d_b200.tablebuild import TILE_FIELDS, TableIn, TableOut

    ny, nx = grid.shape
    nt, rows, k = grid.ntiles, 16, round(grid.dx / pixel)
    keep = []

    def d64(a):
        t = torch.as_tensor(np.ascontiguousarray(a, np.float64), device=dev)
        keep.append(t)
        return t.data_ptr()

    nan = np.full((ny, nx), np.nan)
    mask = torch.as_tensor(np.ascontiguousarray(grid.mask, np.uint8), device=dev)
    tiles = torch.as_tensor(np.ascontiguousarray(grid.tiles, np.int32), device=dev)
    keep += [mask, tiles]
    tin = TableIn(
        d64(z), z.shape[0], z.shape[1], 0, 0, None, d64(np.full((ny, nx), manning)), d64(nan), d64(np.ones((ny, nx))),
        d64(np.zeros((ny, nx))), d64(nan), d64(np.ones((ny, nx))), d64(np.zeros((ny, nx))), None, None,
        mask.data_ptr(), tiles.data_ptr(), nt, ny, nx, k, rows, int(local), margin, float(pixel), 8.0, 16.0, 9.0, 0.05,
    )  # fmt: skip

    def outputs():
        out = {}
        for n in TILE_FIELDS:
            shape = {"dtab": (nt, 32, 32, rows), "ftabx": (nt, 32, 32, rows, 2), "ftaby": (nt, 32, 32, rows, 2)}.get(
                n, (nt, 32, 32)
            )
            out[n] = torch.full(shape, 1.0 if n in ("efx", "efy") else 0.0, dtype=torch.float32, device=dev)
        for n in ("zmin", "rel", "zfx", "zfy"):
            out[n] = torch.zeros((ny, nx), dtype=torch.float64, device=dev)
        return out

    return tin, outputs, keep, TableOut


SHARED_LINE_MAX = 204800 // (9 * 8) - 1  # 2,843: the longest line whose workspace fits a CTA's 200 KiB
ARRAY_LINE_MAX = (32 << 20) // (128 * 9 * 8) - 1  # 3,639: the longest line the 32 MiB array holds for 128 threads


@pytest.mark.parametrize("n, margin", [(64, None), (30, 1500)], ids=["shared_memory_lines", "static_array_lines"])
def test_noalloc_table_build_equals_the_scratch_build_twice_in_a_row(n, margin):
    import torch

    from wadi2d_b200 import _lib
    from wadi2d_b200.tablebuild import TILE_FIELDS

    lib = _lib.lib()
    dev = torch.device("cuda")
    stream = torch.cuda.current_stream().cuda_stream
    grid, (z, pixel, manning, local, _, _), _ = cases.c1_small_inputs(OracleApi(), n=n)
    k = round(grid.dx / pixel)
    if margin is None:
        margin = int(min(np.ceil(9.0 * 16.0 / pixel), max(z.shape)))
        assert k + 2 * margin <= SHARED_LINE_MAX
    else:
        assert SHARED_LINE_MAX < k + 2 * margin <= ARRAY_LINE_MAX  # the face kernel's workspace is the array
    tin, outputs, keep, TableOut = _marshal(torch, dev, grid, z, pixel, manning, local, margin)
    names = TILE_FIELDS + ("zmin", "rel", "zfx", "zfy")

    def out_struct(o, ws=None, threads=0):
        return TableOut(*(o[n].data_ptr() for n in names), None if ws is None else ws.data_ptr(), threads)

    lib.w2b_build_tables.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    lib.w2b_build_tables_noalloc.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    lib.w2b_build_tables_noalloc.restype = ctypes.c_int32

    # the entry point that takes the caller's scratch
    threads = 148 * 8 * 128 if k + 2 * margin <= SHARED_LINE_MAX else 1024
    ws = torch.empty(9 * (k + 2 * margin + 1) * threads, dtype=torch.float64, device=dev)
    ref = outputs()
    assert lib.w2b_build_tables(ctypes.byref(tin), ctypes.byref(out_struct(ref, ws, threads)), stream) == 0
    torch.cuda.synchronize()
    del ws

    # the entry point that allocates nothing, twice in a row
    for call in range(2):
        got = outputs()
        st = lib.w2b_build_tables_noalloc(ctypes.byref(tin), ctypes.byref(out_struct(got)), stream)
        assert st == 0, f"call {call}: status {st}"
        torch.cuda.synchronize()
        for n in names:
            assert torch.equal(got[n], ref[n]), (call, n)
    del keep


def test_noalloc_refuses_lines_beyond_its_scratch():
    import torch

    from wadi2d_b200 import _lib

    lib = _lib.lib()
    grid, (z, pixel, manning, local, _, _), _ = cases.c1_small_inputs(OracleApi())
    tin, outputs, keep, TableOut = _marshal(torch, torch.device("cuda"), grid, z, pixel, manning, local, 4000)
    o = outputs()
    names = list(o)
    st = lib.w2b_build_tables_noalloc(ctypes.byref(tin), ctypes.byref(TableOut(*(o[n].data_ptr() for n in names),
                                                                                   None, 0)), None)  # fmt: skip
    assert st == _lib.EINVAL
    del keep
