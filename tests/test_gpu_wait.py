"""The bounded device wait gives up and says so (w2b_selftest_wait): a barrier that nothing completes, waited on by the
library's own wait, reports W2B_ETIMEOUT after its polls, and the context stays usable (the cube-root self-check runs
after it). The time a poll takes bounds how long the library's limit of 262,144 polls lets a wait that cannot end hold
a kernel: about a second."""

from __future__ import annotations

import pytest

from wadi2d_b200 import _lib

pytestmark = pytest.mark.gpu

LIMIT = 1 << 18  # the polls of every wait in the library


def _wait(polls: int):
    """(status, SM clock cycles, milliseconds by CUDA events on the launching stream) of one self-check."""
    import torch

    out = torch.zeros(2, dtype=torch.int64, device="cuda")
    stream = torch.cuda.current_stream()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    start.record(stream)
    _lib.call("w2b_selftest_wait", polls, out.data_ptr(), stream.cuda_stream)
    end.record(stream)
    torch.cuda.synchronize()
    status, cycles = (int(v) for v in out.cpu())
    return status, cycles, start.elapsed_time(end)


def test_a_wait_that_nothing_completes_gives_up_and_reports():
    import torch

    short, long_ = _wait(1 << 10), _wait(1 << 14)
    assert short[0] == _lib.ETIMEOUT and long_[0] == _lib.ETIMEOUT
    assert 0 < short[1] < long_[1]
    # the context still runs kernels: the cube root of 2^20 floats from 1.0 on, all exact
    out = torch.zeros(5, dtype=torch.int64, device="cuda")
    _lib.call("w2b_selftest_cbrt", 0x3F800000, 1 << 20, out.data_ptr(), torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert int(out[0]) == 0
    per_poll = long_[2] * 1e-3 / (1 << 14)
    print(f"bounded wait: {per_poll * 1e9:.0f} ns and {long_[1] / (1 << 14):.0f} cycles a poll; the library's limit "
          f"ends a wait that cannot end after about {per_poll * LIMIT:.2f} s")
    assert per_poll * LIMIT < 5.0


def test_the_poll_count_is_checked():
    assert _lib.lib().w2b_selftest_wait(0, None, None) == _lib.EINVAL
    assert _lib.lib().w2b_selftest_wait(LIMIT + 1, 1, None) == _lib.EINVAL
