"""The surrogate network's kernels on the B200: the tensor-core GEMM (tcgen05.mma, BF16 operands, FP32 accumulator)
against FP64 products of the same BF16 values, over the shapes the network uses (batches past one 128-row tile, K
in several chunks, N from 16 to 256); and the element-wise training kernels against their definitions."""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _bf16(rng, shape, scale=1.0):
    import torch

    return (torch.as_tensor(rng.standard_normal(shape) * scale, dtype=torch.float32)).to(torch.bfloat16).cuda()


@pytest.mark.parametrize("m,n,k", [(128, 16, 16), (300, 256, 256), (513, 64, 48), (16, 256, 512), (200, 16, 256),
                                   (1000, 128, 160)])  # fmt: skip
def test_tensor_core_gemm_matches_fp64(m, n, k):
    import torch

    from wadi2d_b200 import _lib

    rng = np.random.default_rng(m * 7 + n + k)
    a, b = _bf16(rng, (m, k)), _bf16(rng, (n, k))
    bias = torch.as_tensor(rng.standard_normal(n), dtype=torch.float32).cuda()
    c = torch.full((m, n), np.nan, dtype=torch.float32, device="cuda")
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    _lib.call("w2b_mma_gemm", a.data_ptr(), b.data_ptr(), m, n, k, bias.data_ptr(), c.data_ptr(), status.data_ptr(), s)
    torch.cuda.synchronize()
    assert int(status.item()) == 0
    want = a.double().cpu().numpy() @ b.double().cpu().numpy().T + bias.double().cpu().numpy()
    got = c.cpu().numpy().astype(np.float64)
    assert np.all(np.isfinite(got))
    scale = np.sqrt(k)  # sums of k unit products
    np.testing.assert_allclose(got, want, rtol=0, atol=2e-6 * scale * max(1.0, float(np.abs(want).max())))
    # no bias: the same products
    _lib.call("w2b_mma_gemm", a.data_ptr(), b.data_ptr(), m, n, k, None, c.data_ptr(), status.data_ptr(), s)
    torch.cuda.synchronize()
    np.testing.assert_allclose(c.cpu().numpy(), want - bias.double().cpu().numpy(), rtol=0,
                               atol=2e-6 * scale * max(1.0, float(np.abs(want).max())))  # fmt: skip


def test_elementwise_training_kernels():
    import torch

    from wadi2d_b200 import _lib

    rng = np.random.default_rng(3)
    s = torch.cuda.current_stream().cuda_stream
    z = torch.as_tensor(rng.standard_normal((37, 48)), dtype=torch.float32).cuda()
    out = torch.empty((37, 48), dtype=torch.bfloat16, device="cuda")
    _lib.call("w2b_bf16_act", z.data_ptr(), z.numel(), 1, out.data_ptr(), s)
    assert torch.equal(out, torch.relu(z).to(torch.bfloat16))
    _lib.call("w2b_bf16_act", z.data_ptr(), z.numel(), 0, out.data_ptr(), s)
    assert torch.equal(out, z.to(torch.bfloat16))
    g = torch.as_tensor(rng.standard_normal((37, 48)), dtype=torch.float32).cuda()
    _lib.call("w2b_relu_back", g.data_ptr(), z.data_ptr(), g.numel(), out.data_ptr(), s)
    assert torch.equal(out, torch.where(z > 0, g, torch.zeros_like(g)).to(torch.bfloat16))
    x = _bf16(rng, (37, 48))
    xt = torch.full((48, 64), 7.0, dtype=torch.bfloat16, device="cuda")
    _lib.call("w2b_transpose_bf16", x.data_ptr(), 37, 48, 64, xt.data_ptr(), s)
    assert torch.equal(xt[:, :37], x.T) and torch.all(xt[:, 37:] == 0)
    cs = torch.empty(48, dtype=torch.float32, device="cuda")
    _lib.call("w2b_colsum_bf16", x.data_ptr(), 37, 48, cs.data_ptr(), s)
    np.testing.assert_allclose(cs.cpu().numpy(), x.float().sum(0).cpu().numpy(), rtol=1e-5, atol=1e-5)
    y = torch.as_tensor(rng.standard_normal((40, 16)), dtype=torch.float32).cuda()
    t = torch.as_tensor(rng.standard_normal((40, 16)), dtype=torch.float32).cuda()
    dy = torch.empty((48, 16), dtype=torch.bfloat16, device="cuda")
    part = torch.zeros(64, dtype=torch.float64, device="cuda")
    _lib.call("w2b_mse_grad", y.data_ptr(), t.data_ptr(), 40, 48, 16, 0.5, dy.data_ptr(), part.data_ptr(), s)
    assert torch.equal(dy[:40], (0.5 * (y - t)).to(torch.bfloat16)) and torch.all(dy[40:] == 0)
    assert float(part.sum()) == pytest.approx(float(((y - t).double() ** 2).sum()), rel=1e-12)
    w = torch.as_tensor(rng.standard_normal(1000), dtype=torch.float32).cuda()
    gr = torch.as_tensor(rng.standard_normal(1000), dtype=torch.float32).cuda()
    m1, v1 = torch.zeros_like(w), torch.zeros_like(w)
    wb = torch.empty(1000, dtype=torch.bfloat16, device="cuda")
    w0 = w.clone()
    _lib.call("w2b_adam", w.data_ptr(), gr.data_ptr(), m1.data_ptr(), v1.data_ptr(), 1000, 1e-3, 0.9, 0.999, 1e-8,
              wb.data_ptr(), s)  # fmt: skip
    mm, vv = 0.1 * gr, 0.001 * gr * gr
    np.testing.assert_allclose(w.cpu().numpy(), (w0 - 1e-3 * mm / (torch.sqrt(vv) + 1e-8)).cpu().numpy(), rtol=1e-6,
                               atol=1e-7)  # fmt: skip
    assert torch.equal(wb, w.to(torch.bfloat16))
