"""The surrogate network on the B200 against its FP64 oracle (oracle/mlp.py, which rounds to BF16 where the device
does): forward outputs and every weight and bias gradient on a random batch, and training that fits a smooth map."""

from __future__ import annotations

import numpy as np
import pytest

from oracle import mlp as OM

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


def test_forward_and_gradients_match_the_oracle():
    from wadi2d_b200.surrogate import Network

    net = Network(seed=1)
    rng = np.random.default_rng(2)
    x = rng.standard_normal((200, 16)).astype(np.float32)
    t = rng.standard_normal((200, 16)).astype(np.float32)
    w = net.weights()
    y = net.predict(x)
    yo, _, _ = OM.forward(w, x)
    assert _rel(y, yo) < 2e-3
    loss, gW, gb = net.gradients(x, t)
    lo, gWo, gbo = OM.gradients(w, x, t)
    assert float(loss) == pytest.approx(lo, rel=1e-3)
    for i in range(len(gW)):
        assert _rel(gW[i].cpu().numpy(), gWo[i]) < 1e-2, i
        assert _rel(gb[i].cpu().numpy(), gbo[i]) < 1e-2, i


def test_training_fits_a_smooth_map():
    from wadi2d_b200.surrogate import Network

    rng = np.random.default_rng(5)
    a = rng.standard_normal((16, 16)) / 4.0
    x = rng.standard_normal((1024, 16)).astype(np.float32)
    t = np.tanh(x @ a).astype(np.float32) + 0.1 * (x[:, :1] ** 2)
    t = ((t - t.mean(0)) / t.std(0)).astype(np.float32)
    net = Network(seed=3, lr=2e-3)
    losses = net.fit(x[:896], t[:896], iters=1500, batch=256)
    assert losses[-1] < 0.05 * losses[0]
    err = np.mean((net.predict(x[896:]) - t[896:]) ** 2)
    assert err < 0.25  # held-out rows: the mean alone scores 1 on standardised targets


def test_training_replayed_as_a_graph_equals_stepping_from_the_host():
    """The captured training step, replayed with each step's batch and step size read on the device, gives the same
    weights, bit for bit, and the same losses as the same steps launched one by one from the host."""
    from wadi2d_b200.surrogate import Network

    rng = np.random.default_rng(8)
    x = rng.standard_normal((300, 16)).astype(np.float32)
    t = rng.standard_normal((300, 16)).astype(np.float32)
    nets = [Network(seed=4), Network(seed=4)]
    lg = nets[0].fit(x, t, iters=250, batch=96, seed=6, graph=True)
    lh = nets[1].fit(x, t, iters=250, batch=96, seed=6, graph=False)
    assert lg == lh
    for (wg, bg), (wh, bh) in zip(nets[0].weights(), nets[1].weights(), strict=True):
        assert np.array_equal(wg, wh) and np.array_equal(bg, bh)
    assert nets[0].t == nets[1].t == 250
    # a second fit continues the step count and the moments the same way
    lg = nets[0].fit(x, t, iters=120, batch=96, seed=7, graph=True)
    lh = nets[1].fit(x, t, iters=120, batch=96, seed=7, graph=False)
    assert lg == lh
    assert all(np.array_equal(a[0], b[0]) for a, b in zip(nets[0].weights(), nets[1].weights(), strict=True))
