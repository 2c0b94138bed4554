"""The network oracle (oracle/mlp.py) on CPU: its gradients against central finite differences of its own loss in
plain FP64, for every layer's weights and biases, and the BF16 rounding against known values."""

from __future__ import annotations

import numpy as np
import pytest

from oracle import mlp as OM


def _weights(rng, dims=(16, 32, 32, 16)):
    return [(rng.standard_normal((o, i)) * np.sqrt(2.0 / i), rng.standard_normal(o) * 0.1)
            for i, o in zip(dims[:-1], dims[1:], strict=True)]  # fmt: skip


def test_gradients_match_finite_differences():
    rng = np.random.default_rng(0)
    w = _weights(rng)
    x, t = rng.standard_normal((40, 16)), rng.standard_normal((40, 16))
    _, gW, gb = OM.gradients(w, x, t, rounded=False)
    eps = 1e-6
    for layer in range(len(w)):
        for kind in (0, 1):
            d = rng.standard_normal(w[layer][kind].shape)
            plus = [(a.copy(), b.copy()) for a, b in w]
            minus = [(a.copy(), b.copy()) for a, b in w]
            plus[layer] = tuple(v + eps * d if q == kind else v for q, v in enumerate(w[layer]))
            minus[layer] = tuple(v - eps * d if q == kind else v for q, v in enumerate(w[layer]))
            fd = (OM.gradients(plus, x, t, False)[0] - OM.gradients(minus, x, t, False)[0]) / (2 * eps)
            an = float(((gW if kind == 0 else gb)[layer] * d).sum())
            assert fd == pytest.approx(an, rel=1e-5, abs=1e-9), (layer, kind)


def test_bf16_rounds_to_nearest_even():
    x = np.array([1.0, 1.0 + 2.0**-8, 1.0 + 3 * 2.0**-8, 1.0 + 2.0**-9, -3.14159, 0.0])
    assert list(OM.bf16(x)) == [1.0, 1.0, 1.0 + 2.0**-6, 1.0, -3.140625, 0.0]
