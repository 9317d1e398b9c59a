"""The surrogate network's CPU oracle, pinned by central finite differences
(no GPU): its analytic FP64 gradient of the mean squared error matches the
numerical derivative, and its bfloat16 rounding helper rounds to nearest
even."""
from __future__ import annotations

import numpy as np

from oracle.mlp_oracle import MlpOracle, bf16_round


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(3)
    net = MlpOracle(n_in=7, width=64, depth=2, n_out=64)
    p = rng.normal(0, 0.2, net.n_params)
    X = rng.normal(0, 1, (5, 7))
    Y = rng.normal(0, 1, (5, 64))
    _, g = net.loss_grad(p, X, Y)
    # every non-padded parameter of a sample of indices, by central differences
    W0 = net.kin * 64
    idx = [q for q in rng.choice(net.n_params, 400, replace=False) if not (q < W0 and (q % net.kin) >= 7)]
    h = 1e-6
    for q in idx:
        pp, pm = p.copy(), p.copy()
        pp[q] += h
        pm[q] -= h
        num = (net.loss_grad(pp, X, Y)[0] - net.loss_grad(pm, X, Y)[0]) / (2 * h)
        assert abs(num - g[q]) <= 1e-6 * max(1.0, abs(g[q])) + 1e-9, (q, num, g[q])


def test_bf16_rounding_is_nearest_even():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -9, -2.5, 3.1415926], dtype=np.float64)
    r = bf16_round(x)
    assert r[0] == 1.0
    assert r[1] == 1.0                      # halfway: ties to even (1.0)
    assert r[2] == 1.0 + 2 ** -7            # above half: up
    assert r[3] == -2.5
    assert abs(r[4] - 3.140625) < 1e-12
