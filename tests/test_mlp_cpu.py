# SPDX-License-Identifier: MIT
"""The CPU restatement of the warm-start MLP (oracle/mlp.py): its analytic
gradient equals central finite differences of its own loss (float64, no
BF16 rounding), and padding parameters receive exactly zero gradient."""
import numpy as np

import mlp as M


def _batch(n, seed):
    rng = np.random.default_rng(seed)
    f = rng.uniform(-1.0, 1.0, (n, M.FEATURES))
    y = rng.uniform(-0.5, 1.5, (n, 2))
    w = np.full(n, 1.0 / n)
    return f, y, w


def test_gradient_matches_finite_differences():
    f, y, w = _batch(24, 3)
    p = M.init_params(7).astype(np.float64)
    _, g, _ = M.forward_backward(f, y, w, p, bf16_round=False)
    rng = np.random.default_rng(11)
    live = [i for i in range(M.PARAMS) if g[i] != 0.0]
    idx = list(rng.choice(live, 60, replace=False)) + [M.W1 + 8, M.W2 + 64, M.W3 + 64, M.W3 + M.HIDDEN_K + 64]
    eps = 1e-6
    for i in idx:
        q = p.copy()
        q[i] += eps
        lp = M.forward_backward(f, y, w, q, bf16_round=False)[2]
        q[i] -= 2 * eps
        lm = M.forward_backward(f, y, w, q, bf16_round=False)[2]
        fd = (lp - lm) / (2 * eps)
        assert abs(fd - g[i]) <= 1e-6 + 1e-4 * abs(g[i]), (i, fd, g[i])


def test_padding_parameters_get_no_gradient():
    f, y, w = _batch(50, 5)
    p = M.init_params(2)
    _, g, _ = M.forward_backward(f, y, w, p)
    w1 = g[M.W1:M.W2].reshape(M.HIDDEN, M.IN)
    w2 = g[M.W2:M.W3].reshape(M.HIDDEN, M.HIDDEN_K)
    w3 = g[M.W3:].reshape(M.OUT_N, M.HIDDEN_K)
    assert not w1[:, M.FEATURES + 1:].any()
    assert not w2[:, M.HIDDEN + 1:].any()
    assert not w3[M.OUT:].any() and not w3[:, M.HIDDEN + 1:].any()
    assert w1[:, M.FEATURES].any() and w2[:, M.HIDDEN].any() and w3[:M.OUT, M.HIDDEN].any()


def test_bf16_rounding_is_nearest_even():
    v = np.array([1.0, 1.00390625, 1.005859375, 1.0078125 + 2 ** -9, -3.14159], np.float32)
    r = M.bf16(v)
    assert r[0] == 1.0 and r[1] == 1.0          # halfway rounds to even
    assert r[2] == 1.0078125                    # above halfway rounds up
    assert abs(r[4] + 3.140625) < 1e-12
