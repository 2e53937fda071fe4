"""The predictor oracle's gradient against central differences of its own loss (CPU)."""

import numpy as np

from oracle import mlp


def loss(w, norm, X, y, pw):
    """Weighted binary cross-entropy from the logits (softplus form, stable when saturated)."""
    _, (x, h1, h2, h3) = mlp.forward(w, norm, X)
    W1, b1, W2, b2, W3, b3, w4, b4 = mlp.unpack(w)
    z = h3 @ w4 + b4
    ws = np.where(y > 0.5, pw, 1.0) / len(y)
    return float((ws * (np.logaddexp(0.0, z) - y * z)).sum())


def test_gradient_matches_central_differences():
    rng = np.random.default_rng(0)
    w = rng.normal(0, 0.1, mlp.PARAMS)
    norm = np.concatenate([rng.normal(0, 1, 8), 1 + rng.random(8)])
    X = rng.normal(0, 1, (40, 8))
    y = (rng.random(40) < 0.3).astype(float)
    g = mlp.gradient(w, norm, X, y, 3.0)
    idx = rng.choice(mlp.PARAMS, 60, replace=False).tolist() + [mlp.OFF["b4"], mlp.OFF["w4"], 0]
    for i in idx:
        h = 1e-6
        wp, wm = w.copy(), w.copy()
        wp[i] += h
        wm[i] -= h
        fd = (loss(wp, norm, X, y, 3.0) - loss(wm, norm, X, y, 3.0)) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 + 1e-5 * abs(fd), (i, fd, g[i])


def test_adam_first_step_moves_by_lr():
    w = np.zeros(4)
    g = np.array([1.0, -2.0, 0.5, 0.0])
    w2, m, v = mlp.adam(w, g, np.zeros(4), np.zeros(4), 1, 0.01)
    np.testing.assert_allclose(w2[:3], -0.01 * np.sign(g[:3]), rtol=1e-6)
    assert w2[3] == 0.0
