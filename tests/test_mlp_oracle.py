"""The emulator's CPU oracle (oracle/mlp_oracle.py) against finite differences."""

import numpy as np

from oracle import mlp_oracle


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    sizes = (5, 12, 9, 1)
    n = sum(a * b + b for a, b in zip(sizes[:-1], sizes[1:]))
    p = rng.normal(0, 0.4, n)
    X = rng.uniform(-1, 1, (40, 5))
    t = rng.normal(0, 1, 40)
    w = rng.uniform(0.5, 1.5, 40)
    loss, g = mlp_oracle.loss_and_grad(p, p, sizes, X, t, w)
    h = 1e-6
    fd = np.empty(n)
    for i in range(n):
        e = np.zeros(n)
        e[i] = h
        lp, _ = mlp_oracle.loss_and_grad(p + e, p + e, sizes, X, t, w)
        lm, _ = mlp_oracle.loss_and_grad(p - e, p - e, sizes, X, t, w)
        fd[i] = (lp - lm) / (2 * h)
    assert np.max(np.abs(g - fd)) <= 1e-7 * max(1.0, np.max(np.abs(fd)))
    assert loss > 0
