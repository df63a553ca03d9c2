"""The CPU oracle of the surrogate network, pinned by finite differences
(float64), before it is used to check the GPU gradients."""
from __future__ import annotations

import numpy as np

from oracle import mlp_oracle as mo


def test_layout_size():
    _, total = mo.layout()
    assert total == 4 * 128 + 128 + 2 * (128 * 128 + 128) + 128 + 1 == 33793


def test_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    _, total = mo.layout()
    theta = rng.normal(0, 0.2, total)
    x = mo.features(np.column_stack([rng.uniform(0, 6.28, 40), rng.uniform(0, 1.05, 40), np.zeros(40)]))
    y = rng.normal(size=40)
    loss, g = mo.loss_and_grad(theta, x, y)
    for k in rng.choice(total, 60, replace=False):
        e = np.zeros(total)
        e[k] = 1e-6
        fd = (mo.loss_and_grad(theta + e, x, y)[0] - mo.loss_and_grad(theta - e, x, y)[0]) / 2e-6
        assert abs(fd - g[k]) <= 1e-6 + 1e-5 * abs(fd), (k, fd, g[k])


def test_adam_first_step_is_signed_lr():
    g = np.array([0.3, -2.0, 1e-3])
    th, m, v = mo.adam_step(np.zeros(3), g, np.zeros(3), np.zeros(3), 1, 0.01)
    assert np.allclose(th, -0.01 * np.sign(g), rtol=1e-4)
