"""The learned-CDF CPU oracle's gradient is the derivative of its loss
(finite differences).  CPU only."""
import numpy as np

import cdf_oracle


def test_cpu_oracle_gradient_is_the_derivative():
    rng = np.random.default_rng(2)
    keys = np.sort(rng.integers(0, 1 << 30, 4000))
    L = 4
    lo, sc = float(keys[0]), 1.0 / float(keys[-1] - keys[0])
    p = np.array([0.95, 0.02, 0.9, 0.05, 1.1, -0.02, 0.7, 0.1, 1.0, 0.0], dtype=np.float32)
    _, g = cdf_oracle.loss_grad(keys, L, p, lo, sc)
    for i in range(2, 2 + 2 * L):  # leaf parameters (root changes the leaf assignment)
        h = 1e-3
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd = (cdf_oracle.loss_grad(keys, L, pp, lo, sc)[0] - cdf_oracle.loss_grad(keys, L, pm, lo, sc)[0]) / (
            float(pp[i]) - float(pm[i]))
        assert abs(fd - g[i]) < 1e-4 + 1e-2 * abs(g[i])
