"""fp64 NumPy restatement of the learned-CDF model's loss and gradient
(the formulas documented in include/pyg_learned.h), used by the tests to
check the GPU forward / backward kernels.  TEST INFRASTRUCTURE ONLY.

There is no reference counterpart (the reference splits key ranges with the
equal-width ExactRangeValueHasher, hash.h:452-487); this oracle is pinned by
a finite-difference check of its own gradient in the tests.
"""
import numpy as np


def norm_keys(sorted_keys, key_lo, key_scale):
    x = (sorted_keys.astype(np.float64) - key_lo) * key_scale
    return x.astype(np.float32).astype(np.float64)  # the device rounds x to fp32


def loss_grad(sorted_keys, L, params, key_lo, key_scale):
    """Returns (loss, grad) for params = [a0, b0, a_0, b_0, ..., a_{L-1}, b_{L-1}]."""
    p = np.asarray(params, dtype=np.float32).astype(np.float64)
    n = sorted_keys.shape[0]
    x = norm_keys(sorted_keys, key_lo, key_scale)
    y = np.arange(n, dtype=np.float64) / n
    a0, b0 = p[0], p[1]
    r = a0 * x + b0
    e = r - y
    loss = float(np.sum(e * e) / n)
    grad = np.zeros(2 + 2 * L)
    grad[0] = 2.0 / n * np.sum(e * x)
    grad[1] = 2.0 / n * np.sum(e)
    leaf = np.clip(np.floor(L * r), 0, L - 1).astype(np.int64)
    u = np.clip(L * r - leaf, 0.0, 1.0)
    idx = np.arange(n)
    for l in np.unique(leaf):
        m = leaf == l
        lo, hi = idx[m].min(), idx[m].max() + 1
        nl = hi - lo
        ylo, yhi = lo / n, hi / n
        t = (y[m] - ylo) / (yhi - ylo) if yhi > ylo else np.zeros(nl)
        g = p[2 + 2 * l] * u[m] + p[3 + 2 * l] - t
        loss += float(np.sum(g * g) / nl / L)
        grad[2 + 2 * l] = 2.0 / (nl * L) * np.sum(g * u[m])
        grad[3 + 2 * l] = 2.0 / (nl * L) * np.sum(g)
    return loss, grad


def imbalance(keys, splitters):
    """max / mean partition size of keys under range splitters."""
    fan = len(splitters) + 1
    b = np.searchsorted(np.asarray(splitters), keys, side="right")
    c = np.bincount(b, minlength=fan)
    return c.max() / (len(keys) / fan)
