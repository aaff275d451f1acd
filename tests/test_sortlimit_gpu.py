"""Top-k (pyg_sortlimit, the reference's `sortlimit`) vs the oracle: the
first `limit` tuples in key order, ties in input order, ascending and
descending, single int64 / int32 keys and (int32, int32) pairs."""
import numpy as np
import pytest

import oracle as O
import pyg
from util import I32, I64, alloc, dev_rel, from_device, host_rel, rows, struct

pytestmark = pytest.mark.gpu


def run(ctx, torch, A, types, by, asc, limit, on_device=True):
    rel = dev_rel(torch, A, types) if on_device else host_rel(A, types)
    cap = max(1, min(limit, A.shape[0]))
    out = alloc(torch, cap * A.dtype.itemsize)
    rc, n = ctx.sortlimit(rel, by, asc, limit, out, cap)
    assert rc == pyg.PYG_OK
    return from_device(torch, out, n, A.dtype)


@pytest.mark.parametrize("asc", [1, 0])
@pytest.mark.parametrize("limit", [1, 10, 1000, 8192])
@pytest.mark.parametrize("dist", ["wide", "ties", "skew"])
def test_sortlimit_int64_vs_oracle(ctx, torch_cuda, asc, limit, dist):
    rng = np.random.default_rng(limit + asc + len(dist))
    n = 1 << 20
    if dist == "wide":
        k = rng.integers(np.iinfo(np.int64).min, np.iinfo(np.int64).max, n)
    elif dist == "ties":
        k = rng.integers(-50, 50, n)  # many ties: input order decides
    else:
        k = (rng.zipf(1.3, n) % 1000).astype(np.int64) * (1 << 40)
    A = struct([k, np.arange(n, dtype=np.int64)], [I64, I64])
    got = run(ctx, torch_cuda, A, [I64, I64], [0], asc, limit)
    assert rows(got) == rows(O.sortlimit(A, [I64, I64], [0], asc, limit))


@pytest.mark.parametrize("asc", [1, 0])
def test_sortlimit_composite_and_int32(ctx, torch_cuda, asc):
    rng = np.random.default_rng(4 + asc)
    n = 300000
    A = struct([rng.integers(-4, 4, n), rng.integers(-(1 << 31), 1 << 31, n), np.arange(n)], [I32, I32, I64])
    for by in ([0, 1], [1], [0]):
        for limit in (5, 4096):
            got = run(ctx, torch_cuda, A, [I32, I32, I64], by, asc, limit)
            assert rows(got) == rows(O.sortlimit(A, [I32, I32, I64], by, asc, limit))
        # A limit above the input size: every tuple, in order.
        small = A[:3000]
        got = run(ctx, torch_cuda, small, [I32, I32, I64], by, asc, 3010)
        assert rows(got) == rows(O.sortlimit(small, [I32, I32, I64], by, asc, 3010))


def test_sortlimit_edges(ctx, torch_cuda):
    A = struct([np.array([5, 3, 5, 1], dtype=np.int64), np.arange(4, dtype=np.int64)], [I64, I64])
    assert run(ctx, torch_cuda, A, [I64, I64], [0], 1, 0).shape[0] == 0
    assert run(ctx, torch_cuda, A[:0], [I64, I64], [0], 1, 5).shape[0] == 0
    # Host input, limit above n.
    got = run(ctx, torch_cuda, A, [I64, I64], [0], 0, 10, on_device=False)
    assert rows(got) == [(5, 0), (5, 2), (3, 1), (1, 3)]
    out = alloc(torch_cuda, 16)
    rc, n = ctx.sortlimit(dev_rel(torch_cuda, A, [I64, I64]), [0], 1, 3, out, 1)
    assert rc == pyg.PYG_ERR_CAPACITY and n == 3


def test_sortlimit_golden(ctx, torch_cuda, golden):
    """The reference engine's own sortlimit output (tests/golden)."""
    g = golden("sortlimit")
    for asc in (1, 0):
        for limit in (1, 100, 5000):
            got = run(ctx, torch_cuda, g["A"], [I64, I64], [0], asc, limit)
            assert got.tolist() == g[f"a_{asc}_{limit}"].tolist()
            got = run(ctx, torch_cuda, g["B"], [I32, I32, I64], [0, 1], asc, limit)
            assert got.tolist() == g[f"b_{asc}_{limit}"].tolist()
