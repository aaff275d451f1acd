"""The one-shot direct join (pyg_hashjoin_agg, JOIN_DIRECT on 16-byte device
relations): a power-of-two table indexed by the top bits of the radix hash,
tiles of 256 x 4 tuples per block.  Checked against the oracle's hash join
(operators/join.cpp:548-800 restated in oracle/pyg_oracle.c) on the edges
of that layout: ragged tails of a tile, table sizes at a power-of-two
boundary for every load factor, strided and extreme keys, empty-marker keys
on both sides, and the plain configuration R 2^20 x S 2^24 scaled by 1/4.
Integer results must be identical."""
import numpy as np
import pytest

import oracle as O
import pyg
from util import I64, dev_rel, struct

pytestmark = pytest.mark.gpu
PROJ = [(0, 1), (1, 1)]
MN = np.iinfo(np.int64).min


def join(ctx, torch, R, S, lf=0.5, proj=PROJ):
    (cnt, sums), st = ctx.hashjoin_agg(dev_rel(torch, R, [I64, I64]), [0], dev_rel(torch, S, [I64, I64]), [0], proj,
                                       pyg.JOIN_DIRECT, 0, lf, stats=True)
    assert st.algorithm == pyg.JOIN_DIRECT
    return cnt, sums


def pkfk(rng, n, m, keys=None, miss=0.1):
    k = keys if keys is not None else rng.permutation(n).astype(np.int64) + 1
    R = struct([k, rng.integers(-(1 << 62), 1 << 62, n)], [I64, I64])
    fk = rng.choice(k, m) + (rng.random(m) < miss)
    S = struct([fk, rng.integers(-(1 << 62), 1 << 62, m)], [I64, I64])
    return R, S


@pytest.mark.parametrize("n,m", [(1, 1), (1, 1023), (7, 1024), (255, 1025), (1023, 4097), (1024, 3),
                                 (1025, 100000)])
def test_ragged_tiles(ctx, torch_cuda, n, m):
    rng = np.random.default_rng(n * 31 + m)
    R, S = pkfk(rng, n, m)
    assert join(ctx, torch_cuda, R, S) == O.hashjoin_agg(R, [I64, I64], [0], S, [I64, I64], [0], PROJ, buckets=n)


@pytest.mark.parametrize("lf", [0.25, 0.5, 0.75, 0.95])
@pytest.mark.parametrize("n", [32, 61, 64, 4096, 4097, 1 << 16])
def test_load_factors_at_power_of_two_sizes(ctx, torch_cuda, lf, n):
    """n / lf on either side of a power of two: the table is the next power
    of two with more slots than n / lf."""
    rng = np.random.default_rng(n)
    R, S = pkfk(rng, n, 8 * n + 5)
    want = O.hashjoin_agg(R, [I64, I64], [0], S, [I64, I64], [0], PROJ, buckets=n)
    assert join(ctx, torch_cuda, R, S, lf) == want


@pytest.mark.parametrize("stride", [1 << 16, 1 << 32, 987, 1 << 47, -(1 << 40)])
def test_strided_keys(ctx, torch_cuda, stride):
    rng = np.random.default_rng(abs(stride) % 1000)
    n = 1 << 15
    keys = (rng.permutation(n).astype(np.int64) * np.int64(stride)).astype(np.int64)
    keys = np.unique(keys)
    R, S = pkfk(rng, keys.shape[0], 1 << 18, keys=keys)
    want = O.hashjoin_agg(R, [I64, I64], [0], S, [I64, I64], [0], PROJ, buckets=keys.shape[0])
    assert join(ctx, torch_cuda, R, S) == want


def test_extreme_and_empty_marker_keys(ctx, torch_cuda):
    """INT64_MIN (the table's empty marker) on both sides goes through the
    side list; INT64_MAX, -1 and 0 are ordinary keys."""
    rng = np.random.default_rng(5)
    n = 5000
    keys = rng.permutation(n).astype(np.int64) * 3 + 10
    keys[:4] = [MN, np.iinfo(np.int64).max, -1, 0]
    keys[4:10] = MN  # seven empty-marker build tuples
    R, S = pkfk(rng, n, 200000, keys=keys)
    Sk = S["c0"]
    Sk[::101] = MN
    for proj in (PROJ, [(1, 1)], [(0, 1)], []):
        want = O.hashjoin_agg(R, [I64, I64], [0], S, [I64, I64], [0], proj, buckets=n)
        assert join(ctx, torch_cuda, R, S, proj=proj) == want


def test_plain_configuration_quarter_scale(ctx, torch_cuda):
    """R = a permutation of 1..2^18 with payload 7 key, S = 2^22 fks uniform
    over R's keys with values in 0..999 (the plain configuration at 1/4
    scale), projection P$1 and both columns; twice on one context."""
    rng = np.random.default_rng(20)
    n, m = 1 << 18, 1 << 22
    k = rng.permutation(n).astype(np.int64) + 1
    R = struct([k, 7 * k], [I64, I64])
    S = struct([rng.integers(1, n + 1, m), rng.integers(0, 1000, m)], [I64, I64])
    for proj in ([(1, 1)], PROJ):
        want = O.hashjoin_agg(R, [I64, I64], [0], S, [I64, I64], [0], proj, buckets=n)
        assert want[0] == m
        for _ in range(2):
            assert join(ctx, torch_cuda, R, S, proj=proj) == want
