"""Group-by aggregation on the GPU vs the oracle and the reference's golden
outputs (bit-exact sums and counts, output ordered by key)."""
import numpy as np
import pytest

import oracle as O
import pyg
from util import I32, I64, alloc, dev_rel, from_device, host_rel, rows, struct

pytestmark = pytest.mark.gpu


def run_groupby(ctx, torch, A, types, keys, flags, sum_col, expected, on_device=True, sort=True):
    rel = dev_rel(torch, A, types) if on_device else host_rel(A, types)
    dt = O.groupby_dtype(types, keys, flags, sum_col)
    cap = max(1, A.shape[0])
    out = alloc(torch, cap * dt.itemsize)
    rc, g = ctx.groupby(rel, keys, flags, sum_col, sort, expected, out, cap)
    assert rc == pyg.PYG_OK
    return from_device(torch, out, g, dt)


@pytest.mark.parametrize("expected", [1024, 0, 16])
def test_groupby_int64_golden(ctx, torch_cuda, golden, expected):
    g = golden("groupby_int64")
    out = run_groupby(ctx, torch_cuda, g["A"], [I64, I64], [0], 3, 1, expected)
    assert [(r[0], r[1]) for r in rows(out)] == rows(g["sum_rows"])
    assert [(r[0], r[2]) for r in rows(out)] == rows(g["count_rows"])


@pytest.mark.parametrize("on_device", [True, False])
def test_groupby_composite_golden(ctx, torch_cuda, golden, on_device):
    g = golden("groupby_composite")
    out = run_groupby(ctx, torch_cuda, g["A"], [I32, I32, I32], [0, 1], 3, 2, 256, on_device)
    assert [(r[0], r[1], r[3]) for r in rows(out)] == rows(g["count_rows"])
    assert [(r[0], r[1], r[2]) for r in rows(out)] == rows(g["sum_rows"])


@pytest.mark.parametrize("G,expected", [(16, 16), (1 << 10, 1 << 10), (1 << 16, 1 << 16), (1 << 16, 0)])
@pytest.mark.parametrize("zipf", [False, True])
def test_groupby_random_vs_oracle(ctx, torch_cuda, G, expected, zipf):
    rng = np.random.default_rng(G + zipf)
    n = 1 << 20
    if zipf:
        gid = (rng.zipf(1.1, n) - 1) % G
    else:
        gid = rng.integers(0, G, n)
    perm = rng.permutation(G).astype(np.int64) * 1000003 - (1 << 40)
    A = struct([perm[gid], rng.integers(0, 1 << 20, n)], [I64, I64])
    out = run_groupby(ctx, torch_cuda, A, [I64, I64], [0], 3, 1, expected)
    ref = O.groupby(A, [I64, I64], [0], 3, 1, buckets=G)
    assert rows(out) == rows(ref)


@pytest.mark.parametrize("G,expected,n", [(1 << 21, 1 << 21, (1 << 25) + 777),  # two passes, sampled layout
                                          (1 << 18, 1 << 12, 1 << 22),          # estimate 64x too small
                                          (3000, 3000, 1 << 22)])                # one shared table per CTA
def test_groupby_shared_memory_paths(ctx, torch_cuda, G, expected, n):
    """16-byte (int64, int64) tuples with a group estimate are aggregated in
    shared memory, partitioned by hash when the estimate is large; keys that
    do not fit a shared table go to the HBM table, so a wrong estimate only
    costs time."""
    rng = np.random.default_rng(G + n)
    gid = rng.integers(0, G, n)
    perm = rng.permutation(G).astype(np.int64) * 7919 - (1 << 50)
    A = struct([perm[gid], rng.integers(-(1 << 62), 1 << 62, n)], [I64, I64])
    out = run_groupby(ctx, torch_cuda, A, [I64, I64], [0], 3, 1, expected)
    assert rows(out) == rows(O.groupby(A, [I64, I64], [0], 3, 1, buckets=G))


def zipf_ranks(rng, n, G, theta):
    """Ranks in [0, G) with P(r) ~ (r + 1)^-theta (CDF inversion in fp64)."""
    w = np.arange(1, G + 1, dtype=np.float64) ** (-theta)
    cdf = np.cumsum(w)
    cdf /= cdf[-1]
    return np.minimum(np.searchsorted(cdf, rng.random(n), side="right"), G - 1)


@pytest.mark.parametrize("G", [1 << 10, 1 << 16, 1 << 20])
@pytest.mark.parametrize("zipf", [False, True])
def test_groupby_composite_config3_cardinalities(ctx, torch_cuda, G, zipf):
    """Group-by over a composite (int32, int32) key, the second key form of
    the 2^28-tuple group-by workload (operators/genericaggregate.cpp:247-289
    with the `bytes` hasher over both columns): 2^22 tuples (int32 hi, int32
    lo, int64 value) where the group id g (uniform, or Zipf(1.0) ranks
    through a seeded permutation) is split as hi = g >> ceil(log2 G / 2),
    lo = g & mask; values uniform in [0, 2^20).  Sum and count per group,
    ordered by (hi, lo), identical to the oracle."""
    rng = np.random.default_rng(G * 3 + zipf)
    n = 1 << 22
    rank = zipf_ranks(rng, n, G, 1.0) if zipf else rng.integers(0, G, n)
    g = rng.permutation(G).astype(np.int64)[rank]
    half = ((G - 1).bit_length() + 1) // 2
    hi, lo = (g >> half).astype(np.int32), (g & ((1 << half) - 1)).astype(np.int32)
    # Spread the halves over the signed int32 range so the lexicographic
    # order of (hi, lo) differs from the order of g.
    hi = (hi.astype(np.int64) * 2654435761 % (1 << 32) - (1 << 31)).astype(np.int32)
    lo = (lo.astype(np.int64) * 40503 - (1 << 20)).astype(np.int32)
    A = struct([hi, lo, rng.integers(0, 1 << 20, n)], [I32, I32, I64])
    types = [I32, I32, I64]
    ref = O.groupby(A, types, [0, 1], 3, 2, buckets=G, bytes_hash=True)
    for expected in (G, 0):
        out = run_groupby(ctx, torch_cuda, A, types, [0, 1], 3, 2, expected)
        assert out.shape[0] == ref.shape[0]
        assert rows(out) == rows(ref)


def test_groupby_uniform_warps_and_sentinel(ctx, torch_cuda):
    """Runs of one key (whole warps fold with one reduction) mixed with the
    INT64_MIN group and count-only output."""
    mn = np.iinfo(np.int64).min
    rng = np.random.default_rng(5)
    n = (1 << 20) + 100
    k = np.repeat(rng.integers(0, 50, n // 64 + 1), 64)[:n].astype(np.int64)
    k[rng.random(n) < 0.01] = mn
    A = struct([k, rng.integers(0, 1 << 40, n)], [I64, I64])
    for flags in (3, 2, 1):
        out = run_groupby(ctx, torch_cuda, A, [I64, I64], [0], flags, 1, 64)
        assert rows(out) == rows(O.groupby(A, [I64, I64], [0], flags, 1))


def test_groupby_edge_cases(ctx, torch_cuda):
    mn = np.iinfo(np.int64).min
    A = struct([np.array([mn, 3, mn, 3, 9, -1], dtype=np.int64), np.array([1, 2, 3, 4, 5, 6], dtype=np.int64)],
               [I64, I64])
    for exp in (0, 4):
        out = run_groupby(ctx, torch_cuda, A, [I64, I64], [0], 3, 1, exp)
        assert rows(out) == rows(O.groupby(A, [I64, I64], [0], 3, 1))
    # Unordered output is the same multiset.
    out = run_groupby(ctx, torch_cuda, A, [I64, I64], [0], 3, 1, 0, sort=False)
    assert sorted(rows(out)) == rows(O.groupby(A, [I64, I64], [0], 3, 1))
    # No GROUP BY, and empty input.
    out = run_groupby(ctx, torch_cuda, A, [I64, I64], [], 3, 1, 0)
    assert rows(out) == [(int(A["c1"].sum()), 6)]
    E = A[:0]
    assert run_groupby(ctx, torch_cuda, E, [I64, I64], [0], 3, 1, 0).shape[0] == 0
    assert run_groupby(ctx, torch_cuda, E, [I64, I64], [], 3, 1, 0).shape[0] == 0
    # Count only, sum only.
    assert rows(run_groupby(ctx, torch_cuda, A, [I64, I64], [0], 2, 1, 0)) == rows(O.groupby(A, [I64, I64], [0], 2, 1))
    assert rows(run_groupby(ctx, torch_cuda, A, [I64, I64], [0], 1, 1, 0)) == rows(O.groupby(A, [I64, I64], [0], 1, 1))


def test_groupby_capacity_error(ctx, torch_cuda):
    A = struct([np.arange(100, dtype=np.int64)] * 2, [I64, I64])
    out = alloc(torch_cuda, 10 * 24)
    rc, g = ctx.groupby(dev_rel(torch_cuda, A, [I64, I64]), [0], 3, 1, True, 100, out, 10)
    assert rc == pyg.PYG_ERR_CAPACITY and g == 100


def test_groupby_full_size_property(ctx, torch_cuda):
    """2^26 tuples over 2^20 groups: counts sum to n, sums sum to the total."""
    torch = torch_cuda
    n, G = 1 << 26, 1 << 20
    S = torch.empty(n * 2, dtype=torch.int64, device="cuda")
    ctx.gen_fk(S, n, G, 1.0, 3, 1 << 20, 4)
    rel = pyg.Rel(S, n, [I64, I64])
    out = torch.empty(G * 3, dtype=torch.int64, device="cuda")
    rc, g = ctx.groupby(rel, [0], 3, 1, True, G, out, G)
    assert rc == pyg.PYG_OK and 0 < g <= G
    o = out[: 3 * g].view(g, 3)
    assert int(o[:, 2].sum().item()) == n
    assert int(o[:, 1].sum().item()) == int(S.view(n, 2)[:, 1].sum().item())
    assert bool((o[1:, 0] > o[:-1, 0]).all().item())
    assert int(torch.unique(S.view(n, 2)[:, 0]).numel()) == g


@pytest.mark.parametrize("case", ["zipf1.0", "zipf1.5", "alternating"])
def test_groupby_hot_keys_in_warp_registers(ctx, torch_cuda, case):
    """Skewed 16-byte tuples through the partitioned shared-memory fold,
    where each warp keeps its hot key's combined sum and count in registers
    and folds them when another large group's key takes its place: Zipf ids
    (theta 1.0 and 1.5), and runs of 64 tuples alternating between two hot
    keys with a third spread among them, so the hot key changes every few
    batches.  Values near 2^62 make the int64 sums wrap."""
    rng = np.random.default_rng(len(case))
    G, n = 1 << 16, (1 << 22) + 333
    if case == "alternating":
        run = (np.arange(n) // 64) % 3
        gid = np.where(run == 0, 5, np.where(run == 1, 77, rng.integers(0, G, n)))
        gid[rng.random(n) < 0.2] = 1234
    else:
        gid = zipf_ranks(rng, n, G, float(case[4:]))
    perm = rng.permutation(G).astype(np.int64) * 104729 + (1 << 45)
    A = struct([perm[gid], rng.integers((1 << 62) - (1 << 40), 1 << 62, n)], [I64, I64])
    out = run_groupby(ctx, torch_cuda, A, [I64, I64], [0], 3, 1, G)
    assert rows(out) == rows(O.groupby(A, [I64, I64], [0], 3, 1, buckets=G))
