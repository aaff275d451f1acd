"""Partition, sort and lower-bound on the GPU vs the oracle and the
reference's golden partition output."""
import numpy as np
import pytest

import oracle as O
import pyg
from util import I32, I64, alloc, canon_rows, dev_rel, from_device, rows, struct

pytestmark = pytest.mark.gpu


def run_partition(ctx, torch, A, types, key, kind, fanout, **kw):
    out = alloc(torch, A.nbytes)
    offs = ctx.partition(dev_rel(torch, A, types), key, kind, fanout, out, **kw)
    return from_device(torch, out, A.shape[0], A.dtype), offs


def test_partition_exactrange_golden(ctx, torch_cuda, golden):
    g = golden("partition_exactrange")
    fan = int(g["fanout"])
    out, offs = run_partition(ctx, torch_cuda, g["A"], [I64, I64], 0, pyg.SPLIT_EXACTRANGE, fan,
                              range_min=int(g["mn"]), range_max=int(g["mx"]))
    ref = g["out"]
    for b in range(fan):
        theirs = ref[ref["c0"] == b]
        t2 = np.empty(theirs.shape[0], dtype=out.dtype)
        t2["c0"], t2["c1"] = theirs["c1"], theirs["c2"]
        assert canon_rows(out[offs[b]:offs[b + 1]]) == canon_rows(t2)


@pytest.mark.parametrize("fanout", [1, 8, 256, 1 << 12, 1 << 14])
def test_partition_radix_and_range_vs_oracle(ctx, torch_cuda, fanout):
    rng = np.random.default_rng(fanout)
    n = 300001
    A = struct([rng.integers(-(1 << 40), 1 << 40, n), np.arange(n, dtype=np.int64)], [I64, I64])
    out, offs = run_partition(ctx, torch_cuda, A, [I64, I64], 0, pyg.SPLIT_RADIX, fanout)
    ref, roffs = O.partition(A, [I64, I64], 0, 2, fanout)
    assert np.array_equal(offs, roffs)
    for b in range(0, fanout, max(1, fanout // 64)):
        assert canon_rows(out[offs[b]:offs[b + 1]]) == canon_rows(ref[roffs[b]:roffs[b + 1]])
    assert canon_rows(out) == canon_rows(A)
    mn, mx = int(A["c0"].min()), int(A["c0"].max())
    out, offs = run_partition(ctx, torch_cuda, A, [I64, I64], 0, pyg.SPLIT_EXACTRANGE, fanout, range_min=mn,
                              range_max=mx)
    ref, roffs = O.partition(A, [I64, I64], 0, 0, fanout, mn, mx)
    assert np.array_equal(offs, roffs)
    for b in range(0, fanout, max(1, fanout // 64)):
        assert canon_rows(out[offs[b]:offs[b + 1]]) == canon_rows(ref[roffs[b]:roffs[b + 1]])
    if fanout > 1:
        spl = np.sort(rng.choice(A["c0"], fanout - 1))
        out, offs = run_partition(ctx, torch_cuda, A, [I64, I64], 0, pyg.SPLIT_SPLITTERS, fanout, splitters=spl)
        ref, roffs = O.partition(A, [I64, I64], 0, 1, fanout, splitters=spl)
        assert np.array_equal(offs, roffs)
        for b in range(0, fanout, max(1, fanout // 64)):
            assert canon_rows(out[offs[b]:offs[b + 1]]) == canon_rows(ref[roffs[b]:roffs[b + 1]])


def test_partition_hash_invariants(ctx, torch_cuda):
    rng = np.random.default_rng(9)
    n = 100000
    A = struct([rng.integers(0, 5000, n), np.arange(n, dtype=np.int64)], [I64, I64])
    out, offs = run_partition(ctx, torch_cuda, A, [I64, I64], 0, pyg.SPLIT_HASH, 64)
    assert offs[0] == 0 and offs[-1] == n and np.all(np.diff(offs) >= 0)
    assert canon_rows(out) == canon_rows(A)
    where = {}
    for b in range(64):
        for k in np.unique(out["c0"][offs[b]:offs[b + 1]]):
            assert where.setdefault(int(k), b) == b


def test_partition_exactrange_out_of_range_is_an_error(ctx, torch_cuda):
    A = struct([np.array([1, 2, 300], dtype=np.int64)] * 2, [I64, I64])
    with pytest.raises(pyg.PygError):
        run_partition(ctx, torch_cuda, A, [I64, I64], 0, pyg.SPLIT_EXACTRANGE, 4, range_min=0, range_max=100)


@pytest.mark.parametrize("n", [0, 1, 7, 2049, 1 << 20])
def test_sort_int64_vs_oracle(ctx, torch_cuda, n):
    rng = np.random.default_rng(n)
    A = struct([rng.integers(-(1 << 62), 1 << 62, n), np.arange(n, dtype=np.int64)], [I64, I64])
    out = alloc(torch_cuda, A.nbytes)
    ctx.sort(dev_rel(torch_cuda, A, [I64, I64]), 0, out)
    assert rows(from_device(torch_cuda, out, n, A.dtype)) == rows(O.sort(A, [I64, I64], 0))
    # key in the second column, with heavy duplicates (stability matters)
    B = struct([np.arange(n, dtype=np.int64), rng.integers(-3, 3, n)], [I64, I64])
    ctx.sort(dev_rel(torch_cuda, B, [I64, I64]), 1, out)
    assert rows(from_device(torch_cuda, out, n, B.dtype)) == rows(O.sort(B, [I64, I64], 1))


def test_sort_generic_layout(ctx, torch_cuda):
    rng = np.random.default_rng(4)
    n = 50000
    A = struct([rng.integers(0, 100, n).astype(np.int32), rng.integers(-1000, 1000, n).astype(np.int32),
                np.arange(n, dtype=np.int64)], [I32, I32, I64])
    out = alloc(torch_cuda, A.nbytes)
    ctx.sort(dev_rel(torch_cuda, A, [I32, I32, I64]), 1, out)
    assert rows(from_device(torch_cuda, out, n, A.dtype)) == rows(O.sort(A, [I32, I32, I64], 1))


def test_lower_bound(ctx, torch_cuda):
    torch = torch_cuda
    rng = np.random.default_rng(2)
    n = 100000
    keys = np.sort(rng.integers(-1000, 1000, n))
    A = struct([keys, np.arange(n, dtype=np.int64)], [I64, I64])
    rel = dev_rel(torch, A, [I64, I64])
    q = rng.integers(-1100, 1100, 5000).astype(np.int64)
    qd = torch.from_numpy(q).cuda()
    out = torch.empty(5000, dtype=torch.int64, device="cuda")
    ctx.lower_bound(rel, 0, qd, 5000, out)
    ctx.sync()
    assert np.array_equal(out.cpu().numpy(), np.searchsorted(keys, q, side="left"))
