"""Hash join on the GPU vs the oracle and the reference's golden outputs.

Integer results must be bit-identical: the match count, every wrapped int64
or int32 sum, and the multiset of materialised tuples."""
import numpy as np
import pytest

import oracle as O
import pyg
from util import I32, I64, alloc, canon_rows, dev_rel, from_device, host_rel, struct

pytestmark = pytest.mark.gpu


def run_join(ctx, torch, R, rt, rk, S, st, sk, proj, on_device=True, lf=0.5):
    Rr = dev_rel(torch, R, rt) if on_device else host_rel(R, rt)
    Sr = dev_rel(torch, S, st) if on_device else host_rel(S, st)
    bcols = sorted({c for s, c in proj if s == 0})
    ht = ctx.hashjoin_build(Rr, rk, bcols, pyg.HT_MATERIALIZE, lf)
    dt = O.proj_dtype(rt, st, proj)
    rc, n = ctx.hashjoin_probe_materialize(ht, Sr, sk, proj, None, 0)
    assert rc in (pyg.PYG_OK, pyg.PYG_ERR_CAPACITY)
    out = alloc(torch, n * dt.itemsize)
    rc, n2 = ctx.hashjoin_probe_materialize(ht, Sr, sk, proj, out, n)
    assert rc == pyg.PYG_OK and n2 == n
    mat = from_device(torch, out, n, dt)
    ht.free()
    hta = ctx.hashjoin_build(Rr, rk, bcols, pyg.HT_AGGREGATE, lf)
    cnt, sums = ctx.hashjoin_probe_agg(hta, Sr, sk, proj)
    hta.free()
    return mat, cnt, sums


@pytest.mark.parametrize("name", ["join_pkfk", "join_dups", "join_composite"])
@pytest.mark.parametrize("on_device", [True, False])
def test_join_golden(ctx, torch_cuda, golden, name, on_device):
    g = golden(name)
    rt, st = [int(x) for x in g["rtypes"]], [int(x) for x in g["stypes"]]
    proj = [tuple(int(v) for v in p) for p in g["proj"]]
    mat, cnt, sums = run_join(ctx, torch_cuda, g["R"], rt, [int(x) for x in g["rk"]], g["S"], st,
                              [int(x) for x in g["sk"]], proj, on_device)
    assert canon_rows(mat) == canon_rows(g["out"])
    assert cnt == g["out"].shape[0]
    for i in range(len(proj)):
        assert sums[i] == int(g["out"][f"c{i}"].astype(np.int64).sum(dtype=np.int64))


def test_join_sum_plan_golden(ctx, torch_cuda, golden):
    g = golden("join_sum")
    _, cnt, sums = run_join(ctx, torch_cuda, g["R"], [I64, I64], [0], g["S"], [I64, I64], [0], [(0, 1), (1, 1)])
    assert cnt == int(g["count"]) and sums[1] == int(g["sum"])


@pytest.mark.parametrize("lf", [0.25, 0.5, 0.9])
def test_join_random_vs_oracle(ctx, torch_cuda, lf):
    rng = np.random.default_rng(11)
    n, m = 1 << 16, 1 << 19
    k = rng.permutation(n).astype(np.int64) * 3 - 70000
    R = struct([k, rng.integers(-(1 << 62), 1 << 62, n)], [I64, I64])
    S = struct([rng.choice(k, m) + rng.integers(0, 2, m), rng.integers(-(1 << 62), 1 << 62, m)], [I64, I64])
    proj = [(0, 1), (1, 1)]
    mat, cnt, sums = run_join(ctx, torch_cuda, R, [I64, I64], [0], S, [I64, I64], [0], proj, lf=lf)
    c2, s2 = O.hashjoin_agg(R, [I64, I64], [0], S, [I64, I64], [0], proj)
    assert (cnt, sums) == (c2, s2)
    assert canon_rows(mat) == canon_rows(O.hashjoin_materialize(R, [I64, I64], [0], S, [I64, I64], [0], proj))


def test_join_edge_cases(ctx, torch_cuda):
    proj = [(0, 1), (1, 1)]
    mn = np.iinfo(np.int64).min
    # Keys equal to the table's empty marker, duplicates, and misses.
    R = struct([np.array([mn, mn, 5, 5, 5, 7], dtype=np.int64), np.arange(6, dtype=np.int64) + 100], [I64, I64])
    S = struct([np.array([mn, 5, 6, 7, mn, 5], dtype=np.int64), np.arange(6, dtype=np.int64)], [I64, I64])
    mat, cnt, sums = run_join(ctx, torch_cuda, R, [I64, I64], [0], S, [I64, I64], [0], proj)
    assert (cnt, sums) == O.hashjoin_agg(R, [I64, I64], [0], S, [I64, I64], [0], proj)
    assert canon_rows(mat) == canon_rows(O.hashjoin_materialize(R, [I64, I64], [0], S, [I64, I64], [0], proj))
    # Empty build, empty probe.
    E = struct([np.zeros(0, dtype=np.int64)] * 2, [I64, I64])
    for a, b in ((E, S), (R, E)):
        mat, cnt, sums = run_join(ctx, torch_cuda, a, [I64, I64], [0], b, [I64, I64], [0], proj)
        assert cnt == 0 and sums == [0, 0] and mat.shape[0] == 0
    # All build tuples share one key.
    R = struct([np.full(2000, 42, dtype=np.int64), np.arange(2000, dtype=np.int64)], [I64, I64])
    S = struct([np.array([42, 41, 42], dtype=np.int64), np.array([1, 2, 3], dtype=np.int64)], [I64, I64])
    mat, cnt, sums = run_join(ctx, torch_cuda, R, [I64, I64], [0], S, [I64, I64], [0], proj)
    assert (cnt, sums) == O.hashjoin_agg(R, [I64, I64], [0], S, [I64, I64], [0], proj)
    assert cnt == 4000


def test_join_int32_key_and_int32_sum_wrap(ctx, torch_cuda):
    rng = np.random.default_rng(5)
    R = struct([rng.integers(-1000, 1000, 5000).astype(np.int32), rng.integers(1 << 29, 1 << 31, 5000).astype(np.int32)],
               [I32, I32])
    S = struct([rng.integers(-1000, 1000, 20000).astype(np.int32), rng.integers(0, 1 << 31, 20000).astype(np.int32)],
               [I32, I32])
    proj = [(0, 1), (1, 1), (1, 0)]
    mat, cnt, sums = run_join(ctx, torch_cuda, R, [I32, I32], [0], S, [I32, I32], [0], proj)
    assert (cnt, sums) == O.hashjoin_agg(R, [I32, I32], [0], S, [I32, I32], [0], proj)
    assert canon_rows(mat) == canon_rows(O.hashjoin_materialize(R, [I32, I32], [0], S, [I32, I32], [0], proj))


def test_materialize_capacity_error(ctx, torch_cuda):
    R = struct([np.arange(10, dtype=np.int64)] * 2, [I64, I64])
    S = struct([np.arange(10, dtype=np.int64)] * 2, [I64, I64])
    ht = ctx.hashjoin_build(dev_rel(torch_cuda, R, [I64, I64]), [0], [1], pyg.HT_MATERIALIZE, 0.5)
    out = alloc(torch_cuda, 5 * 16)
    rc, n = ctx.hashjoin_probe_materialize(ht, dev_rel(torch_cuda, S, [I64, I64]), [0], [(0, 1), (1, 1)], out, 5)
    assert rc == pyg.PYG_ERR_CAPACITY and n == 10
    ht.free()


def test_full_size_pkfk_properties(ctx, torch_cuda):
    """Configuration-1 sizes (R = 2^20 PK tuples, S = 2^24 FK tuples)
    generated on the device; size-independent checks: every fk matches once,
    sum(B$1) = 7 * sum(fk), sum(P$1) = sum(val)."""
    torch = torch_cuda
    nR, nS = 1 << 20, 1 << 24
    R = torch.empty(nR * 2, dtype=torch.int64, device="cuda")
    S = torch.empty(nS * 2, dtype=torch.int64, device="cuda")
    ctx.gen_pk(R, nR, 7, 1)
    ctx.gen_fk(S, nS, nR, 0.0, 1, 1000, 2)
    Rr = pyg.Rel(R, nR, [I64, I64])
    Sr = pyg.Rel(S, nS, [I64, I64])
    ht = ctx.hashjoin_build(Rr, [0], [1], pyg.HT_AGGREGATE, 0.5)
    e, cap, dups = ht.stats()
    assert e == nR and dups == 0
    cnt, (sb, sp) = ctx.hashjoin_probe_agg(ht, Sr, [0], [(0, 1), (1, 1)])
    ht.free()
    Sv = S.view(nS, 2)
    keys = R.view(nR, 2)[:, 0]
    assert torch.equal(torch.sort(keys).values, torch.arange(1, nR + 1, device="cuda"))
    assert cnt == nS
    assert sb == int((Sv[:, 0] * 7).sum().item())
    assert sp == int(Sv[:, 1].sum().item())
