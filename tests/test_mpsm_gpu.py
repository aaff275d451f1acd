"""MPSM sort-merge join on the GPU vs the oracle and the reference's golden
output; identical results under every splitter kind, and the learned /
sampled splitters' balance against the equal-width ranges on skewed keys."""
import numpy as np
import pytest

import oracle as O
import pyg
from util import I32, I64, alloc, canon_rows, dev_rel, from_device, host_rel, rows, struct

pytestmark = pytest.mark.gpu
KINDS = [pyg.MPSM_EXACTRANGE, pyg.MPSM_SAMPLED, pyg.MPSM_LEARNED]


def mpsm_mat(ctx, torch, R, rt, S, st, proj, kind=pyg.MPSM_SAMPLED, fan=64, on_device=True):
    Rr = dev_rel(torch, R, rt) if on_device else host_rel(R, rt)
    Sr = dev_rel(torch, S, st) if on_device else host_rel(S, st)
    o = ctx.mpsm_opts(kind, fan, 0.05, 64)
    rc, n = ctx.mpsm_join_materialize(Rr, 0, Sr, 0, proj, o, None, 0)
    assert rc in (pyg.PYG_OK, pyg.PYG_ERR_CAPACITY)
    dt = O.proj_dtype(rt, st, proj)
    out = alloc(torch, n * dt.itemsize)
    rc, n2 = ctx.mpsm_join_materialize(Rr, 0, Sr, 0, proj, o, out, n)
    assert rc == pyg.PYG_OK and n2 == n
    return from_device(torch, out, n, dt)


def test_mpsm_golden(ctx, torch_cuda, golden):
    g = golden("mpsm_pkfk")
    proj = [tuple(int(v) for v in p) for p in g["proj"]]
    for kind in KINDS:
        out = mpsm_mat(ctx, torch_cuda, g["R"], [I64, I64], g["S"], [I64, I64], proj, kind, 4)
        assert canon_rows(out) == canon_rows(g["out"])
        assert np.all(np.diff(out["c0"]) >= 0)  # ordered by key


@pytest.mark.parametrize("fan", [1, 7, 256, 4096])
@pytest.mark.parametrize("kind", KINDS)
def test_mpsm_agg_vs_oracle(ctx, torch_cuda, fan, kind):
    rng = np.random.default_rng(fan * 3 + kind)
    n, m = 40000, 300000
    R = struct([rng.integers(-50000, 50000, n), rng.integers(-(1 << 50), 1 << 50, n)], [I64, I64])
    S = struct([rng.integers(-60000, 60000, m), rng.integers(-(1 << 50), 1 << 50, m)], [I64, I64])
    proj = [(0, 1), (1, 1)]
    cnt, sums, st = ctx.mpsm_join_agg(dev_rel(torch_cuda, R, [I64, I64]), 0, dev_rel(torch_cuda, S, [I64, I64]), 0,
                                      proj, ctx.mpsm_opts(kind, fan, 0.02, 256))
    assert (cnt, sums) == O.mpsm_join(R, [I64, I64], 0, S, [I64, I64], 0, proj)
    assert st.max_partition_imbalance >= 1.0 or m == 0


@pytest.mark.parametrize("kind", KINDS)
def test_mpsm_agg_two_passes_and_chunked_ranges(ctx, torch_cuda, kind):
    """The aggregate sink on 16-byte device tuples: two range-partition
    passes (2^22 probe tuples), one build key repeated 20000 times (its range
    spans several sorted build chunks), INT64_MAX keys on both sides."""
    mx = np.iinfo(np.int64).max
    rng = np.random.default_rng(40 + kind)
    n, m = 1 << 18, 1 << 22
    rk = rng.integers(-(1 << 40), 1 << 40, n)
    rk[:20000] = 12345
    rk[20000:20003] = mx
    R = struct([rk, rng.integers(-(1 << 50), 1 << 50, n)], [I64, I64])
    sk = rk[rng.integers(0, n, m)]
    sk[::101] = rng.integers(-(1 << 40), 1 << 40, sk[::101].shape[0])  # mostly misses
    S = struct([sk, rng.integers(-(1 << 50), 1 << 50, m)], [I64, I64])
    proj = [(0, 1), (1, 1)]
    cnt, sums, _ = ctx.mpsm_join_agg(dev_rel(torch_cuda, R, [I64, I64]), 0, dev_rel(torch_cuda, S, [I64, I64]), 0,
                                     proj, ctx.mpsm_opts(kind, 4096, 0.01, 256))
    assert (cnt, sums) == O.mpsm_join(R, [I64, I64], 0, S, [I64, I64], 0, proj)


def test_mpsm_materialize_duplicates_int32_and_host(ctx, torch_cuda):
    rng = np.random.default_rng(6)
    R = struct([rng.integers(-30, 30, 3000).astype(np.int32), np.arange(3000, dtype=np.int64)], [I32, I64])
    S = struct([rng.integers(-40, 40, 5000).astype(np.int32), np.arange(5000, dtype=np.int64)], [I32, I64])
    proj = [(0, 0), (0, 1), (1, 1)]
    want = O.mpsm_join(R, [I32, I64], 0, S, [I32, I64], 0, proj, materialize=True)
    for kind in KINDS:
        for on_device in (True, False):
            out = mpsm_mat(ctx, torch_cuda, R, [I32, I64], S, [I32, I64], proj, kind, 16, on_device)
            assert canon_rows(out) == canon_rows(want)
            # deterministic order: key, probe row, build row
            order = np.lexsort((out["c1"], out["c2"], out["c0"]))
            assert np.array_equal(order, np.arange(out.shape[0]))


def test_mpsm_edge_cases(ctx, torch_cuda):
    proj = [(0, 1), (1, 1)]
    E = struct([np.zeros(0, dtype=np.int64)] * 2, [I64, I64])
    A = struct([np.array([5, 5, 7], dtype=np.int64), np.array([1, 2, 3], dtype=np.int64)], [I64, I64])
    for a, b in ((E, A), (A, E), (E, E)):
        cnt, sums, _ = ctx.mpsm_join_agg(dev_rel(torch_cuda, a, [I64, I64]), 0, dev_rel(torch_cuda, b, [I64, I64]), 0,
                                         proj, ctx.mpsm_opts(pyg.MPSM_SAMPLED, 8))
        assert cnt == 0 and sums == [0, 0]
    mn, mx = np.iinfo(np.int64).min, np.iinfo(np.int64).max
    B = struct([np.array([mn, mx, 0, mn, mx], dtype=np.int64), np.arange(5, dtype=np.int64)], [I64, I64])
    for kind in KINDS:
        cnt, sums, _ = ctx.mpsm_join_agg(dev_rel(torch_cuda, B, [I64, I64]), 0, dev_rel(torch_cuda, B, [I64, I64]), 0,
                                         proj, ctx.mpsm_opts(kind, 4, 1.0, 4))
        assert (cnt, sums) == O.mpsm_join(B, [I64, I64], 0, B, [I64, I64], 0, proj)


@pytest.mark.parametrize("theta", [1.0, 1.5])
def test_learned_and_sampled_splitters_balance_skew(ctx, torch_cuda, theta):
    """Zipf probe keys over a wide key domain: equal-width ranges put most
    tuples in a few partitions; learned and sampled splitters keep the
    largest partition near the heaviest single key, with identical joins."""
    rng = np.random.default_rng(7)
    N = 1 << 16
    keys = np.sort(rng.choice(1 << 40, N, replace=False)).astype(np.int64)
    w = np.arange(1, N + 1, dtype=np.float64) ** -theta
    c = np.cumsum(w)
    c /= c[-1]
    m = 1 << 21
    fk = keys[np.minimum(np.searchsorted(c, rng.random(m)), N - 1)]
    R = struct([keys, keys * 3], [I64, I64])
    S = struct([fk, rng.integers(0, 1 << 20, m)], [I64, I64])
    Rd, Sd = dev_rel(torch_cuda, R, [I64, I64]), dev_rel(torch_cuda, S, [I64, I64])
    proj = [(0, 1), (1, 1)]
    want = O.mpsm_join(R, [I64, I64], 0, S, [I64, I64], 0, proj)
    imb = {}
    for kind in KINDS:
        cnt, sums, st = ctx.mpsm_join_agg(Rd, 0, Sd, 0, proj, ctx.mpsm_opts(kind, 256, 0.01, 1024))
        assert (cnt, sums) == want
        imb[kind] = st.max_partition_imbalance
    heavy = np.bincount(np.searchsorted(keys, fk)).max() / (m / 256)
    assert imb[pyg.MPSM_LEARNED] <= max(1.5 * imb[pyg.MPSM_SAMPLED], heavy + 0.5), imb
    assert imb[pyg.MPSM_LEARNED] < imb[pyg.MPSM_EXACTRANGE], imb
