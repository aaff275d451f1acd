"""Batched fragments (persistent kernel in a captured CUDA graph) vs the
oracle per fragment, against the plain sequential path, plus the autotuner
cache and the bounded device-side wait (a stall that nothing resolves must
end in PYG_ERR_TIMEOUT with the context still usable)."""
import numpy as np
import pytest

import oracle as O
import pyg
from util import I64, struct, to_device

pytestmark = pytest.mark.gpu
PROJ = [(0, 1), (1, 1)]


def make_fragments(torch, n, seed, max_log=14):
    rng = np.random.default_rng(seed)
    host, dev = [], []
    mn = np.iinfo(np.int64).min
    for i in range(n):
        nb = int(2 ** rng.uniform(4, max_log))
        npr = nb * int(rng.integers(4, 33))
        if i % 5 == 3:
            keys = rng.integers(0, nb // 2 + 1, nb)  # duplicate build keys
        else:
            keys = rng.permutation(nb).astype(np.int64) * 3 + i
        R = struct([keys, rng.integers(-(1 << 40), 1 << 40, nb)], [I64, I64])
        if i % 2:
            fk = keys[np.minimum(rng.zipf(1.2, npr) - 1, nb - 1)]
        else:
            fk = rng.choice(keys, npr) + (rng.random(npr) < 0.1)
        if i % 7 == 0:
            R["c0"][:2] = mn
            fk[:5] = mn
        S = struct([fk, rng.integers(0, 1 << 20, npr)], [I64, I64])
        host.append((R, S))
        dev.append((to_device(torch, R), nb, to_device(torch, S), npr))
    if n > 2:  # an empty probe side and an empty build side
        R, S = host[1]
        host[1] = (R, S[:0])
        dev[1] = (dev[1][0], dev[1][1], dev[1][2], 0)
        R, S = host[2]
        host[2] = (R[:0], S)
        dev[2] = (dev[2][0], 0, dev[2][2], dev[2][3])
    return host, dev


def expected(host):
    out = []
    for R, S in host:
        c, (a, b) = O.hashjoin_agg(R, [I64, I64], [0], S, [I64, I64], [0], PROJ, buckets=max(1024, R.shape[0]))
        out.append((c, (a + b + (1 << 63)) % (1 << 64) - (1 << 63)))
    return out


def test_batch_matches_oracle_and_replays(ctx, torch_cuda):
    host, dev = make_fragments(torch_cuda, 24, 1)
    frags = ctx.fragments(dev)
    want = expected(host)
    b = ctx.batch_create(frags)
    try:
        for _ in range(3):  # graph replays give the same answer
            rc, c, s, lat = ctx.batch_run(b, len(dev))
            assert rc == pyg.PYG_OK
            assert [(int(x), int(y)) for x, y in zip(c, s)] == want
            assert np.all(lat >= 0)
    finally:
        ctx.batch_free(b)
    c, s, lat = ctx.batch_run_plain(frags)
    assert [(int(x), int(y)) for x, y in zip(c, s)] == want
    assert np.all(np.diff(lat) >= 0)


def test_batch_config5_sizes_match_oracle(ctx, torch_cuda):
    """Fragments of the mixed-size batch workload's shape
    (drivers/executemultiplequery.cpp:134-180 runs each as its own
    hashjoin -> aggregate_sum plan): builds log-uniform in 2^12..2^22 with the
    extremes included, probes 4-32x the build, unique build keys (a seeded
    permutation), uniform or Zipf(1.0) foreign keys, int64 payloads.  Both the
    batched form and the plain path must equal the oracle per fragment."""
    torch = torch_cuda
    rng = np.random.default_rng(55)
    logs = [12.0, 22.0] + list(rng.uniform(12, 22, 6))
    host, dev = [], []
    for i, lg in enumerate(logs):
        nb = int(2 ** lg)
        mult = 4 if nb > (1 << 20) else int(rng.integers(4, 33))
        npr = nb * mult
        keys = rng.permutation(nb).astype(np.int64) * 5 + 1
        R = struct([keys, keys * 7], [I64, I64])
        if i % 2:
            w = np.arange(1, nb + 1, dtype=np.float64) ** -1.0
            cdf = np.cumsum(w)
            cdf /= cdf[-1]
            rank = np.minimum(np.searchsorted(cdf, rng.random(npr), side="right"), nb - 1)
        else:
            rank = rng.integers(0, nb, npr)
        S = struct([keys[rank], rng.integers(0, 1 << 20, npr)], [I64, I64])
        host.append((R, S))
        dev.append((to_device(torch, R), nb, to_device(torch, S), npr))
    frags = ctx.fragments(dev)
    want = expected(host)
    b = ctx.batch_create(frags)
    try:
        for _ in range(2):
            rc, c, s, lat = ctx.batch_run(b, len(dev))
            assert rc == pyg.PYG_OK
            assert [(int(x), int(y)) for x, y in zip(c, s)] == want
    finally:
        ctx.batch_free(b)
    c, s, _ = ctx.batch_run_plain(frags)
    assert [(int(x), int(y)) for x, y in zip(c, s)] == want


@pytest.mark.parametrize("tuning", [(256, 1, 0.5, 256), (1024, 2, 0.8, 65536), (512, 4, 0.7, 4096)])
def test_batch_tunings_give_identical_results(ctx, torch_cuda, tuning):
    host, dev = make_fragments(torch_cuda, 10, 2, max_log=12)
    frags = ctx.fragments(dev)
    t = pyg.pyg_tuning(*tuning, 0)
    b = ctx.batch_create(frags, t)
    try:
        rc, c, s, _ = ctx.batch_run(b, len(dev))
        assert rc == pyg.PYG_OK
        assert [(int(x), int(y)) for x, y in zip(c, s)] == expected(host)
    finally:
        ctx.batch_free(b)


def test_autotune_caches_choice(ctx, torch_cuda, tmp_path):
    host, dev = make_fragments(torch_cuda, 6, 3, max_log=10)
    frags = ctx.fragments(dev)
    path = str(tmp_path / "tune.txt")
    t1 = ctx.autotune(frags, path)
    assert t1.block_threads in (256, 512, 1024) and 0 < t1.load_factor <= 0.9
    with open(path) as f:
        assert len(f.read().split()) == 6
    t2 = ctx.autotune(frags, path)
    assert (t2.block_threads, t2.blocks_per_sm, t2.chunk_tuples) == (t1.block_threads, t1.blocks_per_sm,
                                                                      t1.chunk_tuples)
    b = ctx.batch_create(frags)  # picks the cached tuning
    try:
        rc, c, s, _ = ctx.batch_run(b, len(dev))
        assert rc == pyg.PYG_OK and [(int(x), int(y)) for x, y in zip(c, s)] == expected(host)
    finally:
        ctx.batch_free(b)


def test_bounded_wait_reports_timeout_and_context_survives(ctx, torch_cuda):
    host, dev = make_fragments(torch_cuda, 4, 4, max_log=10)
    frags = ctx.fragments(dev)
    b = ctx.batch_create(frags)
    try:
        pyg.check(pyg.lib().pyg_batch_inject_stall(ctx.h, b, 0))
        rc, _, _, _ = ctx.batch_run(b, len(dev))
        assert rc == pyg.PYG_ERR_TIMEOUT
    finally:
        ctx.batch_free(b)
    # the context still works
    b = ctx.batch_create(frags)
    try:
        rc, c, s, _ = ctx.batch_run(b, len(dev))
        assert rc == pyg.PYG_OK and [(int(x), int(y)) for x, y in zip(c, s)] == expected(host)
    finally:
        ctx.batch_free(b)


@pytest.mark.parametrize("large_build", [1 << 8, 1 << 11])
def test_large_fragments_run_as_their_own_joins(ctx, torch_cuda, large_build):
    """Fragments with at least large_build build tuples leave the queue and
    run after the graph as their own joins (duplicate keys, INT64_MIN keys
    and empty sides among them); every fragment's result still equals the
    oracle's, latencies are reported for all, and the stall hook refuses a
    fragment that is not queued."""
    host, dev = make_fragments(torch_cuda, 16, 8, max_log=13)
    frags = ctx.fragments(dev)
    b = ctx.batch_create(frags, pyg.pyg_tuning(512, 2, 0.7, 4096, large_build))
    try:
        for _ in range(2):
            rc, c, s, lat = ctx.batch_run(b, len(dev))
            assert rc == pyg.PYG_OK
            assert [(int(x), int(y)) for x, y in zip(c, s)] == expected(host)
            assert all(x >= 0 for x in lat)
        large = [i for i, d in enumerate(dev) if d[1] >= large_build]
        assert large
        assert pyg.lib().pyg_batch_inject_stall(ctx.h, b, large[0]) == pyg.PYG_ERR_ARG
    finally:
        ctx.batch_free(b)
