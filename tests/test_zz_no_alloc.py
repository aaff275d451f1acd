"""The allocation-free hash join + sum (pyg_hashjoin_agg_noalloc).

Some callers cannot call cudaMalloc where they join: an engine whose device
memory all belongs to another allocator (a framework's caching pool, a
query runtime's arena) that a library must not bypass, or a latency-critical
path where an allocation could block on the device.  This entry point keeps
its table in a fixed array inside the library.  Checked here, through the
C ABI, against the allocating entry point (pyg_hashjoin_agg) and the oracle
on two calls in a row, so the second call must not see the first call's
table.  Integer results must be identical.  Collected last so a failure
here never hides other tests.
"""
import numpy as np
import pytest

import oracle as O
import pyg
from util import I64, dev_rel, struct, to_device

pytestmark = pytest.mark.gpu
LIMIT = pyg.NOALLOC_MAX_BUILD


def relations(seed, n, m):
    rng = np.random.default_rng(seed)
    keys = rng.integers(-(1 << 40), 1 << 40, n)
    keys[: n // 50] = keys[n // 50: 2 * (n // 50)]  # some duplicate build keys
    keys[:3] = np.iinfo(np.int64).min                 # and the table's empty marker
    R = struct([keys, rng.integers(-(1 << 50), 1 << 50, n)], [I64, I64])
    fk = rng.choice(keys, m) + (rng.random(m) < 0.2)
    fk[::997] = np.iinfo(np.int64).min
    S = struct([fk, rng.integers(-(1 << 50), 1 << 50, m)], [I64, I64])
    return R, S


def test_noalloc_matches_allocating_join_and_oracle_twice(ctx, torch_cuda):
    torch = torch_cuda
    out = torch.zeros(3, dtype=torch.int64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    # The first build is exactly at the limit (table capacity = 2 x build).
    for seed, n, m in ((1, LIMIT, 1 << 21), (2, 777, 50000)):
        R, S = relations(seed, n, m)
        Rd, Sd = to_device(torch, R), to_device(torch, S)
        rc = pyg.lib().pyg_hashjoin_agg_noalloc(Rd.data_ptr(), n, Sd.data_ptr(), m, out.data_ptr(), stream)
        assert rc == pyg.PYG_OK, pyg.lib().pyg_last_error()
        torch.cuda.synchronize()
        got = [int(x) for x in out.cpu()]
        cnt, (sb, sp) = ctx.hashjoin_agg(dev_rel(torch, R, [I64, I64]), [0], dev_rel(torch, S, [I64, I64]), [0],
                                         [(0, 1), (1, 1)], pyg.JOIN_DIRECT)
        assert got == [cnt, sb, sp]
        ocnt, (ob, op) = O.hashjoin_agg(R, [I64, I64], [0], S, [I64, I64], [0], [(0, 1), (1, 1)], buckets=n)
        assert got == [ocnt, ob, op]


def test_noalloc_rejects_oversized_build(ctx, torch_cuda):
    torch = torch_cuda
    out = torch.zeros(3, dtype=torch.int64, device="cuda")
    big = torch.zeros(2 * (LIMIT + 1), dtype=torch.int64, device="cuda")
    rc = pyg.lib().pyg_hashjoin_agg_noalloc(big.data_ptr(), LIMIT + 1, big.data_ptr(), 1, out.data_ptr(), None)
    assert rc == pyg.PYG_ERR_ARG
    assert b"limit" in pyg.lib().pyg_last_error()
