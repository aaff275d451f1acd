"""Page sort of 8-byte {int32 rid, int32 key} records (pyg_bitonic_sort,
the reference's TupleBuffer::bitonicsort): keys ascending (signed), every
record kept intact (unit_tests/testpagebitonicsort.cpp checks the same),
ties in rid order."""
import numpy as np
import pytest

import pyg

pytestmark = pytest.mark.gpu
REC = np.dtype([("rid", "<i4"), ("key", "<i4")])


def sort_on_gpu(ctx, torch, recs):
    raw = recs.view(np.uint8)
    t = torch.zeros(max(raw.shape[0], 16), dtype=torch.uint8, device="cuda")
    if raw.shape[0]:
        t[: raw.shape[0]].copy_(torch.from_numpy(raw.copy()))
    pyg.check(pyg.lib().pyg_bitonic_sort(ctx.h, t.data_ptr(), recs.shape[0]))
    return t[: raw.shape[0]].cpu().numpy().view(REC)


@pytest.mark.parametrize("n", [0, 1, 5, 4096, 4097, 1 << 13, (1 << 16) + 3, 1 << 20])
@pytest.mark.parametrize("dist", ["wide", "ties"])
def test_bitonic_page_sort(ctx, torch_cuda, n, dist):
    rng = np.random.default_rng(n + len(dist))
    recs = np.zeros(n, dtype=REC)
    recs["rid"] = rng.permutation(n).astype(np.int32) if n else []
    if dist == "wide":
        recs["key"] = rng.integers(np.iinfo(np.int32).min, np.iinfo(np.int32).max, n, dtype=np.int64)
    else:
        recs["key"] = rng.integers(-3, 3, n)
    got = sort_on_gpu(ctx, torch_cuda, recs)
    assert np.all(np.diff(got["key"].astype(np.int64)) >= 0)  # sorted by signed key
    # Every record intact, and ties in (unsigned) rid order.
    order = np.lexsort((recs["rid"].view(np.uint32), recs["key"]))
    assert np.array_equal(got, recs[order])


def test_bitonic_reference_shape(ctx, torch_cuda):
    """The reference's own test shape: 2^k records with constant payload
    bytes and lrand48-style non-negative 31-bit keys."""
    rng = np.random.default_rng(9)
    n = 1 << 15
    recs = np.zeros(n, dtype=REC)
    recs["rid"] = int.from_bytes(b"abcd", "little")
    recs["key"] = rng.integers(0, 1 << 31, n)
    got = sort_on_gpu(ctx, torch_cuda, recs)
    assert np.all(got["rid"] == recs["rid"][0])
    assert np.array_equal(np.sort(recs["key"]), got["key"])
