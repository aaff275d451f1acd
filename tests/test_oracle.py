"""Pins the C oracle: against the reference engine's own outputs (golden
fixtures made by tests/golden/make_golden.py from oracle/_ref/executequery)
and against the known answers the reference's unit tests assert.  CPU only.
"""
import numpy as np
import pytest

import oracle as O

I32, I64 = 1, 2


def canon(a):
    return O.canonical(a)


def as_rows(a):
    return [tuple(int(x) for x in r) for r in a.tolist()]


@pytest.mark.parametrize("name", ["join_pkfk", "join_dups", "join_composite"])
def test_oracle_join_matches_reference(golden, name):
    g = golden(name)
    rt, st = list(g["rtypes"]), list(g["stypes"])
    proj = [tuple(p) for p in g["proj"]]
    out = O.hashjoin_materialize(g["R"], rt, list(g["rk"]), g["S"], st, list(g["sk"]), proj,
                                 buckets=int(g["buckets"]), bytes_hash=bool(g["bytes_hash"]))
    assert as_rows(canon(out)) == as_rows(canon(g["out"]))
    cnt, sums = O.hashjoin_agg(g["R"], rt, list(g["rk"]), g["S"], st, list(g["sk"]), proj, int(g["buckets"]),
                               bool(g["bytes_hash"]))
    assert cnt == g["out"].shape[0]
    for i in range(len(proj)):
        col = g["out"][f"c{i}"].astype(np.int64)
        assert sums[i] == int(col.sum(dtype=np.int64))


def test_oracle_join_sum_plan(golden):
    g = golden("join_sum")
    cnt, sums = O.hashjoin_agg(g["R"], [I64, I64], [0], g["S"], [I64, I64], [0], [(0, 1), (1, 1)])
    assert cnt == int(g["count"])
    assert sums[1] == int(g["sum"])


def test_oracle_groupby_int64(golden):
    g = golden("groupby_int64")
    out = O.groupby(g["A"], [I64, I64], [0], 3, 1)
    assert as_rows(out[["c0", "c1"]]) == as_rows(g["sum_rows"])
    assert [(r[0], r[2]) for r in as_rows(out)] == as_rows(g["count_rows"])


def test_oracle_groupby_composite_bytes_hash_and_int32_wrap(golden):
    g = golden("groupby_composite")
    out = O.groupby(g["A"], [I32, I32, I32], [0, 1], 3, 2, buckets=256, bytes_hash=True)
    assert [(r[0], r[1], r[3]) for r in as_rows(out)] == as_rows(g["count_rows"])
    # int32 sums wrap at 32 bits exactly like `CtInt +=` in the reference.
    assert [(r[0], r[1], r[2]) for r in as_rows(out)] == as_rows(g["sum_rows"])


def test_oracle_partition_matches_reference(golden):
    g = golden("partition_exactrange")
    fan = int(g["fanout"])
    out, offs = O.partition(g["A"], [I64, I64], 0, 0, fan, int(g["mn"]), int(g["mx"]))
    ref = g["out"]
    for b in range(fan):
        mine = canon(out[offs[b]:offs[b + 1]])
        theirs = ref[ref["c0"] == b]
        theirs2 = np.empty(theirs.shape[0], dtype=out.dtype)
        theirs2["c0"], theirs2["c1"] = theirs["c1"], theirs["c2"]
        assert as_rows(mine) == as_rows(canon(theirs2))


def test_oracle_mpsm_matches_reference(golden):
    g = golden("mpsm_pkfk")
    proj = [tuple(p) for p in g["proj"]]
    out = O.mpsm_join(g["R"], [I64, I64], 0, g["S"], [I64, I64], 0, proj, materialize=True)
    assert as_rows(canon(out)) == as_rows(canon(g["out"]))


# ---- known answers asserted by the reference's unit tests ----------------

def test_known_answer_pk_pk_join():
    """unit_tests/queryhashjoin.cpp:85-92, 211-218: a PK-PK join of 20 keys
    where every key appears exactly once on the output."""
    k = np.arange(1, 21, dtype=np.int64)
    R = O.as_struct(np.stack([k, k], 1), [I64, I64])
    S = O.as_struct(np.stack([k, k * 10 + 1], 1), [I64, I64])
    out = O.hashjoin_materialize(R, [I64, I64], [0], S, [I64, I64], [0], [(0, 1), (1, 1)], buckets=16)
    assert sorted(out["c0"].tolist()) == list(range(1, 21))
    assert all(b == a * 10 + 1 for a, b in zip(out["c0"], out["c1"]))


def test_known_answer_aggsum():
    """unit_tests/queryaggsum.cpp:84-90: group v holds 1..v, sum v(v+1)/2."""
    rows = [(v, j) for v in range(1, 21) for j in range(1, v + 1)]
    A = O.as_struct(np.array(rows, dtype=np.int64), [I64, I64])
    out = O.groupby(A, [I64, I64], [0], 1, 1, buckets=4)
    assert [(r[0], r[1]) for r in as_rows(out)] == [(v, v * (v + 1) // 2) for v in range(1, 21)]


def test_known_answer_mpsm_pkfk():
    """unit_tests/querympsmpkfkjoin.cpp: key i has (i & 3) + 1 matches."""
    n = 1000
    k = np.arange(n, dtype=np.int64)
    R = O.as_struct(np.stack([k, k], 1), [I64, I64])
    fk = np.concatenate([np.full((i & 3) + 1, i, dtype=np.int64) for i in range(n)])
    S = O.as_struct(np.stack([fk, fk], 1), [I64, I64])
    out = O.mpsm_join(R, [I64, I64], 0, S, [I64, I64], 0, [(0, 0)], materialize=True)
    counts = np.bincount(out["c0"], minlength=n)
    assert all(counts[i] == (i & 3) + 1 for i in range(n))


def test_known_answer_exactrange_boundaries():
    """unit_tests/testhash.cpp:120-144 (testExactRange): 80 buckets; max
    hashes below 80; minimumforbucket(j) - 1 -> j - 1 and
    minimumforbucket(j) -> j."""
    rng = np.random.default_rng(7)
    for _ in range(200):
        mx = int(rng.integers(2, 1 << 31)) & ~1
        mn = int(rng.integers(0, mx))
        assert O.exactrange_bucket(mx, mn, mx, 80) <= 79
        for j in range(1, 80):
            m = O.exactrange_min_for_bucket(j, mn, mx, 80)
            assert O.exactrange_bucket(m - 1, mn, mx, 80) == j - 1
            assert O.exactrange_bucket(m, mn, mx, 80) == j


def test_oracle_sort_is_stable_and_ordered():
    rng = np.random.default_rng(3)
    A = O.as_struct(np.stack([rng.integers(-50, 50, 5000), np.arange(5000)], 1).astype(np.int64), [I64, I64])
    out = O.sort(A, [I64, I64], 0)
    assert np.all(np.diff(out["c0"]) >= 0)
    ref = A[np.argsort(A["c0"], kind="stable")]
    assert np.array_equal(out, ref)


def test_oracle_sortlimit_matches_reference(golden):
    """SortLimit top-k (operators/sortlimit.cpp), as the reference engine
    printed it for int64 and (int32, int32) keys, both directions, with
    ties decided by input order."""
    g = golden("sortlimit")
    for asc in (1, 0):
        for limit in (1, 100, 5000):
            got = O.sortlimit(g["A"], [2, 2], [0], asc, limit)
            assert got.tolist() == g[f"a_{asc}_{limit}"].tolist()
            got = O.sortlimit(g["B"], [1, 1, 2], [0, 1], asc, limit)
            assert got.tolist() == g[f"b_{asc}_{limit}"].tolist()
