"""Generates the golden fixtures in tests/golden/*.npz by running the
reference engine (oracle/_ref/executequery, built from the reference's own
sources by `make -f oracle/ref.mk`) on seeded inputs.

Each fixture holds the input relations and the reference's output rows.
Run from the repository root:  python tests/golden/make_golden.py
The fixtures are committed; tests never need the reference at run time.
"""
import os
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle as O  # noqa: E402
import refrun  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))
I32, I64 = 1, 2
T = 4


def struct(cols, types):
    dt = O.dtype_of(types)
    a = np.empty(len(cols[0]), dtype=dt)
    for i, c in enumerate(cols):
        a[f"c{i}"] = c
    return a


def rows_array(rows, types):
    if not rows:
        return np.zeros(0, dtype=O.dtype_of(types))
    cols = list(zip(*rows))
    return struct([np.array(c, dtype=np.int64) for c in cols], types)


def save(name, **arrays):
    np.savez_compressed(os.path.join(OUT, name + ".npz"), **arrays)
    print("wrote", name, {k: v.shape for k, v in arrays.items()})


def join_case(name, R, rt, S, st, proj, buckets, rk=(0,), sk=(0,), hashfn="modulo"):
    with tempfile.TemporaryDirectory() as d:
        rf = refrun.write_rel(d, "R", R, T)
        sf = refrun.write_rel(d, "S", S, T)
        rows, _, _ = refrun.run(d, refrun.plan_join_rows(T, rf, rt, sf, st, proj, buckets, hashfn=hashfn,
                                                         bkeys=rk, pkeys=sk))
    otypes = [(st if s else rt)[c] for s, c in proj]
    save(name, R=R, S=S, rtypes=np.array(rt), stypes=np.array(st), rk=np.array(rk), sk=np.array(sk),
         proj=np.array(proj), buckets=np.array(buckets), bytes_hash=np.array(hashfn == "bytes"),
         out=rows_array(rows, otypes))


def main():
    if not refrun.available():
        sys.exit("oracle/_ref/executequery missing: run `make -f oracle/ref.mk` first")
    rng = np.random.default_rng(20240601)

    # PK-FK join, config-1 shape scaled down: R keys a permutation of 1..n,
    # payload key*7; S fk uniform over 1..1.25n (some misses), val 0..999.
    n, m = 1 << 12, 1 << 15
    k = rng.permutation(n).astype(np.int64) + 1
    R = struct([k, k * 7], [I64, I64])
    S = struct([rng.integers(1, n + n // 4 + 1, m), rng.integers(0, 1000, m)], [I64, I64])
    join_case("join_pkfk", R, [I64, I64], S, [I64, I64], [(0, 1), (1, 1)], 1 << 12)

    # Duplicate build keys (keys 1..300 repeated), mixed projection order.
    R = struct([rng.integers(1, 301, 1500), rng.integers(-(1 << 40), 1 << 40, 1500)], [I64, I64])
    S = struct([rng.integers(1, 350, 6000), rng.integers(-1000, 1000, 6000)], [I64, I64])
    join_case("join_dups", R, [I64, I64], S, [I64, I64], [(1, 1), (0, 1), (1, 0)], 256)

    # Composite (int32, int32) key with the FNV `bytes` hash; int64 payloads.
    a = rng.integers(-50, 50, 2000).astype(np.int32)
    b = rng.integers(-20, 20, 2000).astype(np.int32)
    R = struct([a, b, rng.integers(0, 1 << 50, 2000)], [I32, I32, I64])
    S = struct([rng.integers(-50, 50, 8000).astype(np.int32), rng.integers(-20, 20, 8000).astype(np.int32),
                rng.integers(0, 1 << 50, 8000)], [I32, I32, I64])
    join_case("join_composite", R, [I32, I32, I64], S, [I32, I32, I64], [(0, 2), (1, 2)], 1024,
              rk=(0, 1), sk=(0, 1), hashfn="bytes")

    # Config-1 plan shape: count via printer_tuplecount, sum of P$1.
    n, m = 1 << 12, 1 << 15
    k = rng.permutation(n).astype(np.int64) + 1
    R = struct([k, k * 7], [I64, I64])
    S = struct([rng.integers(1, n + 1, m), rng.integers(0, 1000, m)], [I64, I64])
    with tempfile.TemporaryDirectory() as d:
        rf = refrun.write_rel(d, "R", R, T)
        sf = refrun.write_rel(d, "S", S, T)
        rows, _, total = refrun.run(d, refrun.plan_join_sum(T, rf, [I64, I64], sf, [I64, I64], [(0, 1), (1, 1)], 1,
                                                            1 << 12))
    save("join_sum", R=R, S=S, sum=np.array(rows[0][0], dtype=np.int64), count=np.array(total, dtype=np.int64))

    # Group-by: int64 key (Zipf-like skew over 1000 groups), sum and count.
    m = 1 << 15
    g = (rng.zipf(1.3, m) % 1000).astype(np.int64) - 500
    A = struct([g, rng.integers(0, 1 << 20, m)], [I64, I64])
    with tempfile.TemporaryDirectory() as d:
        af = refrun.write_rel(d, "A", A, T)
        rs, _, _ = refrun.run(d, refrun.plan_groupby(T, af, [I64, I64], [0], "sum", 1, 1024))
        rc, _, _ = refrun.run(d, refrun.plan_groupby(T, af, [I64, I64], [0], "count", 1, 1024))
    save("groupby_int64", A=A, sum_rows=rows_array(sorted(rs), [I64, I64]), count_rows=rows_array(sorted(rc), [I64, I64]))

    # Group-by: composite (int32, int32) key with the `bytes` hash, counts;
    # int32 value column whose sums wrap at 32 bits.
    m = 1 << 14
    A = struct([rng.integers(-8, 8, m).astype(np.int32), rng.integers(-8, 8, m).astype(np.int32),
                rng.integers(1 << 28, 1 << 30, m).astype(np.int32)], [I32, I32, I32])
    with tempfile.TemporaryDirectory() as d:
        af = refrun.write_rel(d, "A", A, T)
        rc, _, _ = refrun.run(d, refrun.plan_groupby(T, af, [I32, I32, I32], [0, 1], "count", 2, 256, hashfn="bytes"))
        rs, _, _ = refrun.run(d, refrun.plan_groupby(T, af, [I32, I32, I32], [0, 1], "sum", 2, 256, hashfn="bytes"))
    save("groupby_composite", A=A, count_rows=rows_array(sorted(rc), [I32, I32, I64]),
         sum_rows=rows_array(sorted(rs), [I32, I32, I32]))

    # Partition (exactrange, 8 buckets) with the partition id prepended.
    m = 1 << 14
    A = struct([rng.integers(0, 100000, m), rng.integers(0, 1 << 40, m)], [I64, I64])
    with tempfile.TemporaryDirectory() as d:
        af = refrun.write_rel(d, "A", A, 8)
        rows, _, _ = refrun.run(d, refrun.plan_partition(8, af, [I64, I64], 0, 0, 99999, m))
    save("partition_exactrange", A=A, mn=np.array(0), mx=np.array(99999), fanout=np.array(8),
         out=rows_array(rows, [I32, I64, I64]))

    # MPSM join: build range-partitioned upstream, PK-FK with (i & 3) + 1
    # matches per key as in unit_tests/querympsmpkfkjoin.cpp.
    n = 4096
    k = rng.permutation(n).astype(np.int64)
    R = struct([k, k * 3 + 1], [I64, I64])
    fk = np.concatenate([np.full((i & 3) + 1, i, dtype=np.int64) for i in range(n)])
    fk = fk[rng.permutation(fk.shape[0])]
    S = struct([fk, rng.integers(0, 1 << 30, fk.shape[0])], [I64, I64])
    with tempfile.TemporaryDirectory() as d:
        rf = refrun.write_rel(d, "R", R, T)
        sf = refrun.write_rel(d, "S", S, T)
        rows, _, _ = refrun.run(d, refrun.plan_mpsm(T, rf, [I64, I64], sf, [I64, I64], [(0, 0), (0, 1), (1, 1)], 0,
                                                    n - 1, 2 * n, 2 * S.shape[0]))
    save("mpsm_pkfk", R=R, S=S, proj=np.array([(0, 0), (0, 1), (1, 1)]), out=rows_array(rows, [I64, I64, I64]))
    sortlimit_cases()


def sortlimit_cases():
    """Top-k with ties (input order decides), ascending and descending, on
    an int64 key and on an (int32, int32) pair; one input file so the
    arrival order is the file order."""
    rng = np.random.default_rng(20241201)
    m = 20000
    A = struct([rng.integers(-300, 300, m), np.arange(m, dtype=np.int64)], [I64, I64])
    B = struct([rng.integers(-5, 5, m).astype(np.int32), rng.integers(-40, 40, m).astype(np.int32),
                np.arange(m, dtype=np.int64)], [I32, I32, I64])
    out = {}
    with tempfile.TemporaryDirectory() as d:
        af = refrun.write_rel(d, "A", A, 1)
        bf = refrun.write_rel(d, "B", B, 1)
        for asc in (1, 0):
            for limit in (1, 100, 5000):
                rows, _, _ = refrun.run(d, refrun.plan_sortlimit(af, [I64, I64], [0], asc, limit))
                out[f"a_{asc}_{limit}"] = rows_array(rows, [I64, I64])
                rows, _, _ = refrun.run(d, refrun.plan_sortlimit(bf, [I32, I32, I64], [0, 1], asc, limit))
                out[f"b_{asc}_{limit}"] = rows_array(rows, [I32, I32, I64])
    save("sortlimit", A=A, B=B, **out)


if __name__ == "__main__":
    if sys.argv[1:] == ["sortlimit"]:
        sortlimit_cases()
    else:
        main()
