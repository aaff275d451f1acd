"""Reference plan files run unchanged through the GPU host engine
(pythia-core_b200/host/pyg_executequery): the same plan text the reference
engine ran to make the golden fixtures gives the same rows."""
import os
import tempfile

import numpy as np
import pytest

import refrun
from util import canon_rows, rows

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "pythia-core_b200", "host", "pyg_executequery")
T = 4


def run_plan(make_plan, *rels):
    with tempfile.TemporaryDirectory() as d:
        files = [refrun.write_rel(d, f"r{i}", r, T) for i, r in enumerate(rels)]
        return refrun.run(d, make_plan(*files), exe=EXE)


def as_struct(rows_, dtype):
    a = np.zeros(len(rows_), dtype=dtype)
    for i, name in enumerate(dtype.names):
        a[name] = [r[i] for r in rows_]
    return a


@pytest.mark.parametrize("name", ["join_pkfk", "join_dups"])
def test_hashjoin_plan(golden, name):
    g = golden(name)
    proj = [tuple(int(v) for v in p) for p in g["proj"]]
    rt, st = [int(x) for x in g["rtypes"]], [int(x) for x in g["stypes"]]
    out, secs, _ = run_plan(lambda rf, sf: refrun.plan_join_rows(T, rf, rt, sf, st, proj, int(g["buckets"])),
                            g["R"], g["S"])
    assert canon_rows(as_struct(out, g["out"].dtype)) == canon_rows(g["out"])
    assert secs >= 0


def test_composite_key_plan(golden):
    g = golden("join_composite")
    proj = [tuple(int(v) for v in p) for p in g["proj"]]
    rt, st = [int(x) for x in g["rtypes"]], [int(x) for x in g["stypes"]]
    out, _, _ = run_plan(lambda rf, sf: refrun.plan_join_rows(T, rf, rt, sf, st, proj, int(g["buckets"]),
                                                              hashfn="bytes", bkeys=(0, 1), pkeys=(0, 1)),
                         g["R"], g["S"])
    assert canon_rows(as_struct(out, g["out"].dtype)) == canon_rows(g["out"])


def test_fused_join_sum_plan(golden):
    """hashjoin -> printer_tuplecount -> aggregate_sum -> merge ->
    aggregate_sum runs as one fused GPU join + aggregate."""
    g = golden("join_sum")
    out, _, total = run_plan(lambda rf, sf: refrun.plan_join_sum(T, rf, [2, 2], sf, [2, 2], [(0, 1), (1, 1)], 1,
                                                                 1 << 12), g["R"], g["S"])
    assert out == [(int(g["sum"]),)]
    assert total == int(g["count"])


def test_groupby_plans(golden):
    g = golden("groupby_int64")
    out, _, _ = run_plan(lambda f: refrun.plan_groupby(T, f, [2, 2], [0], "sum", 1, 1024), g["A"])
    assert sorted(out) == rows(g["sum_rows"])
    out, _, _ = run_plan(lambda f: refrun.plan_groupby(T, f, [2, 2], [0], "count", 1, 1024), g["A"])
    assert sorted(out) == rows(g["count_rows"])
    g = golden("groupby_composite")
    out, _, _ = run_plan(lambda f: refrun.plan_groupby(T, f, [1, 1, 1], [0, 1], "count", 2, 256, hashfn="bytes"),
                         g["A"])
    assert sorted(out) == rows(g["count_rows"])
    out, _, _ = run_plan(lambda f: refrun.plan_groupby(T, f, [1, 1, 1], [0, 1], "sum", 2, 256, hashfn="bytes"),
                         g["A"])
    assert sorted(out) == rows(g["sum_rows"])


def test_mpsm_plan(golden):
    g = golden("mpsm_pkfk")
    proj = [tuple(int(v) for v in p) for p in g["proj"]]
    n = g["R"].shape[0]
    out, _, _ = run_plan(lambda rf, sf: refrun.plan_mpsm(T, rf, [2, 2], sf, [2, 2], proj, 0, n - 1, 2 * n,
                                                         2 * g["S"].shape[0]), g["R"], g["S"])
    assert canon_rows(as_struct(out, g["out"].dtype)) == canon_rows(g["out"])


def test_operator_results_stay_on_the_device(golden):
    """partition -> mpsmjoin -> merge: the partition's output is read by
    the join in device memory; the only device-to-host copy of results is
    the join's rows pulled by the driver (DeviceToHostResultBytes)."""
    import subprocess
    g = golden("mpsm_pkfk")
    proj = [tuple(int(v) for v in p) for p in g["proj"]]
    n = g["R"].shape[0]
    with tempfile.TemporaryDirectory() as d:
        rf = refrun.write_rel(d, "R", g["R"], T)
        sf = refrun.write_rel(d, "S", g["S"], T)
        with open(os.path.join(d, "plan.conf"), "w") as f:
            f.write(refrun.plan_mpsm(T, rf, [2, 2], sf, [2, 2], proj, 0, n - 1, 2 * n, 2 * g["S"].shape[0]))
        r = subprocess.run([EXE, "plan.conf"], cwd=d, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    line = [x for x in r.stdout.splitlines() if x.startswith("DeviceToHostResultBytes:")]
    assert line and int(line[0].split(":")[1]) == g["out"].shape[0] * g["out"].dtype.itemsize


def test_partition_plan_orders_partitions(golden):
    g = golden("partition_exactrange")
    A = g["A"]
    plan = (lambda f: refrun.header() + refrun.scan_node("scan", f, [2, 2])
            + 'part: { type = "partition"; attr = 0; range = [0, 99999]; buckets = 8; maxtuples = 20000; '
              'sort = "yes"; };\n'
            + f'merge: {{ type = "merge"; threads = {T}; }};\n'
            + "treeroot: " + refrun._tree("merge", "part", leaf='{ name: "scan"; }') + ";\n")
    out, _, _ = run_plan(plan, A)
    keys = np.array([r[0] for r in out])
    assert np.all(np.diff(keys) >= 0)  # partitions in order, each sorted
    assert sorted(out) == sorted(rows(A))


def _mpsm_family_plan(jtype, rf, sf, n, m, mfbko=None, presort=False):
    """partition(build) [and partition(probe), each sorted] -> jtype ->
    merge, over (int64, int64) relations with keys in [0, n)."""
    extra = f"mostfreqbuildkeyoccurances = {mfbko}; " if mfbko is not None else ""
    sort = '"yes"' if presort else '"no"'
    part = (lambda name, maxt: f'{name}: {{ type = "partition"; attr = 0; range = [0, {n - 1}]; buckets = {T}; '
            f'maxtuples = {maxt}; sort = {sort}; }};\n')
    probe_leaf = '{ name: "partS"; input: { name: "scanS"; }; }' if presort else '{ name: "scanS"; }'
    return (refrun.header() + refrun.scan_node("scanR", rf, [2, 2]) + refrun.scan_node("scanS", sf, [2, 2])
            + part("partR", 2 * n) + (part("partS", 2 * m) if presort else "")
            + f'join: {{ type = "{jtype}"; maxbuildtuples = {2 * n}; maxprobetuples = {2 * m}; '
              f'threadgroups = ( [{refrun._list(range(T))}] ); buildjattr = 0; probejattr = 0; '
              f'projection = ("B$1", "P$1"); {extra}'
              f'buildprepartitioned: {{ range = [0, {n - 1}]; buckets = {T}; }}; }};\n'
            + f'merge: {{ type = "merge"; threads = {T}; }};\n'
            + "treeroot: " + refrun._tree("merge", leaf=(f'{{ name: "join"; build: {{ name: "partR"; input: '
                                                         f'{{ name: "scanR"; }}; }}; probe: {probe_leaf}; }}'))
            + ";\n")


def _pkfk(n, m, seed, dup_every=0):
    rng = np.random.default_rng(seed)
    dt = np.dtype([("c0", np.int64), ("c1", np.int64)])
    k = rng.permutation(n).astype(np.int64)
    if dup_every:
        k[::dup_every] = k[1]
    R = np.zeros(n, dtype=dt)
    R["c0"], R["c1"] = k, k * 7 + 3
    S = np.zeros(m, dtype=dt)
    S["c0"], S["c1"] = rng.integers(0, n, m), rng.integers(0, 1 << 20, m)
    return R, S


@pytest.mark.parametrize("jtype,mfbko,presort", [("newmpsmjoin", None, False), ("newmpsmjoin", 1, False),
                                                 ("preprejoin", 1, True), ("preprejoin", 4, True)])
def test_mpsm_family_plans_match_oracle(jtype, mfbko, presort):
    """`newmpsmjoin` and `preprejoin` plans (operators/join.cpp:1619-2212;
    preprejoin over sorted partitions of both sides) give the joined rows
    of the oracle on PK-FK inputs, whose build keys occur once."""
    import oracle as O
    n, m = 5000, 40000
    R, S = _pkfk(n, m, 11)
    out, _, _ = run_plan(lambda rf, sf: _mpsm_family_plan(jtype, rf, sf, n, m, mfbko, presort), R, S)
    want = O.hashjoin_materialize(R, [2, 2], [0], S, [2, 2], [0], [(0, 1), (1, 1)], buckets=n)
    assert sorted(out) == sorted(rows(want))


def test_mpsm_family_refuses_build_keys_above_mfbko():
    """A build key that occurs more often than mostfreqbuildkeyoccurances is
    refused with an error (the reference's merge buffer holds only that
    many); a bound that covers the repeats joins normally."""
    import oracle as O
    n, m = 4000, 20000
    R, S = _pkfk(n, m, 12, dup_every=100)  # key k[1] occurs about 41 times
    most = int(np.unique(R["c0"], return_counts=True)[1].max())
    with pytest.raises(RuntimeError, match="mostfreqbuildkeyoccurances"):
        run_plan(lambda rf, sf: _mpsm_family_plan("preprejoin", rf, sf, n, m, most - 1, True), R, S)
    out, _, _ = run_plan(lambda rf, sf: _mpsm_family_plan("preprejoin", rf, sf, n, m, most, True), R, S)
    want = O.hashjoin_materialize(R, [2, 2], [0], S, [2, 2], [0], [(0, 1), (1, 1)], buckets=n)
    assert sorted(out) == sorted(rows(want))


def test_sort_plan():
    """scan -> sort (attr 0) -> merge: every tuple once, keys in order
    (operators/sort.cpp:87-311)."""
    rng = np.random.default_rng(13)
    dt = np.dtype([("c0", np.int64), ("c1", np.int64)])
    A = np.zeros(30000, dtype=dt)
    A["c0"], A["c1"] = rng.integers(-(1 << 40), 1 << 40, A.shape[0]), rng.integers(0, 1000, A.shape[0])
    A["c0"][::7] = 12345  # ties
    plan = (lambda f: refrun.header() + refrun.scan_node("scan", f, [2, 2])
            + f'srt: {{ type = "sort"; attr = 0; maxtuples = ( {", ".join(chr(34) + "1 M" + chr(34) for _ in range(T))} ); }};\n'
            + f'merge: {{ type = "merge"; threads = {T}; }};\n'
            + "treeroot: " + refrun._tree("merge", "srt", leaf='{ name: "scan"; }') + ";\n")
    out, _, _ = run_plan(plan, A)
    keys = [r[0] for r in out]
    assert keys == sorted(keys)
    assert sorted(out) == sorted(rows(A))


def test_sortlimit_plan(golden):
    """scan -> sortlimit gives the reference engine's own top-k rows
    (golden fixture made by the reference from the same plan text)."""
    g = golden("sortlimit")
    for asc in (1, 0):
        for limit in (1, 100, 5000):
            out, _, _ = run_plan(lambda f: refrun.plan_sortlimit(f, [2, 2], [0], asc, limit), g["A"])
            assert out == rows(g[f"a_{asc}_{limit}"])
    out, _, _ = run_plan(lambda f: refrun.plan_sortlimit(f, [1, 1, 2], [0, 1], 0, 100), g["B"])
    assert out == rows(g["b_0_100"])


def test_shmwriter_plan(tmp_path):
    """scan -> shmwriter: the input's tuples land, in order, in segments of
    at most `size` bytes named path + counter, alternating between the two
    paths and advancing the counter after each cycle; the last segment is
    truncated to what it holds (operators/memsegmentwriter.cpp)."""
    rng = np.random.default_rng(17)
    dt = np.dtype([("c0", np.int64), ("c1", np.int64)])
    A = np.zeros(2500, dtype=dt)
    A["c0"], A["c1"] = rng.integers(-(1 << 50), 1 << 50, A.shape[0]), np.arange(A.shape[0])
    pa, pb = str(tmp_path / "segA"), str(tmp_path / "segB")
    size = 1000 * 16 + 8  # 1000 whole tuples per segment
    plan = (lambda f: refrun.header(1 << 12) + refrun.scan_node("scan", f, [2, 2])
            + f'w: {{ type = "shmwriter"; size = {size}; paths = ("{pa}", "{pb}"); }};\n'
            + 'treeroot: { name: "w"; input: { name: "scan"; }; };\n')
    with tempfile.TemporaryDirectory() as d:
        files = [refrun.write_rel(d, "r0", A, 1)]
        out, _, _ = refrun.run(d, plan(files[0]), exe=EXE)
    assert out == []
    names = [pa + "0000000", pb + "0000000", pa + "0000001"]
    segs = [np.fromfile(n, dtype=dt) for n in names]
    assert [s.shape[0] for s in segs] == [1000, 1000, 500]
    assert np.array_equal(np.concatenate(segs), A)
    assert not os.path.exists(pb + "0000001")
