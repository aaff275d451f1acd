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
