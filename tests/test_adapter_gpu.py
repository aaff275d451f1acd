"""GpuHashJoinOp inside the reference engine (pythia-core_b200/adapter):
reference plan files run in the reference's own Query / ParallelScanOp /
MergeOp / aggregate operators, with the hashjoin node replaced by the GPU
operator.  Merge threads call scanStart / getNext / scanStop on it
concurrently (the multi-thread Operator contract: every thread of a group
drains its streams, the leader joins on the GPU between two barriers, each
thread serves its slice); the rows equal the golden rows and the
reference's own HashJoinOp on the same plan (--cpu)."""
import os
import subprocess
import tempfile

import pytest

import refrun
from util import canon_rows

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ADAPTER = os.path.join(ROOT, "pythia-core_b200", "adapter", "_build", "adapter_query")
T = 4

needs_adapter = pytest.mark.skipif(not os.path.exists(ADAPTER),
                                   reason="adapter not built (needs the reference sources at build time)")


def run_adapter(plan_text, rels, cpu=False):
    with tempfile.TemporaryDirectory() as d:
        files = [refrun.write_rel(d, f"r{i}", r, T) for i, r in enumerate(rels)]
        with open(os.path.join(d, "plan.conf"), "w") as f:
            f.write(plan_text(*files))
        r = subprocess.run([ADAPTER] + (["--cpu"] if cpu else []) + ["plan.conf"], cwd=d, capture_output=True,
                           text=True, timeout=300)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    lines = r.stdout.splitlines()
    stats = dict(x.split(": ", 1) for x in lines if x.startswith(("GpuHashJoinOps", "GpuKernelLaunches")))
    rows = [tuple(int(v) for v in x.split("|")) for x in lines if refrun._ROW.match(x.strip())]
    return rows, stats


def struct_rows(rows, dtype):
    import numpy as np
    a = np.zeros(len(rows), dtype=dtype)
    for i, name in enumerate(dtype.names):
        a[name] = [r[i] for r in rows]
    return canon_rows(a)


def join_plan(g, **kw):
    proj = [tuple(int(v) for v in p) for p in g["proj"]]
    rt, st = [int(x) for x in g["rtypes"]], [int(x) for x in g["stypes"]]
    return lambda rf, sf: refrun.plan_join_rows(T, rf, rt, sf, st, proj, int(g["buckets"]), **kw)


@needs_adapter
def test_reference_hashjoin_through_the_adapter_driver(golden):
    """--cpu: the driver runs the plan on the reference's own HashJoinOp."""
    g = golden("join_pkfk")
    rows, stats = run_adapter(join_plan(g), [g["R"], g["S"]], cpu=True)
    assert stats["GpuHashJoinOps"] == "0"
    assert struct_rows(rows, g["out"].dtype) == canon_rows(g["out"])


@needs_adapter
@pytest.mark.gpu
@pytest.mark.parametrize("name,kw", [("join_pkfk", {}), ("join_dups", {}),
                                     ("join_composite", {"hashfn": "bytes", "bkeys": (0, 1), "pkeys": (0, 1)})])
def test_gpu_hashjoin_in_the_reference_engine(golden, name, kw):
    g = golden(name)
    rows, stats = run_adapter(join_plan(g, **kw), [g["R"], g["S"]])
    assert stats["GpuHashJoinOps"] == "1"
    assert int(stats["GpuKernelLaunches"]) > 0
    assert struct_rows(rows, g["out"].dtype) == canon_rows(g["out"])


@needs_adapter
@pytest.mark.gpu
def test_thread_groups_join_their_own_threads(golden):
    """threadgroups ([0,1],[2,3]): each group joins only the tuples its own
    threads scanned, exactly as the reference's HashJoinOp does."""
    g = golden("join_dups")
    proj = [tuple(int(v) for v in p) for p in g["proj"]]
    rt, st = [int(x) for x in g["rtypes"]], [int(x) for x in g["stypes"]]

    def plan(rf, sf):
        text = refrun.plan_join_rows(T, rf, rt, sf, st, proj, int(g["buckets"]))
        return text.replace("threadgroups = ( [0, 1, 2, 3] )", "threadgroups = ( [0, 1], [2, 3] )")

    gpu, _ = run_adapter(plan, [g["R"], g["S"]])
    cpu, _ = run_adapter(plan, [g["R"], g["S"]], cpu=True)
    assert sorted(gpu) == sorted(cpu)
    assert len(gpu) < g["out"].shape[0]  # groups really were separate


@needs_adapter
@pytest.mark.gpu
def test_join_feeds_reference_aggregates(golden):
    """hashjoin -> printer_tuplecount -> aggregate_sum -> merge ->
    aggregate_sum: the reference's aggregates consume the GPU operator's
    pages on every merge thread."""
    g = golden("join_sum")
    rows, _ = run_adapter(lambda rf, sf: refrun.plan_join_sum(T, rf, [2, 2], sf, [2, 2], [(0, 1), (1, 1)], 1,
                                                               1 << 12), [g["R"], g["S"]])
    assert rows == [(int(g["sum"]),)]


@needs_adapter
@pytest.mark.gpu
def test_small_pages_and_empty_slices(golden):
    """buffsize of 64 bytes: many pages per thread, and threads whose slice
    of the output is empty (an output smaller than the thread count)."""
    g = golden("join_pkfk")
    base = join_plan(g)
    rows, _ = run_adapter(lambda rf, sf: base(rf, sf).replace("buffsize = 1048576;", "buffsize = 64;"),
                          [g["R"], g["S"]])
    assert struct_rows(rows, g["out"].dtype) == canon_rows(g["out"])
    R, S = g["R"], g["S"]
    tiny_s = S[:T].copy()
    rows, _ = run_adapter(join_plan(g), [R, tiny_s])
    cpu, _ = run_adapter(join_plan(g), [R, tiny_s], cpu=True)
    assert sorted(rows) == sorted(cpu)
