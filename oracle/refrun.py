"""Runs the reference engine (oracle/_ref/executequery, built by oracle/ref.mk
from the reference's sources) on seeded relations.

TEST INFRASTRUCTURE ONLY: used to generate golden fixtures (tests/golden/)
and as bench.py's `--impl reference` CPU arm.  Never on the product path.

Each worker thread of the reference reads its own binary file: a
`parallelscan` group holds one file, and a binary file is served as one
page, so relations are split into T non-empty files mapped one per thread
(`mapping = ((0), (1), ...)`).  A thread that receives no probe tuple makes
HashJoinOp::scanStart return Finished, after which GenericAggregate skips
scanStop and the other threads wait on the scan's barrier forever
(operators/join.cpp:626-631, operators/genericaggregate.cpp:305-307); the
non-empty split avoids that.
"""
import os
import re
import subprocess
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
EXE = os.path.join(HERE, "_ref", "executequery")
TYPENAME = {1: "int", 2: "long"}


def available():
    return os.path.exists(EXE)


def write_rel(dirpath, name, arr, T):
    """Writes arr (packed structured array) as T binary files; returns paths."""
    assert arr.shape[0] >= T, "each reference thread needs at least one tuple"
    paths = []
    for t, chunk in enumerate(np.array_split(arr, T)):
        p = f"{name}_{t:03d}.bin"
        np.ascontiguousarray(chunk).tofile(os.path.join(dirpath, p))
        paths.append(p)
    return paths


def _list(xs):
    return ", ".join(str(x) for x in xs)


def scan_node(node, files, types):
    fl = ", ".join(f'"{f}"' for f in files)
    mp = ", ".join(f"({t})" for t in range(len(files)))
    sc = ", ".join(f'"{TYPENAME[t]}"' for t in types)
    return (f'{node}: {{ type = "parallelscan"; filetype = "binary"; files = ({fl}); '
            f'mapping = ({mp}); schema = ({sc}); }};\n')


def header(buffsize=1 << 20):
    return f'path = "./";\nbuffsize = {buffsize};\n'


def _tree(*names, leaf=None):
    """Nested single-input tree: _tree('a','b', leaf='x') -> a(b(x))."""
    s = leaf
    for n in reversed(names):
        s = f'{{ name: "{n}"; input: {s}; }}'
    return s


def join_leaf(join, build, probe):
    return f'{{ name: "{join}"; build: {{ name: "{build}"; }}; probe: {{ name: "{probe}"; }}; }}'


def hashjoin_node(T, buckets, proj, tuplesperbucket=4, hashfn="modulo", bkeys=(0,), pkeys=(0,)):
    pj = ", ".join(f'"{"P" if s else "B"}${c}"' for s, c in proj)
    bk = bkeys[0] if len(bkeys) == 1 else f"[{_list(bkeys)}]"
    pk = pkeys[0] if len(pkeys) == 1 else f"[{_list(pkeys)}]"
    return (f'join: {{ type = "hashjoin"; hash: {{ fn = "{hashfn}"; buckets = {buckets}; }}; '
            f'tuplesperbucket = {tuplesperbucket}; buildjattr = {bk}; probejattr = {pk}; '
            f'projection = ({pj}); threadgroups = ( [{_list(range(T))}] ); allocpolicy = "local"; }};\n')


def plan_join_rows(T, rfiles, rtypes, sfiles, stypes, proj, buckets, **kw):
    return (header() + scan_node("scanR", rfiles, rtypes) + scan_node("scanS", sfiles, stypes)
            + hashjoin_node(T, buckets, proj, **kw) + f'merge: {{ type = "merge"; threads = {T}; }};\n'
            + "treeroot: " + _tree("merge", leaf=join_leaf("join", "scanR", "scanS")) + ";\n")


def plan_join_sum(T, rfiles, rtypes, sfiles, stypes, proj, sum_proj_index, buckets):
    """hashjoin -> printer_tuplecount -> aggregate_sum(fields=[]) -> merge
    -> aggregate_sum: the config-1 plan shape."""
    return (header() + scan_node("scanR", rfiles, rtypes) + scan_node("scanS", sfiles, stypes)
            + hashjoin_node(T, buckets, proj)
            + 'cnt: { type = "printer_tuplecount"; };\n'
            + f'agg1: {{ type = "aggregate_sum"; fields = [ ]; sumfield = {sum_proj_index}; }};\n'
            + f'merge: {{ type = "merge"; threads = {T}; }};\n'
            + 'agg2: { type = "aggregate_sum"; fields = [ ]; sumfield = 0; };\n'
            + "treeroot: " + _tree("agg2", "merge", "agg1", "cnt", leaf=join_leaf("join", "scanR", "scanS"))
            + ";\n")


def plan_groupby(T, files, types, key_cols, op, sum_col, buckets, hashfn="modulo"):
    """Thread-local aggregate -> merge -> re-aggregate (unit_tests/
    queryaggsum.cpp).  op is 'sum' or 'count'; the final operator sums the
    partial column (sums of partial sums / of partial counts)."""
    nk = len(key_cols)
    if nk == 1:
        keys1 = f"field = {key_cols[0]};"
        keys2 = "field = 0;"
        h1 = f'hash: {{ fn = "{hashfn}"; buckets = {buckets}; field = {key_cols[0]}; }};'
        h2 = f'hash: {{ fn = "{hashfn}"; buckets = {buckets}; field = 0; }};'
    else:
        keys1 = f"fields = [{_list(key_cols)}];"
        keys2 = f"fields = [{_list(range(nk))}];"
        h1 = (f'hash: {{ fn = "{hashfn}"; buckets = {buckets}; '
              f'fieldrange = [{key_cols[0]}, {key_cols[-1]}]; }};')
        h2 = f'hash: {{ fn = "{hashfn}"; buckets = {buckets}; fieldrange = [0, {nk - 1}]; }};'
    if op == "sum":
        a1 = f'agg1: {{ type = "aggregate_sum"; {keys1} sumfield = {sum_col}; {h1} }};\n'
    else:
        a1 = f'agg1: {{ type = "aggregate_count"; {keys1} {h1} }};\n'
    a2 = f'agg2: {{ type = "aggregate_sum"; {keys2} sumfield = {nk}; {h2} }};\n'
    return (header() + scan_node("scan", files, types) + a1 + f'merge: {{ type = "merge"; threads = {T}; }};\n'
            + a2 + "treeroot: " + _tree("agg2", "merge", "agg1", leaf='{ name: "scan"; }') + ";\n")


def plan_partition(T, files, types, attr, mn, mx, maxtuples):
    """partition(exactrange, buckets = T) -> threadidprepend -> merge: every
    output row carries its partition (= thread) id in front."""
    return (header() + scan_node("scan", files, types)
            + f'part: {{ type = "partition"; attr = {attr}; range = [{mn}, {mx}]; buckets = {T}; '
            f'maxtuples = {maxtuples}; sort = "no"; }};\n'
            + 'tid: { type = "threadidprepend"; };\n'
            + f'merge: {{ type = "merge"; threads = {T}; }};\n'
            + "treeroot: " + _tree("merge", "tid", "part", leaf='{ name: "scan"; }') + ";\n")


def plan_sortlimit(files, types, by, asc, limit):
    """scan -> sortlimit as the root: SortLimit runs on thread 0 only
    (operators/sortlimit.cpp:224-228), so the plan has no merge above it."""
    cols = ", ".join(f'"${c}"' for c in by)
    return (header() + scan_node("scan", files, types)
            + f'top: {{ type = "sortlimit"; by = ({cols}); asc = [{asc}]; limit = [{limit}]; }};\n'
            + 'treeroot: { name: "top"; input: { name: "scan"; }; };\n')


def plan_mpsm(T, rfiles, rtypes, sfiles, stypes, proj, mn, mx, maxb, maxp):
    """partition(build, exactrange) -> mpsmjoin(buildprepartitioned) -> merge
    (unit_tests/querypartitionedmpsmpkfkjoin.cpp)."""
    pj = ", ".join(f'"{"P" if s else "B"}${c}"' for s, c in proj)
    return (header() + scan_node("scanR", rfiles, rtypes) + scan_node("scanS", sfiles, stypes)
            + f'part: {{ type = "partition"; attr = 0; range = [{mn}, {mx}]; buckets = {T}; '
            f'maxtuples = {maxb}; sort = "no"; }};\n'
            + f'join: {{ type = "mpsmjoin"; maxbuildtuples = {maxb}; maxprobetuples = {maxp}; '
            f'threadgroups = ( [{_list(range(T))}] ); buildjattr = 0; probejattr = 0; projection = ({pj}); '
            f'buildprepartitioned: {{ range = [{mn}, {mx}]; buckets = {T}; }}; }};\n'
            + f'merge: {{ type = "merge"; threads = {T}; }};\n'
            + "treeroot: " + _tree("merge", leaf=(f'{{ name: "join"; build: {{ name: "part"; input: '
                                                  f'{{ name: "scanR"; }}; }}; probe: {{ name: "scanS"; }}; }}'))
            + ";\n")


_ROW = re.compile(r"^-?\d+(\|-?\d+)*$")


def run(workdir, plan_text, timeout=600, exe=None):
    """Runs a plan with the reference engine (or another driver with the
    same output format, `exe`); returns (rows as list of int tuples,
    ResponseTimeInSec, tuple count printed by printer_tuplecount or None)."""
    p = os.path.join(workdir, "plan.conf")
    with open(p, "w") as f:
        f.write(plan_text)
    t0 = time.time()
    r = subprocess.run([exe or EXE, "plan.conf"], cwd=workdir, capture_output=True, text=True, timeout=timeout)
    wall = time.time() - t0
    out = r.stdout.splitlines()
    rows, rt, total = [], None, None
    in_rows = False
    for line in out:
        if line.startswith("BUFFSIZE:"):
            in_rows = True
            continue
        if line.startswith("ResponseTimeInCycles:"):
            in_rows = False
            continue
        if line.startswith("ResponseTimeInSec:"):
            rt = float(line.split(":")[1])
            continue
        m = re.search(r"TupleCountPrinter \(total=([\d,]+) tuples\)", line)
        if m and total is None:
            total = int(m.group(1).replace(",", ""))
        if in_rows and _ROW.match(line.strip()):
            rows.append(tuple(int(x) for x in line.strip().split("|")))
    if rt is None:
        raise RuntimeError(f"reference run failed (rc={r.returncode}, {wall:.1f}s): {r.stdout[-2000:]} {r.stderr[-2000:]}")
    return rows, rt, total
