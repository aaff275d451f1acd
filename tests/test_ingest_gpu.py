"""Overlapped ingest (pyg_upload_*): bytes streamed through the pinned
staging ring land in device memory unchanged, in order, across slot reuse
and destination growth; the plan engine's scans feed GPU operators through
it."""
import os
import subprocess
import tempfile

import numpy as np
import pytest

import pyg
import refrun

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "pythia-core_b200", "host", "pyg_executequery")


@pytest.fixture(scope="module")
def ctx():
    c = pyg.Ctx(0, use_torch_stream=False)
    yield c
    c.close()


@pytest.mark.parametrize("capacity", [0, 1000, 1 << 22])
def test_upload_round_trip(ctx, capacity):
    rng = np.random.default_rng(7)
    sizes = [0, 1, 4095, 4096, 4097, 70000, 3, 1 << 18]
    chunks = [rng.integers(0, 256, s, dtype=np.uint8) for s in sizes]
    # 4 KiB slots, 3 of them: every chunk above spans several slots, slots
    # are refilled while earlier copies run, and capacity 0 / 1000 forces
    # the destination to grow.
    buf = ctx.upload(chunks, capacity=capacity, slot_bytes=4096, slots=3)
    want = np.concatenate(chunks)
    assert buf.nbytes == want.size
    got = np.empty(want.size, np.uint8)
    ctx.d2h(got, buf)
    assert np.array_equal(got, want)
    buf.free()


def test_upload_empty_and_bad_arguments(ctx):
    buf = ctx.upload([], capacity=0, slot_bytes=1024, slots=2)
    assert buf.nbytes == 0
    buf.free()
    with pytest.raises(pyg.PygError):
        ctx.upload([np.zeros(10, np.uint8)], slot_bytes=1024, slots=1)  # needs >= 2 slots


def test_scan_streams_files_into_device_for_gpu_parents(golden):
    """scan -> hashjoin -> sum: both scans are streamed into HBM through the
    upload ring (IngestToDeviceBytes = the files' bytes) and the join reads
    them there; the aggregate matches the golden rows."""
    g = golden("join_pkfk")
    proj = [tuple(int(v) for v in p) for p in g["proj"]]
    rt, st = [int(x) for x in g["rtypes"]], [int(x) for x in g["stypes"]]
    with tempfile.TemporaryDirectory() as d:
        rf = refrun.write_rel(d, "R", g["R"], 4)
        sf = refrun.write_rel(d, "S", g["S"], 4)
        with open(os.path.join(d, "plan.conf"), "w") as f:
            f.write(refrun.plan_join_rows(4, rf, rt, sf, st, proj, int(g["buckets"])))
        r = subprocess.run([EXE, "plan.conf"], cwd=d, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    stats = dict(x.split(": ", 1) for x in r.stdout.splitlines() if x.startswith(("Ingest", "DeviceToHost")))
    assert int(stats["IngestToDeviceBytes"]) == g["R"].nbytes + g["S"].nbytes
    assert float(stats["IngestSeconds"]) >= 0
    assert int(stats["DeviceToHostResultBytes"]) == g["out"].nbytes
