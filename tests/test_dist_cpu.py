"""Multi-rank harness of bench.py on CPU (gloo, world size 2): each rank
joins its own relations (replicas, no data exchange) and the job's time is
the max over ranks."""
import os
import socket
import sys

import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench

    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        r, w, local = bench.dist_env()
        ms = bench.max_over_ranks(10.0 * (rank + 1), dist, "cpu")
        q.put((r, w, local, ms))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    assert [(r, w, l) for r, w, l, _ in res] == [(0, 2, 0), (1, 2, 1)]
    assert all(ms == 20.0 for *_, ms in res)


def test_single_rank_is_identity():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.max_over_ranks(3.5, None, "cpu") == 3.5
