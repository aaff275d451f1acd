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


class _OracleBackend:
    """CPU stand-in for the GPU kernels behind dist.py (test only): the C
    oracle's partition (low key bits) and join + sum over host buffers."""

    def __init__(self, O):
        self.O = O

    def empty(self, nbytes):
        import torch
        return torch.empty(max(nbytes, 16), dtype=torch.uint8)

    def _view(self, buf, n, types):
        dt = self.O.dtype_of(types)
        return buf[: n * dt.itemsize].numpy().view(dt)

    def partition(self, buf, n, types, key_col, fanout):
        import torch
        out, offs = self.O.partition(self._view(buf, n, types).copy(), types, key_col, 2, fanout)
        t = self.empty(out.nbytes)
        t[: out.nbytes].copy_(torch.from_numpy(out.view("u1").copy()))
        return t, [int(x) for x in offs]

    def join_agg(self, R, nR, rtypes, rkeys, S, nS, stypes, skeys, proj):
        A, B = self._view(R, nR, rtypes).copy(), self._view(S, nS, stypes).copy()
        return self.O.hashjoin_agg(A, rtypes, rkeys, B, stypes, skeys, proj, buckets=max(16, nR))


def _shard(seed, rank, world):
    """Rank `rank`'s shards of R (unique keys spread over all ranks) and S."""
    import numpy as np
    rng = np.random.default_rng(seed)
    nR, nS = 3000 * world, 20000 * world
    keys = rng.permutation(nR).astype(np.int64) * 7 - 9000  # some negative keys
    R = np.zeros(nR, dtype=[("c0", "<i8"), ("c1", "<i8")])
    R["c0"], R["c1"] = keys, rng.integers(-(1 << 62), 1 << 62, nR)
    S = np.zeros(nS, dtype=[("c0", "<i8"), ("c1", "<i8")])
    S["c0"] = keys[rng.integers(0, nR, nS)] + (rng.random(nS) < 0.1)
    S["c1"] = rng.integers(-(1 << 62), 1 << 62, nS)
    return R, S, np.ascontiguousarray(R[rank::world]), np.ascontiguousarray(S[rank::world])


def _dist_join_rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, os.path.join(ROOT, "pythia-core_b200"))
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import torch
    import dist as pyg_dist
    import oracle as O

    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        R, S, Rl, Sl = _shard(7, rank, world)
        be = _OracleBackend(O)
        Rt = torch.from_numpy(Rl.view("u1").copy())
        St = torch.from_numpy(Sl.view("u1").copy())
        types = [2, 2]
        got = pyg_dist.join_agg(dist, be, Rt, Rl.shape[0], types, 0, St, Sl.shape[0], types, 0, [(0, 1), (1, 1)])
        # Each key sits on exactly one rank after the shuffle.
        Rr, mR = pyg_dist.shuffle(dist, be, Rt, Rl.shape[0], types, 0)
        mine = set(be._view(Rr, mR, types)["c0"].tolist())
        allk = [None] * world
        dist.all_gather_object(allk, mine)
        want = O.hashjoin_agg(R, types, [0], S, types, [0], [(0, 1), (1, 1)], buckets=R.shape[0])
        q.put((rank, got, want, sum(len(k) for k in allk), len(set().union(*allk)), R.shape[0]))
    finally:
        dist.destroy_process_group()


def test_partitioned_join_exchange_gloo():
    """The partitioned multi-GPU join's host logic on two gloo ranks: hash
    buckets to contiguous per-rank ranges, the size and tuple exchanges, the
    local join and the all-reduce of (count, sums) give the oracle's result
    over the union of both ranks' relations; each key lands on one rank."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_dist_join_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(180)
        assert p.exitcode == 0
    res = [q.get(timeout=10) for _ in range(2)]
    for rank, got, want, nkeys, ndistinct, nR in res:
        assert (got[0], got[1]) == want
        assert nkeys == ndistinct == nR


def test_bucket_ranges_cover_ranks():
    sys.path.insert(0, os.path.join(ROOT, "pythia-core_b200"))
    import dist as pyg_dist

    for world in (1, 2, 3, 5, 8):
        F = pyg_dist.bucket_count(world)
        assert F & (F - 1) == 0 and F >= 64 * world
        owners = [pyg_dist.rank_of_bucket(b, world, F) for b in range(F)]
        assert owners == sorted(owners) and set(owners) == set(range(world))
        sizes = [owners.count(r) for r in range(world)]
        assert max(sizes) - min(sizes) <= 1
