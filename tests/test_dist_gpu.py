"""The partitioned join (dist.py) with its GPU backend on one GPU: a
world-size-1 NCCL group, so the hash partition (pyg_partition, SPLIT_HASH),
the all_to_all exchanges on device buffers, the local join and the
all-reduce all run on cuda:0 through the product code.  Same result as the
oracle.  (Several GPUs are exercised by the gloo test of the same logic.)"""
import os
import socket

import numpy as np
import pytest

import oracle as O
import pyg
from util import I64, struct, to_device

pytestmark = pytest.mark.gpu


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_partitioned_join_one_gpu(ctx, torch_cuda):
    import datetime

    import torch.distributed as dist

    import dist as pyg_dist

    torch = torch_cuda
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(_free_port()))
    dist.init_process_group("nccl", rank=0, world_size=1, timeout=datetime.timedelta(seconds=60),
                            device_id=torch.device("cuda:0"))
    try:
        rng = np.random.default_rng(41)
        n, m = 1 << 16, 1 << 20
        k = rng.permutation(n).astype(np.int64) * 3 - 100
        R = struct([k, rng.integers(-(1 << 62), 1 << 62, n)], [I64, I64])
        S = struct([k[rng.integers(0, n, m)] + (rng.random(m) < 0.1), rng.integers(-(1 << 62), 1 << 62, m)],
                   [I64, I64])
        be = pyg_dist.GpuBackend(ctx, torch.device("cuda:0"))
        got = pyg_dist.join_agg(dist, be, to_device(torch, R), n, [I64, I64], 0, to_device(torch, S), m, [I64, I64], 0,
                                [(0, 1), (1, 1)])
        want = O.hashjoin_agg(R, [I64, I64], [0], S, [I64, I64], [0], [(0, 1), (1, 1)], buckets=n)
        assert (got[0], got[1]) == want
    finally:
        dist.destroy_process_group()
