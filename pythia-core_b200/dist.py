"""Partitioned hash join + aggregation across GPUs, one process per GPU.

The reference scales a join out by shuffling both relations by a hash of the
key to the node that owns it (the hash-repartitioning shuffle,
operators/shuffle.cpp:274-287, with the data_sender_shuffle_* /
data_recver_* operator pairs carrying the tuples), joining locally and
combining the partial aggregates.  Here, per rank:

  1. partition    both local relations by a hash of the key into F = a
                  power of two >= 64 x world buckets on the device
                  (pyg_partition, SPLIT_HASH); bucket b belongs to rank
                  b * world // F, so each rank's tuples are one contiguous
                  byte range of the partitioned buffer;
  2. exchange     the per-rank sizes, then the tuples, with one
                  all_to_all_single each (NCCL over NVLink / NVSwitch on GPUs;
                  received tuples land in this rank's memory before any
                  kernel reads them);
  3. join         the received relations with the one-shot join + sum
                  (pyg_hashjoin_agg), every key now on exactly one rank;
  4. combine      all_reduce(SUM) of (count, sums): int64 sums wrap modulo
                  2^64 as the reference's `CtLong +=` does.

The kernels are behind a small backend interface (partition by key hash,
join + sum, allocation) so that the exchange logic can also run on CPU
ranks over gloo; the product backend is `GpuBackend`, which calls libpyg
and has no CPU fallback.
"""
import torch

import pyg

MIN_BUCKETS_PER_RANK = 64


def bucket_count(world):
    f = MIN_BUCKETS_PER_RANK * world
    return 1 << (f - 1).bit_length()


def rank_of_bucket(b, world, fanout):
    return b * world // fanout


class GpuBackend:
    """libpyg on this rank's GPU: hash partition, join + sum, device buffers."""

    def __init__(self, ctx, device):
        self.ctx = ctx
        self.device = device

    def empty(self, nbytes):
        return torch.empty(max(nbytes, 16), dtype=torch.uint8, device=self.device)

    def partition(self, buf, n, types, key_col, fanout):
        out = self.empty(n * _tuple_bytes(types))
        offs = self.ctx.partition(pyg.Rel(buf, n, types), key_col, pyg.SPLIT_HASH, fanout, out)
        return out, [int(x) for x in offs]

    def join_agg(self, R, nR, rtypes, rkeys, S, nS, stypes, skeys, proj):
        return self.ctx.hashjoin_agg(pyg.Rel(R, nR, rtypes), rkeys, pyg.Rel(S, nS, stypes), skeys, proj)


def _tuple_bytes(types):
    return sum(4 if t == pyg.INT32 else 8 for t in types)


def shuffle(dist, backend, buf, n, types, key_col):
    """Sends every tuple of the local relation to the rank that owns its
    key's hash bucket; returns (received buffer, received tuples)."""
    world = dist.get_world_size()
    tb = _tuple_bytes(types)
    fanout = bucket_count(world)
    part, offs = backend.partition(buf, n, types, key_col, fanout)
    # Contiguous bucket ranges per destination rank.
    starts = [offs[min(fanout, -(-r * fanout // world))] for r in range(world)] + [offs[fanout]]
    send = [starts[r + 1] - starts[r] for r in range(world)]
    assert all(rank_of_bucket(b, world, fanout) == r for r in range(world)
               for b in range(-(-r * fanout // world), -(-(r + 1) * fanout // world)))
    dev = part.device
    scount = torch.tensor(send, dtype=torch.int64, device=dev)
    rcount = torch.empty(world, dtype=torch.int64, device=dev)
    dist.all_to_all_single(rcount, scount)
    recv = [int(x) for x in rcount.tolist()]
    m = sum(recv)
    out = backend.empty(m * tb)
    dist.all_to_all_single(out[: m * tb], part[: n * tb], [c * tb for c in recv], [c * tb for c in send])
    return out, m


def join_agg(dist, backend, R, nR, rtypes, rkey, S, nS, stypes, skey, proj):
    """Distributed PK-FK or general hash join + sum over the ranks' local
    relations: (match count, [wrapped sum of each projected column])."""
    Rr, mR = shuffle(dist, backend, R, nR, rtypes, rkey)
    Sr, mS = shuffle(dist, backend, S, nS, stypes, skey)
    cnt, sums = backend.join_agg(Rr, mR, rtypes, [rkey], Sr, mS, stypes, [skey], proj)
    vals = [cnt] + [((s + (1 << 63)) % (1 << 64)) - (1 << 63) for s in sums]
    t = torch.tensor(vals, dtype=torch.int64, device=Rr.device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    out = [int(x) for x in t.tolist()]
    return out[0], out[1:]
