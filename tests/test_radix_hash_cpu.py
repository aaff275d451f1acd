"""The radix operators' partition / slot hash (rj_hash and rj_slot in
pythia-core_b200/csrc/radixpart.cuh), restated on the host: dense key ranges
must spread evenly, and keys on a regular stride (powers of two, Fibonacci
numbers) must not pile into long linear-probe chains inside a partition's
shared-memory table.  The GPU side is covered by test_radix_strided_keys."""
import numpy as np
import pytest

MUL = np.uint64(0x9E3779B97F4A7C15)
TS = 12288  # 16-byte slots of the join's 192 KB table


def rj_hash(k):
    k = k.astype(np.uint64)
    k = k ^ (k >> np.uint64(32))
    k = k ^ (k >> np.uint64(21))
    k = k ^ (k >> np.uint64(16))
    return k * MUL


def probes_per_insert(slots):
    """Mean linear-probe length of inserting `slots` (no wrap-around): the
    occupied positions, and so the total displacement, do not depend on the
    insertion order; in sorted order pos_j = j + max_{i <= j}(slot_i - i)."""
    s = np.sort(slots.astype(np.int64))
    j = np.arange(len(s))
    pos = j + np.maximum.accumulate(s - j)
    return float((pos - s + 1).mean())


def worst_partition(keys, fb):
    h = rj_hash(keys)
    part = (h >> np.uint64(64 - fb)).astype(np.int64)
    slot = ((((h >> np.uint64(32 - fb)) & np.uint64(0xFFFFFFFF)) * np.uint64(TS)) >> np.uint64(32)).astype(np.int64)
    counts = np.bincount(part, minlength=1 << fb)
    worst = max(probes_per_insert(slot[part == f]) for f in np.argsort(-counts)[:4])
    return counts.max() / counts.mean(), worst


N = 1 << 16
FB = 4  # 16 partitions of 4096 keys: a third of the table, as at the bench size


@pytest.mark.parametrize("name,keys", [
    ("dense", np.arange(1, N + 1)),
    ("dense, offset", np.arange(N) + 10**9),
    ("x 2^16", np.arange(N) << 16),
    ("x 2^20", np.arange(N) << 20),
    ("x 2^32", np.arange(N) << 32),
    ("x 2^40", np.arange(N) << 40),
    ("x 1000", np.arange(N) * 1000),
    ("x 987", np.arange(N) * 987),
    ("x 1597", np.arange(N) * 1597),
    ("x 4181", np.arange(N) * 4181),
    ("(a << 32) | b", (np.arange(N) // 256 << 32) | (np.arange(N) % 256)),
    ("(a << 20) | b", (np.arange(N) // 256 << 20) | (np.arange(N) % 256)),
])
def test_strided_keys_probe_like_random(name, keys):
    balance, probes = worst_partition(keys, FB)
    assert balance < 1.1, (name, balance)
    assert probes < 1.6, (name, probes)


def test_dense_range_spreads_evenly():
    # Consecutive keys: every partition within one key of the mean, and
    # (almost) no slot shared inside a partition.
    balance, probes = worst_partition(np.arange(1, N + 1), FB)
    assert balance < 1.01 and probes < 1.05


def test_random_keys_reference_point():
    rng = np.random.default_rng(3)
    balance, probes = worst_partition(rng.integers(0, 1 << 62, N), FB)
    assert balance < 1.15 and probes < 1.6
