"""One-shot join + aggregate (pyg_hashjoin_agg): the hash-ordered radix
path and the direct path must give bit-identical count and sums, equal to
the oracle; plus the streamed host-input probe."""
import numpy as np
import pytest

import oracle as O
import pyg
from util import I64, dev_rel, host_rel, struct

pytestmark = pytest.mark.gpu
PROJ = [(0, 1), (1, 1)]


def zipf_keys(rng, n, keys, theta):
    if theta == 0:
        return keys[rng.integers(0, len(keys), n)]
    w = np.arange(1, len(keys) + 1, dtype=np.float64) ** -theta
    c = np.cumsum(w)
    c /= c[-1]
    return keys[np.minimum(np.searchsorted(c, rng.random(n)), len(keys) - 1)]


@pytest.mark.parametrize("stride", [1 << 16, 1 << 32, 1597, 1000])
def test_radix_strided_keys(ctx, torch_cuda, stride):
    """Keys on a regular stride (multiples of 2^16, 2^32, a Fibonacci number,
    1000): the patterns a plain multiplicative hash handles worst.  Every
    probe key is a build key (PK-FK), so the result is known in closed form:
    count = |S|, sums = the build payloads of the drawn rows and the probe
    payloads (below 2^60: no wrap-around).  The oracle is not used here: it
    buckets by the key's low bits, as the reference does, and walks one
    chain of every build key for strides of 2^16 and more."""
    rng = np.random.default_rng(stride % 1000003)
    n, m = 1 << 16, 1 << 20
    k = rng.permutation(n).astype(np.int64) * stride
    rp, idx, sp = rng.integers(0, 1 << 40, n), rng.integers(0, n, m), rng.integers(0, 1 << 40, m)
    R = struct([k, rp], [I64, I64])
    S = struct([k[idx], sp], [I64, I64])
    want = (m, [int(rp[idx].sum()), int(sp.sum())])
    got = ctx.hashjoin_agg(dev_rel(torch_cuda, R, [I64, I64]), [0], dev_rel(torch_cuda, S, [I64, I64]), [0], PROJ,
                           pyg.JOIN_RADIX, 4)
    assert got == want


@pytest.mark.parametrize("theta", [0.0, 0.75, 1.25])
@pytest.mark.parametrize("bits", [0, 3, 8, 12])
def test_radix_equals_direct_equals_oracle(ctx, torch_cuda, theta, bits):
    rng = np.random.default_rng(int(theta * 100) + bits)
    n, m = 1 << 17, 1 << 21
    k = rng.permutation(n).astype(np.int64) * 5 + 11
    R = struct([k, rng.integers(-(1 << 60), 1 << 60, n)], [I64, I64])
    fk = zipf_keys(rng, m, k, theta) + (rng.random(m) < 0.05)  # a few misses
    S = struct([fk, rng.integers(-(1 << 60), 1 << 60, m)], [I64, I64])
    Rd, Sd = dev_rel(torch_cuda, R, [I64, I64]), dev_rel(torch_cuda, S, [I64, I64])
    want = O.hashjoin_agg(R, [I64, I64], [0], S, [I64, I64], [0], PROJ)
    got_r, st = ctx.hashjoin_agg(Rd, [0], Sd, [0], PROJ, pyg.JOIN_RADIX, bits, stats=True)
    assert st.algorithm == pyg.JOIN_RADIX
    got_d = ctx.hashjoin_agg(Rd, [0], Sd, [0], PROJ, pyg.JOIN_DIRECT)
    assert got_r == want and got_d == want


def test_radix_sentinel_keys_and_duplicates(ctx, torch_cuda):
    rng = np.random.default_rng(3)
    mn = np.iinfo(np.int64).min
    n, m = 50000, 400000
    k = rng.integers(-1000, 1000, n)
    k[:7] = mn
    R = struct([k, rng.integers(0, 1 << 40, n)], [I64, I64])
    fk = rng.integers(-1100, 1100, m)
    fk[::1000] = mn
    S = struct([fk, rng.integers(0, 1 << 40, m)], [I64, I64])
    Rd, Sd = dev_rel(torch_cuda, R, [I64, I64]), dev_rel(torch_cuda, S, [I64, I64])
    want = O.hashjoin_agg(R, [I64, I64], [0], S, [I64, I64], [0], PROJ)
    for proj in (PROJ, [(1, 1), (0, 1)], [(1, 1)], [(0, 1)], []):
        w = O.hashjoin_agg(R, [I64, I64], [0], S, [I64, I64], [0], proj)
        assert ctx.hashjoin_agg(Rd, [0], Sd, [0], proj, pyg.JOIN_RADIX, 6) == w
    assert ctx.hashjoin_agg(Rd, [0], Sd, [0], PROJ, pyg.JOIN_RADIX) == want


@pytest.mark.parametrize("case", ["unique", "repeated", "many_sentinels", "empty_probe", "empty_build"])
def test_direct_one_shot_join(ctx, torch_cuda, case):
    """The one-shot direct join (clear, build, probe; the probe reads the
    build's flags on the device) against the oracle, for every projection
    over {B$1, P$1}.  Repeated build keys and more empty-marker build keys
    than its side list holds make the probe stand down and the general path
    answer; the result is the same."""
    rng = np.random.default_rng(len(case))
    mn = np.iinfo(np.int64).min
    n, m = 1 << 16, 1 << 20
    k = rng.permutation(n).astype(np.int64) * 11 - 5000
    if case == "repeated":
        k[: n // 3] = k[n // 3: 2 * (n // 3)]
    if case == "many_sentinels":
        k[:2000] = mn
    R = struct([k, rng.integers(-(1 << 62), 1 << 62, n)], [I64, I64])
    fk = rng.choice(k, m) + (rng.random(m) < 0.1)
    fk[::777] = mn
    S = struct([fk, rng.integers(-(1 << 62), 1 << 62, m)], [I64, I64])
    if case == "empty_probe":
        S = S[:0]
    if case == "empty_build":
        R = R[:0]
    Rd, Sd = dev_rel(torch_cuda, R, [I64, I64]), dev_rel(torch_cuda, S, [I64, I64])
    for proj in (PROJ, [(1, 1), (0, 1)], [(1, 1)], [(0, 1)], []):
        want = O.hashjoin_agg(R, [I64, I64], [0], S, [I64, I64], [0], proj, buckets=n)
        for _ in range(2):  # a second call reuses the context's table
            assert ctx.hashjoin_agg(Rd, [0], Sd, [0], proj, pyg.JOIN_DIRECT) == want


@pytest.mark.parametrize("bits", [4, 9, 11])
def test_radix_duplicate_build_keys(ctx, torch_cuda, bits):
    """Repeated build keys switch the join to its counted slot layout (and
    smaller build chunks); the result must not change."""
    rng = np.random.default_rng(bits)
    n, m = 1 << 18, 1 << 21
    k = rng.integers(0, 1 << 16, n)  # ~4 copies per key
    R = struct([k, rng.integers(-(1 << 50), 1 << 50, n)], [I64, I64])
    S = struct([rng.integers(0, (1 << 16) + 500, m), rng.integers(-(1 << 50), 1 << 50, m)], [I64, I64])
    want = O.hashjoin_agg(R, [I64, I64], [0], S, [I64, I64], [0], PROJ)
    got, st = ctx.hashjoin_agg(dev_rel(torch_cuda, R, [I64, I64]), [0], dev_rel(torch_cuda, S, [I64, I64]), [0], PROJ,
                               pyg.JOIN_RADIX, bits, stats=True)
    assert st.radix_bits == bits and got == want


@pytest.mark.parametrize("bits", [2, 10, 15])
def test_radix_partition_shapes(ctx, torch_cuda, bits):
    """Build partitions larger than one shared-memory table (bits 2: chunked
    build side), two partition passes (bits 10, 15), and one hot probe key
    that spreads over many probe chunks."""
    rng = np.random.default_rng(100 + bits)
    n, m = 1 << 16, 1 << 22
    k = rng.permutation(n).astype(np.int64) - (n // 2)
    R = struct([k, rng.integers(-(1 << 62), 1 << 62, n)], [I64, I64])
    fk = k[rng.integers(0, n, m)]
    fk[: m // 3] = k[7]  # a third of the probe side is one key
    fk[::97] = n + 5     # misses
    S = struct([fk, rng.integers(-(1 << 62), 1 << 62, m)], [I64, I64])
    want = O.hashjoin_agg(R, [I64, I64], [0], S, [I64, I64], [0], PROJ)
    got = ctx.hashjoin_agg(dev_rel(torch_cuda, R, [I64, I64]), [0], dev_rel(torch_cuda, S, [I64, I64]), [0], PROJ,
                           pyg.JOIN_RADIX, bits)
    assert got == want


def test_radix_sampled_probe_layout(ctx, torch_cuda):
    """A probe side of at least 2^25 tuples with two partition passes is laid
    out from a sample; the per-partition counts the passes reach are exact."""
    rng = np.random.default_rng(21)
    n, m = 1 << 17, (1 << 25) + 12345
    k = rng.permutation(n).astype(np.int64) * 3 + 1
    R = struct([k, rng.integers(-(1 << 62), 1 << 62, n)], [I64, I64])
    S = struct([zipf_keys(rng, m, k, 0.9), rng.integers(-(1 << 62), 1 << 62, m)], [I64, I64])
    want = O.hashjoin_agg(R, [I64, I64], [0], S, [I64, I64], [0], PROJ)
    got, st = ctx.hashjoin_agg(dev_rel(torch_cuda, R, [I64, I64]), [0], dev_rel(torch_cuda, S, [I64, I64]), [0], PROJ,
                               pyg.JOIN_RADIX, 11, stats=True)
    assert got == want and st.overflow_tuples == 0 and st.padded_tuples > 0


def test_radix_sample_misjudged_redoes_exactly(ctx, torch_cuda):
    """Every sampled probe tuple (every second one) carries the same key, so
    the sample sizes all other partitions' regions near zero; the passes
    report the overflow and the probe side is redone from an exact
    histogram."""
    rng = np.random.default_rng(22)
    n, m = 1 << 16, 1 << 25
    k = rng.permutation(n).astype(np.int64) + 1000
    R = struct([k, rng.integers(0, 1 << 40, n)], [I64, I64])
    fk = k[rng.integers(0, n, m)]
    fk[0::2] = k[5]
    S = struct([fk, rng.integers(0, 1 << 40, m)], [I64, I64])
    want = O.hashjoin_agg(R, [I64, I64], [0], S, [I64, I64], [0], PROJ)
    got, st = ctx.hashjoin_agg(dev_rel(torch_cuda, R, [I64, I64]), [0], dev_rel(torch_cuda, S, [I64, I64]), [0], PROJ,
                               pyg.JOIN_RADIX, 10, stats=True)
    assert got == want and st.overflow_tuples == 1


@pytest.mark.parametrize("bits", [0, 6, 12, 16])
@pytest.mark.parametrize("case", ["both", "build_only", "probe_only", "near_min"])
def test_radix_packed_intermediates(ctx, torch_cuda, bits, case):
    """Partition passes write 8-byte frame-of-reference words when a
    relation's key and payload ranges each fit in 32 bits, and 16-byte
    tuples otherwise, per relation.  Every combination, at one pass (6
    bits), two passes (12, 16 bits) and the automatic choice, must equal the
    oracle bit for bit.  near_min puts the keys just above INT64_MIN (the
    table's empty marker among them), so the frame arithmetic wraps."""
    rng = np.random.default_rng(bits * 7 + len(case))
    n, m = 1 << 17, 1 << 21
    mn = np.iinfo(np.int64).min
    base = mn if case == "near_min" else -(1 << 35)
    k = rng.permutation(n).astype(np.int64) * 3 + base
    small = lambda c: rng.integers(-(1 << 31), 1 << 31, c)  # noqa: E731
    large = lambda c: rng.integers(-(1 << 62), 1 << 62, c)  # noqa: E731
    R = struct([k, large(n) if case == "probe_only" else small(n)], [I64, I64])
    fk = zipf_keys(rng, m, k, 0.8) + (rng.random(m) < 0.05)  # some misses (keys are 3 apart)
    S = struct([fk, large(m) if case == "build_only" else small(m)], [I64, I64])
    want = O.hashjoin_agg(R, [I64, I64], [0], S, [I64, I64], [0], PROJ, buckets=n)
    got, st = ctx.hashjoin_agg(dev_rel(torch_cuda, R, [I64, I64]), [0], dev_rel(torch_cuda, S, [I64, I64]), [0], PROJ,
                               pyg.JOIN_RADIX, bits, stats=True)
    assert got == want
    assert st.build_packed == (case != "probe_only")
    assert st.probe_packed == (case != "build_only")


@pytest.mark.parametrize("bits", [6, 12])
def test_radix_shared_frame_with_repeated_build_keys(ctx, torch_cuda, bits):
    """Both relations packed in one key frame take the 32-bit-offset join;
    a repeated build key there hands the join to the counted kernel, which
    decodes the packed words.  Same result as the oracle."""
    rng = np.random.default_rng(50 + bits)
    n, m = 1 << 17, 1 << 21
    k = rng.integers(1000, 1000 + (1 << 15), n)  # about 4 copies per key
    R = struct([k, rng.integers(0, 1 << 30, n)], [I64, I64])
    S = struct([rng.integers(900, 1100 + (1 << 15), m), rng.integers(0, 1 << 30, m)], [I64, I64])
    want = O.hashjoin_agg(R, [I64, I64], [0], S, [I64, I64], [0], PROJ, buckets=n)
    got, st = ctx.hashjoin_agg(dev_rel(torch_cuda, R, [I64, I64]), [0], dev_rel(torch_cuda, S, [I64, I64]), [0], PROJ,
                               pyg.JOIN_RADIX, bits, stats=True)
    assert got == want and st.build_packed == 1 and st.probe_packed == 1


def test_radix_packed_frame_missed_redoes(ctx, torch_cuda):
    """A probe side of 2^25 tuples is laid out from a strided sample, which
    also gives the frame of its packed words.  One payload that no sampled
    tuple shows lies far outside that frame: the first pass flags it, and
    the probe side is redone from an exact histogram (whose exact ranges no
    longer fit 32 bits, so the redo is unpacked).  Same result as the
    oracle."""
    rng = np.random.default_rng(23)
    n, m = 1 << 16, 1 << 25
    k = rng.permutation(n).astype(np.int64) + 1
    R = struct([k, k * 7], [I64, I64])
    pay = rng.integers(0, 1 << 20, m)
    pay[1] = 1 << 45  # index 1: between two sampled tuples
    S = struct([k[rng.integers(0, n, m)], pay], [I64, I64])
    want = O.hashjoin_agg(R, [I64, I64], [0], S, [I64, I64], [0], PROJ, buckets=n)
    got, st = ctx.hashjoin_agg(dev_rel(torch_cuda, R, [I64, I64]), [0], dev_rel(torch_cuda, S, [I64, I64]), [0], PROJ,
                               pyg.JOIN_RADIX, 12, stats=True)
    assert got == want
    assert st.overflow_tuples == 1 and st.build_packed == 1 and st.probe_packed == 0


def test_empty_sides(ctx, torch_cuda):
    R = struct([np.arange(100, dtype=np.int64)] * 2, [I64, I64])
    E = R[:0]
    for a, b in ((R, E), (E, R), (E, E)):
        got = ctx.hashjoin_agg(dev_rel(torch_cuda, a, [I64, I64]), [0], dev_rel(torch_cuda, b, [I64, I64]), [0], PROJ,
                               pyg.JOIN_RADIX, 4)
        assert got == (0, [0, 0])


def test_host_probe_streams_in_chunks(ctx, torch_cuda):
    """Host-resident probe relation larger than one 2^25-tuple staging chunk
    (the end-to-end path): same result as the oracle."""
    rng = np.random.default_rng(8)
    n, m = 1 << 16, (1 << 25) + 12345
    k = rng.permutation(n).astype(np.int64)
    R = struct([k, k * 3], [I64, I64])
    S = struct([rng.integers(0, n + 100, m), rng.integers(0, 1 << 20, m)], [I64, I64])
    got = ctx.hashjoin_agg(host_rel(R, [I64, I64]), [0], host_rel(S, [I64, I64]), [0], PROJ, pyg.JOIN_AUTO)
    assert got == O.hashjoin_agg(R, [I64, I64], [0], S, [I64, I64], [0], PROJ, buckets=n)
