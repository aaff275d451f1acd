"""Learned CDF splitter: GPU forward/backward kernels vs the fp64 CPU
oracle, training quality, splitter validity, and the gain over equal-width
ranges (the reference's ExactRangeValueHasher) at the same fan-out."""
import ctypes as C

import numpy as np
import pytest

import cdf_oracle
import pyg

pytestmark = pytest.mark.gpu


def zipf_sample(rng, n, N, theta, perm=None):
    w = np.arange(1, N + 1, dtype=np.float64) ** -theta
    c = np.cumsum(w)
    c /= c[-1]
    r = np.minimum(np.searchsorted(c, rng.random(n)), N - 1)
    return (perm[r] if perm is not None else r + 1).astype(np.int64)


def train(ctx, torch, keys, leaves=64, epochs=300, lr=0.05):
    d = torch.from_numpy(keys).cuda()
    o = pyg.pyg_cdf_train_opts(leaves, epochs, lr, 1)
    h = C.c_void_p()
    pyg.check(pyg.lib().pyg_cdf_train(ctx.h, d.data_ptr(), keys.shape[0], C.byref(o), C.byref(h)))
    return h.value


def splitters(ctx, model, fan):
    out = np.zeros(fan - 1, dtype=np.int64)
    pyg.check(pyg.lib().pyg_cdf_splitters(ctx.h, model, fan, out.ctypes.data_as(C.POINTER(C.c_int64))))
    return out


def params(ctx, model, L):
    p = np.zeros(2 + 2 * L, dtype=np.float32)
    lo, sc = C.c_double(), C.c_double()
    pyg.check(pyg.lib().pyg_cdf_params(ctx.h, model, p.ctypes.data_as(C.POINTER(C.c_float)), p.shape[0],
                                       C.byref(lo), C.byref(sc)))
    return p, lo.value, sc.value


def gpu_loss_grad(ctx, torch, sorted_keys, L, p, lo, sc):
    d = torch.from_numpy(sorted_keys).cuda()
    g = np.zeros(2 + 2 * L, dtype=np.float32)
    loss = C.c_double()
    pyg.check(pyg.lib().pyg_cdf_loss_grad(ctx.h, d.data_ptr(), sorted_keys.shape[0], L,
                                          p.ctypes.data_as(C.POINTER(C.c_float)), lo, sc, C.byref(loss),
                                          g.ctypes.data_as(C.POINTER(C.c_float))))
    return loss.value, g


@pytest.mark.parametrize("theta", [0.0, 1.0])
def test_gradients_match_cpu_oracle(ctx, torch_cuda, theta):
    rng = np.random.default_rng(1)
    keys = np.sort(zipf_sample(rng, 20000, 100000, theta) * 37 if theta else rng.integers(0, 1 << 40, 20000))
    L = 16
    lo, sc = float(keys[0]), 1.0 / float(keys[-1] - keys[0])
    p = np.concatenate([[0.9, 0.05], np.tile([0.8, 0.1], L)]).astype(np.float32)
    p += rng.normal(0, 0.05, p.shape).astype(np.float32)
    p[0::2] = np.abs(p[0::2])
    l_gpu, g_gpu = gpu_loss_grad(ctx, torch_cuda, keys, L, p, lo, sc)
    l_cpu, g_cpu = cdf_oracle.loss_grad(keys, L, p, lo, sc)
    assert abs(l_gpu - l_cpu) <= 1e-9 + 1e-6 * abs(l_cpu)
    np.testing.assert_allclose(g_gpu, g_cpu, rtol=1e-4, atol=1e-7)


@pytest.mark.parametrize("theta", [0.0, 1.0, 1.5])
def test_trained_model_splitters_beat_equal_width(ctx, torch_cuda, theta):
    """Range splitters from the trained model (1024 leaves, 1% sample) give
    far lower max-partition imbalance than the reference's equal-width
    ranges on skewed keys, and stay close to exact sample quantiles."""
    rng = np.random.default_rng(3)
    N = 1 << 20
    perm = np.sort(rng.choice(1 << 40, N, replace=False)).astype(np.int64)  # skewed *values*
    keys = zipf_sample(rng, 1 << 22, N, theta, perm)
    sample = keys[rng.integers(0, keys.shape[0], keys.shape[0] // 100)]
    fan = 256
    model = train(ctx, torch_cuda, sample, leaves=1024, epochs=200)
    try:
        spl = splitters(ctx, model, fan)
        assert np.all(np.diff(spl) >= 0)
        learned = cdf_oracle.imbalance(keys, spl)
        mn, mx = int(keys.min()), int(keys.max())
        br = (mx - mn + fan) // fan
        equal = cdf_oracle.imbalance(keys, mn + br * np.arange(1, fan))
        q = np.sort(sample)[np.ceil(np.arange(1, fan) * len(sample) / fan).astype(np.int64)]
        sampled = cdf_oracle.imbalance(keys, q)
        # A single key heavier than 1/fan of the input bounds every splitter.
        heavy = np.bincount(np.searchsorted(perm, keys)).max() / (len(keys) / fan)
        assert learned <= max(1.35 * sampled, heavy + 0.35), (learned, sampled, heavy)
        assert learned < equal / 2 or equal < 1.5, (learned, equal)
        # training reduced the loss well below the untrained identity model
        srt = np.sort(sample)
        p, lo, sc = params(ctx, model, 1024)
        trained_loss, _ = gpu_loss_grad(ctx, torch_cuda, srt, 1024, p, lo, sc)
        p0 = np.concatenate([[1.0, 0.0], np.tile([1.0, 0.0], 1024)]).astype(np.float32)
        init_loss, _ = gpu_loss_grad(ctx, torch_cuda, srt, 1024, p0, lo, sc)
        assert trained_loss < init_loss
    finally:
        pyg.lib().pyg_cdf_free(ctx.h, model)


def test_predict_and_distinct_estimate(ctx, torch_cuda):
    torch = torch_cuda
    rng = np.random.default_rng(4)
    keys = rng.integers(0, 1 << 16, 200000).astype(np.int64)
    model = train(ctx, torch, keys[:20000], leaves=64)
    try:
        kd = torch.from_numpy(np.sort(keys)).cuda()
        out = torch.empty(keys.shape[0], dtype=torch.float32, device="cuda")
        pyg.check(pyg.lib().pyg_cdf_predict(ctx.h, model, kd.data_ptr(), keys.shape[0], out.data_ptr()))
        ctx.sync()
        pr = out.cpu().numpy()
        assert np.all(np.diff(pr) >= -1e-6)  # monotone
        assert np.abs(pr - np.arange(keys.shape[0]) / keys.shape[0]).max() < 0.02
        est = C.c_int64()
        pyg.check(pyg.lib().pyg_cdf_estimate_distinct(ctx.h, model, keys.shape[0], C.byref(est)))
        true = np.unique(keys).shape[0]
        assert 0.5 * true <= est.value <= 2.0 * true
    finally:
        pyg.lib().pyg_cdf_free(ctx.h, model)


def test_sampled_splitters_are_quantiles(ctx, torch_cuda):
    rng = np.random.default_rng(5)
    keys = rng.integers(-1000000, 1000000, 100000).astype(np.int64)
    d = torch_cuda.from_numpy(keys).cuda()
    fan = 100
    out = np.zeros(fan - 1, dtype=np.int64)
    pyg.check(pyg.lib().pyg_sampled_splitters(ctx.h, d.data_ptr(), keys.shape[0], fan,
                                              out.ctypes.data_as(C.POINTER(C.c_int64))))
    srt = np.sort(keys)
    want = srt[np.ceil(np.arange(1, fan) * len(keys) / fan).astype(np.int64)]
    assert np.array_equal(out, want)


@pytest.mark.parametrize("theta", [1.0, 1.5])
def test_learned_vs_sampled_splitters_on_mpsm_join(ctx, torch_cuda, theta):
    """What the trained model gains over the method without it, on the
    skewed MPSM join: the same join result; a max-partition imbalance no
    worse than sample quantiles (heavy keys get ranges of their own); and a
    splitter cost (sample, sort, least-squares start, fine-tuning epochs)
    of a few milliseconds, not the tens a long gradient training took."""
    torch = torch_cuda
    nR, nS = 1 << 22, 1 << 24
    R = torch.empty(nR * 2, dtype=torch.int64, device="cuda")
    S = torch.empty(nS * 2, dtype=torch.int64, device="cuda")
    ctx.gen_pk(R, nR, 7, 31)
    ctx.gen_fk(S, nS, nR, theta, 31, 1 << 20, 32)
    Rr, Sr = pyg.Rel(R, nR, [pyg.INT64, pyg.INT64]), pyg.Rel(S, nS, [pyg.INT64, pyg.INT64])
    res = {}
    for kind in (pyg.MPSM_SAMPLED, pyg.MPSM_LEARNED):
        opts = ctx.mpsm_opts(kind, 4096, 0.01, 1024)
        ctx.mpsm_join_agg(Rr, 0, Sr, 0, [(0, 1), (1, 1)], opts)  # warm
        cnt, sums, st = ctx.mpsm_join_agg(Rr, 0, Sr, 0, [(0, 1), (1, 1)], opts)
        res[kind] = (cnt, sums, st.max_partition_imbalance, st.splitter_ms)
    assert res[pyg.MPSM_LEARNED][:2] == res[pyg.MPSM_SAMPLED][:2]
    assert res[pyg.MPSM_LEARNED][0] == nS
    assert res[pyg.MPSM_LEARNED][2] <= 1.05 * res[pyg.MPSM_SAMPLED][2] + 0.1
    assert res[pyg.MPSM_LEARNED][3] < 5.0, res


def model_bins(ctx, torch, model, fbits, keys):
    d = torch.from_numpy(np.ascontiguousarray(keys)).cuda()
    out = torch.empty(max(1, keys.shape[0]), dtype=torch.int32, device="cuda")
    pyg.check(pyg.lib().pyg_cdf_bins(ctx.h, model, fbits, d.data_ptr(), keys.shape[0], out.data_ptr()))
    ctx.sync()
    return out[: keys.shape[0]].cpu().numpy().view(np.uint32)


def model_bin_splitters(ctx, model, fbits):
    out = np.zeros((1 << fbits) - 1, dtype=np.int64)
    pyg.check(pyg.lib().pyg_cdf_bin_splitters(ctx.h, model, fbits, out.ctypes.data_as(C.POINTER(C.c_int64))))
    return out


def bin_sample(rng, dist):
    mn, mx = np.iinfo(np.int64).min, np.iinfo(np.int64).max
    if dist == "dense":
        return rng.permutation(1 << 20)[: 1 << 16].astype(np.int64) + 1
    if dist == "zipf":  # heavy keys scattered over a permuted domain
        return zipf_sample(rng, 1 << 17, 1 << 20, 1.2, rng.permutation(1 << 20).astype(np.int64) * 5)
    if dist == "wide":
        return rng.integers(-(1 << 62), 1 << 62, 1 << 16)
    if dist == "heavy":  # one key holds half the sample
        k = rng.integers(0, 1 << 30, 1 << 16)
        k[::2] = 777
        return k
    if dist == "tiny":
        return np.array([9, -3, 100, 4, 4], dtype=np.int64)
    if dist == "equal":
        return np.full(1000, 42, dtype=np.int64)
    # extremes: both ends of the int64 range in the sample
    k = rng.integers(-1000, 1000, 5000)
    k[:3] = [mn, mx, mn]
    return k


@pytest.mark.parametrize("fbits", [1, 7, 15])
@pytest.mark.parametrize("dist", ["dense", "zipf", "wide", "heavy", "tiny", "equal", "extremes"])
def test_model_bins_equal_a_search_of_their_splitters(ctx, torch_cuda, dist, fbits):
    """The MPSM join's learned partitioning computes each key's range from
    the model (pyg_cdf_bins) instead of searching splitters.  It must place
    every key exactly where a search of the model's splitters
    (pyg_cdf_bin_splitters) places it -- bin(k) = number of splitters <= k,
    the rule of the splitter-search path -- for the sample, its neighbours,
    keys outside the sample's range and the int64 extremes."""
    rng = np.random.default_rng(fbits * 7 + len(dist))
    sample = bin_sample(rng, dist).astype(np.int64)
    model = train(ctx, torch_cuda, sample, leaves=1024, epochs=1, lr=0.002)
    try:
        mn, mx = np.iinfo(np.int64).min, np.iinfo(np.int64).max
        lo, hi = int(sample.min()), int(sample.max())
        probe = [sample, np.array([mn, mx, mn + 1, mx - 1, 0, -1, 1], dtype=np.int64),
                 np.array([v for v in (lo - 1, lo, lo + 1, hi - 1, hi, hi + 1) if mn <= v <= mx], dtype=np.int64)]
        sub = sample[: 1 << 14]
        probe += [sub[sub < mx] + 1, sub[sub > mn] - 1]
        if hi - lo > 2:
            probe.append(rng.integers(lo, hi, 1 << 16, dtype=np.int64, endpoint=True))
        keys = np.concatenate(probe)
        spl = model_bin_splitters(ctx, model, fbits)
        assert np.all(np.diff(spl) >= 0)
        got = model_bins(ctx, torch_cuda, model, fbits, keys)
        want = np.searchsorted(spl, keys, side="right")
        assert np.array_equal(got, want), np.nonzero(got != want)[0][:10]
        if dist == "dense" and fbits == 7:
            # a model of a dense key range spreads the sample evenly
            counts = np.bincount(model_bins(ctx, torch_cuda, model, fbits, sample), minlength=1 << fbits)
            assert counts.max() <= 1.5 * sample.shape[0] / (1 << fbits)
    finally:
        pyg.lib().pyg_cdf_free(ctx.h, model)
