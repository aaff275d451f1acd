"""Named single-operator cases on seeded device data, one per kernel family.

Each case builds its inputs on the device, runs the operator `--reps`
times through the C ABI and checks a size-independent property of the
result, so that a profiler can be pointed at one kernel of one small,
known workload:

  python pythia-core_b200/kernel_cases.py <case> [--shift S] [--reps K]

Inputs are sized to exceed the 126 MB L2 while staying a few GB on the
device.  Cases and the kernels they launch:

  radix      R 2^24 x S 2^27 PK-FK radix join      rj_hist, rj_partition, rj_join
  direct     R 2^20 x S 2^24 join, one HBM table    dj_clear, dj_build, dj_probe
  groupby16  2^26 (int64, int64), G = 16 / 1024 / 2^16   gbr_tiny / gbr_direct / gbr_part
  groupby-zipf  2^26 tuples, G = 2^16, Zipf(1.0) ids     rj_hist, rj_partition, gbr_part
  composite  2^25 (int32, int32, int64), G = 2^16    groupby_kernel
  partition  2^25 tuples, exactrange, fan-out 64     pt_hist, pt_scatter
  sort       2^24 tuples                            rs_hist, rs_scatter
  mpsm       R 2^22 x S 2^24, sampled or learned splitters   mp16 path (aggregate sink)
  mpsm-mat   R 2^20 x S 2^22, materialised          mp_tile_sort, mp_merge, mp_join
  cdf        2^21-key sample, 1024 leaves           cdf training kernels
  batch      64 fragments, builds 2^12..2^18        batch_kernel
"""
import argparse
import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

import pyg  # noqa: E402

I64, I32 = pyg.INT64, pyg.INT32


def pkfk(torch, ctx, nR, nS, theta=0.0, seed=1):
    R = torch.empty(nR * 2, dtype=torch.int64, device="cuda")
    S = torch.empty(nS * 2, dtype=torch.int64, device="cuda")
    ctx.gen_pk(R, nR, 7, seed)
    ctx.gen_fk(S, nS, nR, theta, seed, 1 << 20, seed + 1)
    return R, S


def expect_pkfk(S, nS):
    Sv = S.view(nS, 2)
    return int((Sv[:, 0] * 7 + Sv[:, 1]).sum().item()) & 0xFFFFFFFFFFFFFFFF


def case_join(torch, ctx, a, algo, nR, nS):
    R, S = pkfk(torch, ctx, nR, nS, a.theta)
    Rr, Sr = pyg.Rel(R, nR, [I64, I64]), pyg.Rel(S, nS, [I64, I64])
    want = expect_pkfk(S, nS)
    for _ in range(a.reps):
        cnt, (sb, sp) = ctx.hashjoin_agg(Rr, [0], Sr, [0], [(0, 1), (1, 1)], algo, a.bits)
        assert cnt == nS and (sb + sp) & 0xFFFFFFFFFFFFFFFF == want


def case_groupby16(torch, ctx, a):
    n = (1 << 26) >> a.shift
    for G in (16, 1024, 1 << 16):
        ids = torch.randint(0, G, (n,), device="cuda")
        A = torch.stack([ids, torch.randint(0, 1 << 20, (n,), device="cuda")], 1).contiguous().view(-1)
        out = torch.empty(G * 3, dtype=torch.int64, device="cuda")
        for _ in range(a.reps):
            rc, g = ctx.groupby(pyg.Rel(A, n, [I64, I64]), [0], 3, 1, True, G, out, G)
            assert rc == 0 and int(out[: 3 * g].view(g, 3)[:, 2].sum().item()) == n


def case_groupby_zipf(torch, ctx, a):
    """2^26 (int64 id, int64 value), ids Zipf(1.0) over G = 2^16."""
    n, G = (1 << 26) >> a.shift, 1 << 16
    w = torch.arange(1, G + 1, dtype=torch.float64, device="cuda").pow(-1.0)
    ids = torch.cat([torch.multinomial(w / w.sum(), min(n, 1 << 24), replacement=True)
                     for _ in range(max(1, n >> 24))])[:n]
    A = torch.stack([ids, torch.randint(0, 1 << 20, (n,), device="cuda")], 1).contiguous().view(-1)
    out = torch.empty(G * 3, dtype=torch.int64, device="cuda")
    for _ in range(a.reps):
        rc, g = ctx.groupby(pyg.Rel(A, n, [I64, I64]), [0], 3, 1, True, G, out, G)
        assert rc == 0 and int(out[: 3 * g].view(g, 3)[:, 2].sum().item()) == n


def case_composite(torch, ctx, a):
    n, G = (1 << 25) >> a.shift, 1 << 16
    g = torch.randint(0, G, (n,), device="cuda")
    raw = torch.empty(n * 2, dtype=torch.int64, device="cuda")
    v = raw.view(n, 2)
    v[:, 1] = torch.randint(0, 1 << 20, (n,), device="cuda")
    k32 = raw.view(torch.int32).view(n, 4)
    k32[:, 0] = (g >> 8).to(torch.int32)
    k32[:, 1] = (g & 255).to(torch.int32)
    rel = pyg.Rel(raw, n, [I32, I32, I64])
    out = torch.empty(G * 4, dtype=torch.int64, device="cuda")
    for _ in range(a.reps):
        rc, ng = ctx.groupby(rel, [0, 1], 3, 2, True, G, out, G)
        assert rc == 0 and ng <= G


def case_partition(torch, ctx, a):
    n = (1 << 25) >> a.shift
    R, _ = pkfk(torch, ctx, n, 1)
    out = torch.empty_like(R)
    for _ in range(a.reps):
        offs = ctx.partition(pyg.Rel(R, n, [I64, I64]), 0, pyg.SPLIT_EXACTRANGE, 64, out, 1, n)
        assert offs[-1] == n


def case_sort(torch, ctx, a):
    n = (1 << 24) >> a.shift
    R, _ = pkfk(torch, ctx, n, 1)
    out = torch.empty_like(R)
    for _ in range(a.reps):
        ctx.sort(pyg.Rel(R, n, [I64, I64]), 0, out)
        k = out.view(n, 2)[:, 0]
        assert bool((k[1:] >= k[:-1]).all().item())


def case_mpsm(torch, ctx, a, materialize):
    nR, nS = ((1 << 20, 1 << 22) if materialize else (1 << 22, 1 << 24))
    nR, nS = nR >> a.shift, nS >> a.shift
    R, S = pkfk(torch, ctx, nR, nS, a.theta)
    Rr, Sr = pyg.Rel(R, nR, [I64, I64]), pyg.Rel(S, nS, [I64, I64])
    kind = pyg.MPSM_LEARNED if a.splitter == "learned" else pyg.MPSM_SAMPLED
    opts = ctx.mpsm_opts(kind, 1024, 0.01, 1024)
    if materialize:
        out = torch.empty(nS * 2, dtype=torch.int64, device="cuda")
        for _ in range(a.reps):
            rc, cnt = ctx.mpsm_join_materialize(Rr, 0, Sr, 0, [(0, 1), (1, 1)], opts, out, nS)
            assert rc == 0 and cnt == nS
    else:
        want = expect_pkfk(S, nS)
        for _ in range(a.reps):
            cnt, (sb, sp), _ = ctx.mpsm_join_agg(Rr, 0, Sr, 0, [(0, 1), (1, 1)], opts)
            assert cnt == nS and (sb + sp) & 0xFFFFFFFFFFFFFFFF == want


def case_cdf(torch, ctx, a):
    n = (1 << 21) >> a.shift
    keys = torch.sort(torch.randint(-(1 << 40), 1 << 40, (n,), device="cuda"))[0]
    for _ in range(a.reps):
        o = pyg.pyg_cdf_train_opts(1024, 50, 0.01, 1)
        h = C.c_void_p()
        pyg.check(pyg.lib().pyg_cdf_train(ctx.h, keys.data_ptr(), n, C.byref(o), C.byref(h)))
        sp = np.zeros(1023, dtype=np.int64)
        pyg.check(pyg.lib().pyg_cdf_splitters(ctx.h, h, 1024, sp.ctypes.data_as(C.POINTER(C.c_int64))))
        assert bool(np.all(np.diff(sp) >= 0))
        pyg.lib().pyg_cdf_free(ctx.h, h)


def case_batch(torch, ctx, a):
    rng = np.random.default_rng(9)
    pairs, keep = [], []
    for i in range(64):
        nb = max(16, int(2 ** rng.uniform(12, 18)) >> a.shift)
        npr = nb * int(rng.integers(4, 33))
        R, S = pkfk(torch, ctx, nb, npr, 0.0, 100 + i)
        keep += [R, S]
        pairs.append((R, nb, S, npr))
    frags = ctx.fragments(pairs)
    b = ctx.batch_create(frags)
    try:
        for _ in range(a.reps):
            rc, c, s, lat = ctx.batch_run(b, len(pairs))
            assert rc == 0 and all(int(c[i]) == pairs[i][3] for i in range(len(pairs)))
    finally:
        ctx.batch_free(b)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("case", choices=["radix", "direct", "groupby16", "groupby-zipf", "composite", "partition", "sort", "mpsm",
                                     "mpsm-mat", "cdf", "batch"])
    ap.add_argument("--shift", type=int, default=0, help="shrink the inputs by 2^shift")
    ap.add_argument("--reps", type=int, default=2)
    ap.add_argument("--theta", type=float, default=0.0)
    ap.add_argument("--bits", type=int, default=0, help="radix: log2 partition fan-out (0 = automatic)")
    ap.add_argument("--splitter", default="sampled", choices=["sampled", "learned"],
                    help="mpsm: range splitters (learned: the model's own bins)")
    a = ap.parse_args()
    import torch

    torch.manual_seed(5)
    ctx = pyg.Ctx(0)
    try:
        if a.case == "radix":
            case_join(torch, ctx, a, pyg.JOIN_RADIX, (1 << 24) >> a.shift, (1 << 27) >> a.shift)
        elif a.case == "direct":
            case_join(torch, ctx, a, pyg.JOIN_DIRECT, (1 << 20) >> a.shift, (1 << 24) >> a.shift)
        elif a.case == "groupby16":
            case_groupby16(torch, ctx, a)
        elif a.case == "groupby-zipf":
            case_groupby_zipf(torch, ctx, a)
        elif a.case == "composite":
            case_composite(torch, ctx, a)
        elif a.case == "partition":
            case_partition(torch, ctx, a)
        elif a.case == "sort":
            case_sort(torch, ctx, a)
        elif a.case in ("mpsm", "mpsm-mat"):
            case_mpsm(torch, ctx, a, a.case == "mpsm-mat")
        elif a.case == "cdf":
            case_cdf(torch, ctx, a)
        else:
            case_batch(torch, ctx, a)
        torch.cuda.synchronize()
    finally:
        ctx.close()
    print("case", a.case, "ok")


if __name__ == "__main__":
    main()
