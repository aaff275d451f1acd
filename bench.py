"""Benchmark: radix-scale PK-FK hash join + aggregation on one B200.

Workload (the configuration the headline metric is quoted on): build R =
2^27 (int64 key, int64 payload) tuples with unique keys (a seeded
permutation of 1..2^27, payload = key * 7); probe S = 2^30 (int64 fk,
int64 payload) tuples, fk ~ Zipf(theta) over R's keys (theta = 0: uniform),
payload ~ U[0, 2^20).  Output: match count and the wrapped int64 checksum
sum(R.payload + S.payload) over the joined pairs.  A step = build the table
+ probe with the fused count/sum sink.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--theta T] [--impl pyg|reference]

Prints one JSON line (rank 0).  `value` is device-resident throughput
(inputs already in HBM); `e2e` goes through the same C-ABI calls with host
buffers (host->device copies inside the timed region); `cpu_baseline` is
the reference's own CPU engine on a bounded sample of the same workload.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "pythia-core_b200"))

N_BUILD = 1 << 27
N_PROBE = 1 << 30
VMAX = 1 << 20
SEED_KEYS, SEED_PROBE = 12345, 67890
METRIC = "join+agg tuples/sec (R 2^27 PK, S 2^30 FK, hash join + count + checksum, bit-exact)"
UNIT = "tuples/s"
# Bounded CPU sample: 1/16 of both relations, same key distribution.
CPU_SAMPLE_SHIFT = 4


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--theta", type=float, default=0.0)
    ap.add_argument("--impl", default="pyg", choices=["pyg", "reference"])
    ap.add_argument("--load-factor", type=float, default=0.5)
    ap.add_argument("--algo", default=None, choices=["radix", "direct", "auto"],
                    help="join algorithm (default: radix for the headline join, auto for join-small)")
    ap.add_argument("--radix-bits", type=int, default=0, help="log2 partition fan-out (0 = automatic)")
    ap.add_argument("--scale-shift", type=int, default=0, help="shrink both relations by 2^s (debug only)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--dist-mode", default="shuffle", choices=["shuffle", "replicas"],
                    help="join with N > 1 GPUs: the partitioned join with a hash shuffle over NCCL (default), or "
                         "independent replicas")
    ap.add_argument("--no-secondary", action="store_true",
                    help="join: skip the other configurations measured after the headline")
    ap.add_argument("--workload", default="join", choices=["join", "join-radix", "join-small", "groupby", "mpsm",
                                                          "batch"],
                    help="join: the headline configuration (default); join-radix: the same join at --theta as a "
                         "secondary line; the others measure the small join, group-by, MPSM sort-merge join and "
                         "batched-fragment configurations")
    ap.add_argument("--groups", type=int, default=1 << 16, help="groupby: group cardinality G")
    ap.add_argument("--zipf", action="store_true", help="groupby: Zipf(1.0) group ids instead of uniform")
    ap.add_argument("--splitter", default="learned", choices=["learned", "sampled", "exactrange"],
                    help="mpsm: range splitter")
    ap.add_argument("--fanout", type=int, default=4096, help="mpsm: range partitions")
    return ap.parse_args()


# ---------------------------------------------------------------- helpers

class Clocks:
    """Samples SM clocks and clock-event (throttle) reasons every 20 ms during
    the timed region through NVML (read-only queries), else nvidia-smi."""

    Q = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    NAMES = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
    BITS = [0x8, 0x40, 0x20, 0x4]  # NVML clocks-event reason masks, in NAMES order

    def __init__(self, index):
        self.index = index
        self.samples = []  # (sm_mhz, max_mhz, [active reason names])
        self._stop = threading.Event()
        self._t = None

    def _handle(self):
        try:
            import pynvml
            import torch

            pynvml.nvmlInit()
            pr = torch.cuda.get_device_properties(self.index)
            bus = f"{pr.pci_domain_id:08X}:{pr.pci_bus_id:02X}:{pr.pci_device_id:02X}.0"
            return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            return None

    def _run(self, nv):
        while not self._stop.is_set():
            try:
                if nv:
                    m, h = nv
                    sm = m.nvmlDeviceGetClockInfo(h, m.NVML_CLOCK_SM)
                    mx = m.nvmlDeviceGetMaxClockInfo(h, m.NVML_CLOCK_SM)
                    bits = m.nvmlDeviceGetCurrentClocksEventReasons(h)
                    self.samples.append((float(sm), float(mx), [n for n, b in zip(self.NAMES, self.BITS) if bits & b]))
                else:
                    r = subprocess.run(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                        "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                    f = [x.strip() for x in r.stdout.strip().split(",")]
                    if r.returncode == 0 and len(f) == 6:
                        self.samples.append((float(f[0]), float(f[1]),
                                             [n for n, v in zip(self.NAMES, f[2:]) if v == "Active"]))
            except Exception:
                pass
            self._stop.wait(0.02 if nv else 0.2)

    def __enter__(self):
        # NVML is imported and opened here, before the caller's timed region
        # starts: an import on the sampling thread holds the interpreter
        # lock in the middle of the timed steps (measured: 3.5 ms per step of
        # idle GPU over 20 steps of the headline join).
        nv = self._handle()
        self._t = threading.Thread(target=self._run, args=(nv,), daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        return {"sm_mhz": statistics.median(x[0] for x in self.samples),
                "sm_max_mhz": max(x[1] for x in self.samples),
                "reasons": sorted({n for x in self.samples for n in x[2]}), "samples": len(self.samples)}


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            j = json.load(f)
        return float(j["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def zipf_host(rng, n, nkeys, theta):
    """Ranks in [0, nkeys) with P(r) ~ (r+1)^-theta (uniform at theta 0)."""
    if theta == 0:
        return rng.integers(0, nkeys, n)
    w = np.arange(1, nkeys + 1, dtype=np.float64) ** (-theta)
    cdf = np.cumsum(w)
    cdf /= cdf[-1]
    return np.minimum(np.searchsorted(cdf, rng.random(n), side="right"), nkeys - 1)


def cpu_sample(theta, shift=CPU_SAMPLE_SHIFT, seed=7):
    """Host-generated sample with the bench's shapes scaled by 2^-shift."""
    rng = np.random.default_rng(seed)
    nR, nS = N_BUILD >> shift, N_PROBE >> shift
    perm = rng.permutation(nR).astype(np.int64) + 1
    R = np.empty((nR, 2), dtype=np.int64)
    R[:, 0] = perm
    R[:, 1] = perm * 7
    S = np.empty((nS, 2), dtype=np.int64)
    S[:, 0] = perm[zipf_host(rng, nS, nR, theta)]
    S[:, 1] = rng.integers(0, VMAX, nS)
    return R, S


def run_reference_cpu(theta, steps, shift=CPU_SAMPLE_SHIFT):
    """Times the reference engine (oracle/_ref/executequery) on the bounded
    sample with all host cores; falls back to the C oracle port."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import refrun
    R, S = cpu_sample(theta, shift)
    n_tuples = R.shape[0] + S.shape[0]
    cores = os.cpu_count() or 1
    sample = f"R=2^{27 - shift}, S=2^{30 - shift} (1/{1 << shift} of each relation), theta={theta}"
    if refrun.available():
        T = min(cores, 127)
        times = []
        with tempfile.TemporaryDirectory(dir=os.environ.get("PYG_TMP")) as d:
            dt = np.dtype([("c0", np.int64), ("c1", np.int64)])
            rf = refrun.write_rel(d, "R", R.view(dt).reshape(-1), T)
            sf = refrun.write_rel(d, "S", S.view(dt).reshape(-1), T)
            plan = refrun.plan_join_sum(T, rf, [2, 2], sf, [2, 2], [(0, 1), (1, 1)], 1, R.shape[0])
            for _ in range(steps):
                _, rt, _ = refrun.run(d, plan, timeout=900)
                times.append(rt)
        return {"kind": "reference", "cores": T, "sample": sample + f", executequery ResponseTimeInSec, {T} threads",
                "times": times, "tuples": n_tuples}
    import oracle as O
    dt = O.dtype_of([2, 2])
    Rs, Ss = R.view(dt).reshape(-1), S.view(dt).reshape(-1)
    times = []
    for _ in range(steps):
        t0 = time.perf_counter()
        O.hashjoin_agg(Rs, [2, 2], [0], Ss, [2, 2], [0], [(0, 1), (1, 1)], buckets=R.shape[0])
        times.append(time.perf_counter() - t0)
    return {"kind": "port", "cores": 1, "sample": sample + ", C oracle single thread", "times": times,
            "tuples": n_tuples}


def max_over_ranks(ms, dist, device):
    """The job's time: the slowest rank's device-timed milliseconds."""
    if dist is None:
        return ms
    import torch

    t = torch.tensor([ms], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def dist_env():
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    return rank, world, local


# ------------------------------------------------------------ reference arm

def main_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    steps = max(1, args.steps)
    for _ in range(args.warmup if args.warmup < 2 else 1):
        run_reference_cpu(args.theta, 1)
    r = run_reference_cpu(args.theta, steps)
    tot = sum(r["times"])
    value = r["tuples"] * len(r["times"]) / tot
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": steps,
            "warmup": args.warmup, "ms_per_step": 1000 * tot / len(r["times"]), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int64", "data": "synthetic (seeded, host-generated)",
            "impl": "reference",
            "config": {"workload": "hash join + count + checksum, R 2^27 PK / S 2^30 FK (CPU runs a 1/16 sample)",
                       "theta": args.theta},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": r["cores"], "kind": r["kind"],
                             "sample": r["sample"]},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ GPU arm

def main_dist(args):
    """N > 1, the partitioned join (pythia-core_b200/dist.py): rank r holds
    slice r of one global R of N x 2^27 unique keys and its own 2^30 probe
    tuples whose fks range over all N x 2^27 keys; each step shuffles both
    relations by key hash over NCCL, joins locally and all-reduces (count,
    sums).  Per-rank work is fixed (weak scaling); `value` counts the
    tuples of all ranks."""
    import datetime

    import torch
    import torch.distributed as dist

    import dist as pyg_dist
    import pyg

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    torch.cuda.set_stream(torch.cuda.Stream(local))
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device(f"cuda:{local}"))
    nR, nS = N_BUILD >> args.scale_shift, N_PROBE >> args.scale_shift
    ctx = pyg.Ctx(local)
    stream = torch.cuda.current_stream(local)
    G = torch.empty(nR * world * 2, dtype=torch.int64, device="cuda")
    ctx.gen_pk(G, nR * world, 7, SEED_KEYS)
    R = G[rank * nR * 2:(rank + 1) * nR * 2].clone()
    del G
    S = torch.empty(nS * 2, dtype=torch.int64, device="cuda")
    ctx.gen_fk(S, nS, nR * world, args.theta, SEED_KEYS, VMAX, SEED_PROBE + rank)
    torch.cuda.synchronize()
    be = pyg_dist.GpuBackend(ctx, torch.device(f"cuda:{local}"))
    I64 = pyg.INT64
    Rb, Sb = R.view(torch.uint8), S.view(torch.uint8)

    def step():
        cnt, sums = pyg_dist.join_agg(dist, be, Rb, nR, [I64, I64], 0, Sb, nS, [I64, I64], 0, [(0, 1), (1, 1)])
        return cnt, (sums[0] + sums[1]) & 0xFFFFFFFFFFFFFFFF

    cnt, chk = step()
    Sv = S.view(nS, 2)
    local_chk = torch.tensor([int((Sv[:, 0] * 7 + Sv[:, 1]).sum().item())], dtype=torch.int64, device="cuda")
    dist.all_reduce(local_chk)
    if cnt != nS * world or chk != int(local_chk.item()) & 0xFFFFFFFFFFFFFFFF:
        raise SystemExit(f"rank {rank}: result mismatch: count {cnt} vs {nS * world}")
    for _ in range(args.warmup):
        step()
    launches0 = ctx.launches()
    dist.barrier()
    torch.cuda.synchronize()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(local) as clk:
        t0.record(stream)
        for _ in range(args.steps):
            step()
        t1.record(stream)
        torch.cuda.synchronize()
    dist.barrier()
    ms = max_over_ranks(t0.elapsed_time(t1), dist, "cuda")
    launches = ctx.launches() - launches0
    hbm, peak_kind = peaks()
    step_bytes = (nR + nS) * 16
    value = (nR + nS) * args.steps * world / (ms / 1e3)
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "int64", "data": "synthetic (seeded, device-generated)",
                "config": {"workload": "partitioned PK-FK hash join + count + checksum over all ranks",
                           "build_tuples_per_rank": nR, "probe_tuples_per_rank": nS, "tuple_bytes": 16,
                           "theta": args.theta, "parallelism": f"hash-shuffle{world} (NCCL all_to_all)",
                           "l2": "inputs larger than L2; no flush needed"},
                "roofline": {"bound": "hbm", "scope": "whole step per rank", "peak": hbm, "unit": "GB/s",
                             "achieved": round(step_bytes / (ms / args.steps / 1e3) / 1e9, 1),
                             "frac": round(step_bytes / (ms / args.steps / 1e3) / 1e9 / hbm, 4),
                             "peak_source": peak_kind, "traffic": None},
                "cpu_baseline": None,
                "e2e": {"value": None, "skipped": "multi-GPU shuffle mode times device-resident inputs only"},
                "gpu_launches": launches, "clocks": clk.summary()}
        print(json.dumps(line), flush=True)
    ctx.close()
    dist.destroy_process_group()


def main_gpu(args):
    import torch
    import pyg

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    # One dedicated stream shared by torch and the library: the kernels and
    # the timing events are on the same stream.
    torch.cuda.set_stream(torch.cuda.Stream(local))
    dist = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    nR, nS = N_BUILD >> args.scale_shift, N_PROBE >> args.scale_shift
    ctx = pyg.Ctx(local)
    stream = torch.cuda.current_stream(local)

    # Each rank joins its own (R, S) pair: the per-GPU work is fixed (weak
    # scaling); there is no data exchange between ranks.
    R = torch.empty(nR * 2, dtype=torch.int64, device="cuda")
    S = torch.empty(nS * 2, dtype=torch.int64, device="cuda")
    ctx.gen_pk(R, nR, 7, SEED_KEYS)
    ctx.gen_fk(S, nS, nR, args.theta, SEED_KEYS, VMAX, SEED_PROBE + rank)
    torch.cuda.synchronize()
    Rr = pyg.Rel(R, nR, [pyg.INT64, pyg.INT64])
    Sr = pyg.Rel(S, nS, [pyg.INT64, pyg.INT64])
    proj = [(0, 1), (1, 1)]

    algo = {"radix": pyg.JOIN_RADIX, "direct": pyg.JOIN_DIRECT, "auto": pyg.JOIN_AUTO}[args.algo]

    def step(rrel, srel, stats=False):
        r = ctx.hashjoin_agg(rrel, [0], srel, [0], proj, algo, args.radix_bits, args.load_factor, stats=stats)
        (cnt, sums), st = r if stats else (r, None)
        return cnt, (sums[0] + sums[1]) & 0xFFFFFFFFFFFFFFFF, st

    # Size-independent check of the result (every fk matches exactly once;
    # R.payload = 7 * key): count == |S| and checksum == sum(7 fk + val).
    cnt, chk, _ = step(Rr, Sr)
    Sv = S.view(nS, 2)
    expect = int((Sv[:, 0] * 7 + Sv[:, 1]).sum().item()) & 0xFFFFFFFFFFFFFFFF
    if cnt != nS or chk != expect:
        raise SystemExit(f"result mismatch: count {cnt} vs {nS}, checksum {chk} vs {expect}")

    for _ in range(args.warmup):
        step(Rr, Sr)
    launches0 = ctx.launches()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    t_start = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    # Each timed step also reports its phase times: CUDA events the library
    # records on the stream its kernels run on (the step synchronises on its
    # result anyway, so they add no wait).
    phase = []
    with Clocks(local) as clk:
        t_start.record(stream)
        for k in range(args.steps):
            phase.append(step(Rr, Sr, stats=True)[2])
        t_end.record(stream)
        torch.cuda.synchronize()
    launches = ctx.launches() - launches0
    ms = max_over_ranks(t_start.elapsed_time(t_end), dist, "cuda")
    value = (nR + nS) * args.steps * world / (ms / 1000.0)

    hbm, peak_kind = peaks()
    roofline = join_roofline(pyg, phase, nR, nS, ms / args.steps, hbm, peak_kind, args.theta)

    # End to end: the same C-ABI calls with host (pinned) buffers; the
    # library copies each relation to the device inside the timed region.
    e2e = None
    if not args.no_e2e:
        e2e = run_e2e(args, torch, pyg, ctx, R, S, nR, nS, world, dist)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        try:
            r = run_reference_cpu(args.theta, 3)
            cpu = {"value": r["tuples"] * len(r["times"]) / sum(r["times"]), "unit": UNIT, "cores": r["cores"],
                   "kind": r["kind"], "sample": r["sample"]}
        except Exception as ex:  # the CPU leg must not hide the GPU number
            cpu = {"value": None, "unit": UNIT, "cores": None, "kind": "unavailable", "sample": str(ex)[:200]}

    secondary = None
    if world == 1 and not args.no_secondary:
        del R, S, Rr, Sr
        torch.cuda.synchronize()
        torch.cuda.empty_cache()
        secondary = run_secondary(args, torch, pyg, ctx, local, stream)

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "int64", "data": "synthetic (seeded, device-generated)",
                "config": {"workload": "radix-scale PK-FK hash join + count + checksum", "build_tuples": nR,
                           "probe_tuples": nS, "tuple_bytes": 16, "theta": args.theta,
                           "load_factor": args.load_factor, "parallelism": f"replicas{world}",
                           "l2": "inputs (19.3 GB) larger than L2; no flush needed"},
                "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches,
                "clocks": clk.summary()}
        if secondary is not None:
            line["secondary"] = secondary
        print(json.dumps(line), flush=True)
    ctx.close()
    if dist:
        dist.destroy_process_group()


def source_digest(files):
    """Digest of the kernel sources a committed ncu figure was taken from."""
    import hashlib
    h = hashlib.sha256()
    for f in files:
        with open(os.path.join(ROOT, "pythia-core_b200", "csrc", f), "rb") as fh:
            h.update(fh.read())
    return h.hexdigest()[:16]


# The sources each kernel's committed ncu traffic figure depends on.
TRAFFIC_SOURCES = {"partition": ["radixpart.cu", "radixpart.cuh", "bulk.cuh"],
                   "join": ["radixjoin.cu", "radixpart.cuh"]}


def join_roofline(pyg, phase, nR, nS, step_ms, hbm, peak_kind, theta):
    """The roofline object of the join line.

    Every kernel launch is charged the workload's algorithmic bytes for the
    units it processes: 16 B per input tuple read once (a partition pass of
    S processes |S| tuples, the join |R| + |S|).  `frac` is that figure for
    the dominant launch over its CUDA-event time, against the measured copy
    bandwidth.  `kernel_bw_frac` counts the bytes the launch actually moves
    (its reads and writes in the intermediate format), and `step_frac` the
    whole step's algorithmic bytes, (|R| + |S|) x 16, over the step time."""
    mean = lambda f: statistics.fmean(getattr(p, f) for p in phase)  # noqa: E731
    mean2 = lambda f, i: statistics.fmean(getattr(p, f)[i] for p in phase)  # noqa: E731
    radix = int(phase[0].algorithm) == pyg.JOIN_RADIX
    two = radix and int(phase[0].radix_bits) > 9
    launches = {}
    if radix:
        for side, n, packed in (("build", nR, int(phase[0].build_packed)), ("probe", nS, int(phase[0].probe_packed))):
            e = 8 if packed else 16
            p1 = mean2(f"{side}_pass_ms", 0)
            moved1 = n * (16 + e)
            launches[f"{side}_pass1"] = ("rj_partition_kernel", p1, n * 16, moved1, packed)
            if two:
                launches[f"{side}_pass2"] = ("rj_partition_kernel", mean2(f"{side}_pass_ms", 1), n * 16, n * 2 * e,
                                             packed)
        eR = 8 if int(phase[0].build_packed) else 16
        eS = 8 if int(phase[0].probe_packed) else 16
        jk = mean("join_kernel_ms")
        launches["join"] = ("rj_join32_kernel" if jk > 0 else "rj_join_kernel", jk if jk > 0 else mean("probe_ms"),
                            (nR + nS) * 16, nR * eR + nS * eS, None)
    else:
        launches["build"] = ("ht_build16_kernel", mean("build_ms"), nR * 16, nR * 16, None)
        launches["probe"] = ("probe_agg16_kernel", mean("probe_ms"), nS * 16, nS * 16, None)
    ph = {}
    for k, (kern, t, alg, moved, packed) in launches.items():
        ph[k] = {"kernel": kern, "ms": round(t, 4), "algorithmic_bytes": alg, "moved_bytes": moved,
                 "packed": packed,
                 "achieved_gbs": round(alg / (t / 1e3) / 1e9, 1) if t > 0 else None,
                 "frac": round(alg / (t / 1e3) / 1e9 / hbm, 4) if t > 0 else None,
                 "kernel_bw_frac": round(moved / (t / 1e3) / 1e9 / hbm, 4) if t > 0 else None}
    top = max((k for k in ph if ph[k]["ms"] > 0), key=lambda k: ph[k]["ms"])
    step_bytes = (nR + nS) * 16
    roofline = {"bound": "hbm", "kernel": ph[top]["kernel"], "launch": top, "achieved": ph[top]["achieved_gbs"],
                "peak": hbm, "unit": "GB/s", "frac": ph[top]["frac"], "kernel_bw_frac": ph[top]["kernel_bw_frac"],
                "peak_source": peak_kind, "bytes_per_launch": ph[top]["algorithmic_bytes"],
                "moved_bytes_per_launch": ph[top]["moved_bytes"], "ms_per_launch": ph[top]["ms"], "traffic": None,
                "launches": ph, "algorithm": int(phase[0].algorithm), "radix_bits": int(phase[0].radix_bits),
                "histogram_ms": round(mean("histogram_ms"), 3) if radix else None,
                "histogram_tuples": int(phase[0].histogram_tuples) if radix else None,
                # Host round trips inside the step: the layouts formed from the
                # histograms (before the build side's passes), and the work
                # items formed from the partition counts (before the join).
                "host_layout_ms": round(mean("build_partition_ms") - mean2("build_pass_ms", 0)
                                        - mean2("build_pass_ms", 1), 3) if radix else None,
                "host_items_ms": round(mean("probe_ms") - mean("join_kernel_ms"), 3) if radix else None,
                "step_achieved_gbs": round(step_bytes / (step_ms / 1e3) / 1e9, 1),
                "step_frac": round(step_bytes / (step_ms / 1e3) / 1e9 / hbm, 4)}
    # DRAM traffic of the dominant launch from an ncu capture of the same
    # kernel sources (scaled to this launch's tuples); none if the sources
    # changed since the capture.
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if radix and os.path.exists(tpath):
        with open(tpath) as f:
            tj = json.load(f)
        ent = tj.get(f"{top}@theta={theta}")
        kernel = "join" if top == "join" else "partition"
        if ent and ent.get("sources") == source_digest(TRAFFIC_SOURCES[kernel]):
            roofline["traffic"] = ent["bytes_per_tuple"] * (nR + nS if top == "join" else
                                                           (nR if top.startswith("build") else nS))
            roofline["traffic_source"] = ent.get("profile")
    return roofline


def run_e2e(args, torch, pyg, ctx, R, S, nR, nS, world, dist):
    try:
        import psutil
        avail = psutil.virtual_memory().available
    except Exception:
        avail = 0
    # Every rank on this node pins its own copy of the inputs; all ranks
    # take the same decision (they share the collectives below).
    need = (nR + nS) * 16 * world
    ok = not (avail and avail < 3 * need)
    if dist:
        t = torch.tensor([1 if ok else 0], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MIN)
        ok = bool(t.item())
    if not ok:
        return {"value": None, "unit": UNIT, "skipped": "host RAM below 3x the inputs of the node's ranks"}
    hR = pyg.HostBuf(nR * 16)
    hS = pyg.HostBuf(nS * 16)
    try:
        ctx.d2h(hR.np, R)
        ctx.d2h(hS.np, S)
        Rh = pyg.Rel(hR.ptr, nR, [pyg.INT64, pyg.INT64], on_device=0)
        Sh = pyg.Rel(hS.ptr, nS, [pyg.INT64, pyg.INT64], on_device=0)
        proj = [(0, 1), (1, 1)]

        def step():
            cnt, sums = ctx.hashjoin_agg(Rh, [0], Sh, [0], proj, pyg.JOIN_AUTO, 0, args.load_factor)
            return cnt

        step()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        steps = max(1, min(args.steps, 3))
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        stream = torch.cuda.current_stream()
        t0.record(stream)
        for _ in range(steps):
            c = step()
        t1.record(stream)
        torch.cuda.synchronize()
        assert c == nS
        ms = max_over_ranks(t0.elapsed_time(t1), dist, "cuda")
        return {"value": (nR + nS) * steps * world / (ms / 1000.0), "unit": UNIT,
                "h2d_bytes_per_step": (nR + nS) * 16, "d2h_bytes_per_step": 2 * 8 * 4 + 9 * 8,
                "ms_per_step": ms / steps, "host_buffers": "pinned"}
    finally:
        hR.free()
        hS.free()


# ------------------------------------------------- the other configurations

def _device_timed(torch, stream, fn, steps, warmup, dist):
    """W untimed calls, then K calls between CUDA events on `stream`; the
    job's milliseconds are the max over ranks."""
    for _ in range(warmup):
        fn()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    out = [fn() for _ in range(steps)]
    t1.record(stream)
    torch.cuda.synchronize()
    return max_over_ranks(t0.elapsed_time(t1), dist, "cuda"), out


def _reference_rows(rels, plan_fn, steps):
    """Times the reference engine on host arrays {name: (array, types)} with
    all host cores; plan_fn(T, files) builds the plan text."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import refrun
    if not refrun.available():
        return None
    T = min(os.cpu_count() or 1, 127)
    times = []
    with tempfile.TemporaryDirectory(dir=os.environ.get("PYG_TMP")) as d:
        files = {}
        for name, (arr, types) in rels.items():
            files[name] = refrun.write_rel(d, name, arr, T)
        plan = plan_fn(T, files)
        for _ in range(steps):
            _, rt, _ = refrun.run(d, plan, timeout=900)
            times.append(rt)
    return T, times


def main_workload(args):
    import torch
    import pyg

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    torch.cuda.set_stream(torch.cuda.Stream(local))
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    ctx = pyg.Ctx(local)
    stream = torch.cuda.current_stream(local)
    line = workload_line(args, torch, pyg, ctx, rank, world, local, dist, stream)
    if rank == 0:
        print(json.dumps(line), flush=True)
    ctx.close()
    if dist:
        dist.destroy_process_group()


def workload_line(args, torch, pyg, ctx, rank, world, local, dist, stream):
    """Measures one of the other configurations and returns its JSON line."""
    hbm, peak_kind = peaks()
    sh = args.scale_shift
    g = torch.Generator(device="cuda")
    g.manual_seed(1234 + rank)
    I64 = pyg.INT64
    cpu = None
    extra = {}

    if args.workload == "join-small":
        # R: permutation of 1..2^20, payload = 7 key; S: 2^24 fk ~ U over R's keys, val ~ U{0..999}.
        nR, nS = (1 << 20) >> sh, (1 << 24) >> sh
        R = torch.empty(nR * 2, dtype=torch.int64, device="cuda")
        S = torch.empty(nS * 2, dtype=torch.int64, device="cuda")
        ctx.gen_pk(R, nR, 7, SEED_KEYS)
        ctx.gen_fk(S, nS, nR, 0.0, SEED_KEYS, 1000, SEED_PROBE + rank)
        Rr, Sr = pyg.Rel(R, nR, [I64, I64]), pyg.Rel(S, nS, [I64, I64])
        algo = {"radix": pyg.JOIN_RADIX, "direct": pyg.JOIN_DIRECT, "auto": pyg.JOIN_AUTO}[args.algo]
        # One C-ABI call per step (arguments marshalled once): the step is
        # the library's join + sum with its result read back to the host.
        fn = ctx.hashjoin_agg_prepared(Rr, [0], Sr, [0], [(1, 1)], algo)
        cnt, sums = fn()
        Sv = S.view(nS, 2)
        assert cnt == nS and sums[0] & 0xFFFFFFFFFFFFFFFF == int(Sv[:, 1].sum().item()) & 0xFFFFFFFFFFFFFFFF
        units, abytes = nR + nS, (nR + nS) * 16 + 16
        metric = "join+sum tuples/sec (R 2^20 PK, S 2^24 FK, projection P$1)"
        workload = {"workload": "hash join + sum of P$1", "build_tuples": nR, "probe_tuples": nS, "algo": args.algo}
        if rank == 0 and world == 1 and not args.no_cpu:
            sys.path.insert(0, os.path.join(ROOT, "oracle"))
            import refrun
            dt = np.dtype([("c0", np.int64), ("c1", np.int64)])
            Rh, Sh = R.view(nR, 2).cpu().numpy(), S.view(nS, 2).cpu().numpy()
            r = _reference_rows({"R": (Rh.view(dt).reshape(-1), 2), "S": (Sh.view(dt).reshape(-1), 2)},
                                lambda T, f: refrun.plan_join_sum(T, f["R"], [2, 2], f["S"], [2, 2], [(1, 1)], 0, nR), 3)
            if r:
                cpu = {"value": units * len(r[1]) / sum(r[1]), "unit": UNIT, "cores": r[0], "kind": "reference",
                       "sample": f"the whole workload, executequery ResponseTimeInSec, {r[0]} threads"}
    elif args.workload == "join-radix":
        # The headline radix join (R 2^27 PK, S 2^30 FK, count + checksum)
        # with the fks Zipf(theta) over R's keys: the configuration's other
        # skews.  Checked like the headline: count == |S| and checksum ==
        # sum(7 fk + val).
        nR, nS = N_BUILD >> sh, N_PROBE >> sh
        R = torch.empty(nR * 2, dtype=torch.int64, device="cuda")
        S = torch.empty(nS * 2, dtype=torch.int64, device="cuda")
        ctx.gen_pk(R, nR, 7, SEED_KEYS)
        ctx.gen_fk(S, nS, nR, args.theta, SEED_KEYS, VMAX, SEED_PROBE + rank)
        Rr, Sr = pyg.Rel(R, nR, [I64, I64]), pyg.Rel(S, nS, [I64, I64])

        def fn():
            cnt, sums = ctx.hashjoin_agg(Rr, [0], Sr, [0], [(0, 1), (1, 1)], pyg.JOIN_RADIX, args.radix_bits,
                                         args.load_factor)
            return cnt, (sums[0] + sums[1]) & 0xFFFFFFFFFFFFFFFF

        cnt, chk = fn()
        Sv = S.view(nS, 2)
        expect = int((Sv[:, 0] * 7 + Sv[:, 1]).sum().item()) & 0xFFFFFFFFFFFFFFFF
        assert cnt == nS and chk == expect, (cnt, chk, expect)
        units, abytes = nR + nS, (nR + nS) * 16
        metric = METRIC
        workload = {"workload": "radix-scale PK-FK hash join + count + checksum", "build_tuples": nR,
                    "probe_tuples": nS, "theta": args.theta, "l2": "inputs larger than L2; no flush needed"}
    elif args.workload == "groupby":
        # N = 2^28 (int64 group id, int64 value); ids ~ U[0, G) or Zipf(1.0); sum and count per group, sorted.
        N, G = (1 << 28) >> sh, args.groups
        if args.zipf:
            w = torch.arange(1, G + 1, dtype=torch.float64, device="cuda").pow(-1.0)
            ids = torch.multinomial(w / w.sum(), N, replacement=True, generator=g) if N <= (1 << 24) else \
                torch.cat([torch.multinomial(w / w.sum(), 1 << 24, replacement=True, generator=g)
                           for _ in range(N >> 24)])
        else:
            ids = torch.randint(0, G, (N,), device="cuda", generator=g)
        vals = torch.randint(0, 1 << 20, (N,), device="cuda", generator=g)
        A = torch.stack([ids, vals], 1).contiguous().view(-1)
        del ids, vals
        rel = pyg.Rel(A, N, [I64, I64])
        out = torch.empty(G * 3, dtype=torch.int64, device="cuda")

        def fn():
            rc, ng = ctx.groupby(rel, [0], pyg.AGG_SUM | pyg.AGG_COUNT, 1, True, G, out, G)
            assert rc == pyg.PYG_OK
            return ng

        ng = fn()
        o = out[: ng * 3].view(ng, 3)
        Av = A.view(N, 2)
        assert int(o[:, 2].sum().item()) == N and int(o[:, 1].sum().item()) == int(Av[:, 1].sum().item())
        assert bool((o[1:, 0] > o[:-1, 0]).all().item())
        units, abytes = N, N * 16 + ng * 24
        metric = "group-by tuples/sec (N 2^28, sum + count per group, sorted by key)"
        workload = {"workload": "group-by sum+count", "tuples": N, "groups": G, "groups_found": ng,
                    "ids": "zipf1.0" if args.zipf else "uniform"}
        if rank == 0 and world == 1 and not args.no_cpu:
            sys.path.insert(0, os.path.join(ROOT, "oracle"))
            import refrun
            dt = np.dtype([("c0", np.int64), ("c1", np.int64)])
            n_cpu = N >> CPU_SAMPLE_SHIFT
            Ah = Av[:n_cpu].cpu().numpy()
            r = _reference_rows({"A": (Ah.view(dt).reshape(-1), 2)},
                                lambda T, f: refrun.plan_groupby(T, f["A"], [2, 2], [0], "sum", 1, G), 3)
            if r:
                cpu = {"value": n_cpu * len(r[1]) / sum(r[1]), "unit": UNIT, "cores": r[0], "kind": "reference",
                       "sample": f"first 1/{1 << CPU_SAMPLE_SHIFT} of the tuples (aggregate_sum, merge, "
                                 f"re-aggregate), ResponseTimeInSec, {r[0]} threads"}
    elif args.workload == "mpsm":
        # R 2^26 PK, S 2^28 FK ~ Zipf(theta); range partition (learned CDF splitter) -> sort -> merge join.
        nR, nS = (1 << 26) >> sh, (1 << 28) >> sh
        R = torch.empty(nR * 2, dtype=torch.int64, device="cuda")
        S = torch.empty(nS * 2, dtype=torch.int64, device="cuda")
        ctx.gen_pk(R, nR, 7, SEED_KEYS)
        ctx.gen_fk(S, nS, nR, args.theta, SEED_KEYS, VMAX, SEED_PROBE + rank)
        Rr, Sr = pyg.Rel(R, nR, [I64, I64]), pyg.Rel(S, nS, [I64, I64])
        kind = {"learned": pyg.MPSM_LEARNED, "sampled": pyg.MPSM_SAMPLED, "exactrange": pyg.MPSM_EXACTRANGE}[
            args.splitter]
        opts = ctx.mpsm_opts(kind, args.fanout, 0.01, 1024)
        fn = lambda: ctx.mpsm_join_agg(Rr, 0, Sr, 0, [(0, 1), (1, 1)], opts)  # noqa: E731
        fn()
        cnt, sums, st = fn()  # stats of a warm call
        Sv = S.view(nS, 2)
        expect = int((Sv[:, 0] * 7 + Sv[:, 1]).sum().item()) & 0xFFFFFFFFFFFFFFFF
        assert cnt == nS and (sums[0] + sums[1]) & 0xFFFFFFFFFFFFFFFF == expect
        units, abytes = nR + nS, (nR + nS) * 16
        metric = "MPSM join+agg tuples/sec (R 2^26 PK, S 2^28 FK, range partition + sort + merge)"
        workload = {"workload": "MPSM sort-merge join + count + checksum", "build_tuples": nR, "probe_tuples": nS,
                    "theta": args.theta, "splitter": args.splitter, "fanout": args.fanout}
        extra["mpsm"] = {"max_partition_imbalance": round(st.max_partition_imbalance, 3),
                         "splitter_ms": round(st.splitter_ms, 3), "partition_ms": round(st.partition_ms, 3),
                         "sort_ms": round(st.sort_ms, 3), "merge_ms": round(st.merge_ms, 3)}
    else:  # batch
        # 256 fragments: build n_i = 2^U(12, 22), probe n_i x U{4..32}; keys uniform or Zipf(1.0); PK-FK + sum.
        rng = np.random.default_rng(99 + rank)
        pairs, keep, units = [], [], 0
        for i in range(256):
            nb = max(1, int(2 ** rng.uniform(12, 22)) >> sh)
            npr = nb * int(rng.integers(4, 33))
            Rb = torch.empty(nb * 2, dtype=torch.int64, device="cuda")
            Sb = torch.empty(npr * 2, dtype=torch.int64, device="cuda")
            ctx.gen_pk(Rb, nb, 7, 1000 + i)
            ctx.gen_fk(Sb, npr, nb, 1.0 if i % 2 else 0.0, 1000 + i, VMAX, 5000 + i)
            pairs.append((Rb, nb, Sb, npr))
            keep += [Rb, Sb]
            units += nb + npr
        frags = ctx.fragments(pairs)
        tuning = ctx.autotune(frags)
        b = ctx.batch_create(frags, tuning)

        def fn():
            rc, c, sm, lat = ctx.batch_run(b, len(pairs))
            assert rc == pyg.PYG_OK
            return c, lat

        c, _ = fn()
        assert all(int(c[i]) == pairs[i][3] for i in range(len(pairs)))
        abytes = units * 16
        metric = "batched fragments tuples/sec (256 PK-FK join+sum fragments, persistent kernel in a CUDA graph)"
        workload = {"workload": "256 join fragments", "fragments": 256, "tuples": units,
                    "tuning": {"block_threads": tuning.block_threads, "blocks_per_sm": tuning.blocks_per_sm,
                               "load_factor": round(tuning.load_factor, 2), "chunk_tuples": tuning.chunk_tuples,
                               "large_build": tuning.large_build}}

    ms, outs = _device_timed(torch, stream, fn, args.steps, args.warmup, dist)
    # A second timed run with the clock sampler on; the line reports it.
    launches0 = ctx.launches()
    with Clocks(local) as clk:
        ms, _ = _device_timed(torch, stream, fn, args.steps, 0, dist)
    launches = ctx.launches() - launches0
    step_ms = ms / args.steps
    if args.workload == "mpsm":
        # Phase times: medians over the timed calls of the first timed run.
        sts = [o[2] for o in outs]
        med = lambda f: round(float(np.median([getattr(x, f) for x in sts])), 3)  # noqa: E731
        extra["mpsm"].update({f: med(f) for f in ("splitter_ms", "partition_ms", "merge_ms")})
        extra["mpsm"]["phase_stat"] = f"median of {len(sts)} timed calls"
    if args.workload == "batch":
        lat = np.concatenate([o[1] for o in outs])
        extra["fragment_latency_ms"] = {"p50": round(float(np.percentile(lat, 50)), 4),
                                        "p99": round(float(np.percentile(lat, 99)), 4)}
        plain_ms, plain_outs = _device_timed(torch, stream, lambda: ctx.batch_run_plain(frags)[2],
                                             max(1, args.steps // 2), 1, dist)
        plat = np.concatenate(plain_outs)
        extra["plain"] = {"ms_per_step": round(plain_ms / max(1, args.steps // 2), 4),
                          "fragment_latency_ms": {"p50": round(float(np.percentile(plat, 50)), 4),
                                                  "p99": round(float(np.percentile(plat, 99)), 4)},
                          "what": "the same fragments one pyg_hashjoin_agg call after another"}
        extra["batched_over_plain"] = round(extra["plain"]["ms_per_step"] / step_ms, 3)
        ctx.batch_free(b)
    achieved = abytes / (step_ms / 1e3) / 1e9
    line = {"metric": metric, "value": units * args.steps * world / (ms / 1e3), "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int64", "data": "synthetic (seeded, device-generated)",
            "config": dict(workload, parallelism=f"replicas{world}", scale_shift=sh),
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": hbm, "unit": "GB/s",
                         "frac": round(achieved / hbm, 4), "peak_source": peak_kind, "traffic": None,
                         "algorithmic_bytes_per_step": abytes, "scope": "whole step"},
            "cpu_baseline": cpu, "e2e": None, "gpu_launches": launches, "clocks": clk.summary()}
    line.update(extra)
    return line


# Configurations measured beside the headline in the default run, with the
# bench options that select each: the headline join at the other two fk
# skews, the small join, group-by at three
# cardinalities, the MPSM join with both splitters on skewed keys, and the
# batched fragments.
SECONDARY = [
    ("join_theta0.75", dict(workload="join-radix", theta=0.75)),
    ("join_theta1.25", dict(workload="join-radix", theta=1.25)),
    ("join_small", dict(workload="join-small")),
    ("groupby_G16", dict(workload="groupby", groups=16)),
    ("groupby_G2p16", dict(workload="groupby", groups=1 << 16)),
    ("groupby_G2p16_zipf", dict(workload="groupby", groups=1 << 16, zipf=True)),
    ("mpsm_sampled_theta1", dict(workload="mpsm", splitter="sampled", theta=1.0)),
    ("mpsm_learned_theta1", dict(workload="mpsm", splitter="learned", theta=1.0)),
    ("batch", dict(workload="batch")),
]


def run_secondary(args, torch, pyg, ctx, local, stream):
    """Each secondary configuration with 5 timed steps after 3 warm-ups, in
    this process (rank 0 of a 1-GPU run); a compact summary of its line."""
    out = {}
    for name, opts in SECONDARY:
        a = argparse.Namespace(**vars(args))
        a.steps, a.warmup, a.no_cpu, a.scale_shift, a.theta, a.zipf = 5, 3, True, 0, 0.0, False
        a.groups, a.splitter, a.fanout, a.algo = 1 << 16, "learned", 4096, "auto"
        for k, v in opts.items():
            setattr(a, k, v)
        try:
            line = workload_line(a, torch, pyg, ctx, 0, 1, local, None, stream)
            out[name] = {"metric": line["metric"], "value": line["value"], "ms_per_step": line["ms_per_step"],
                         "roofline_frac": line["roofline"]["frac"], "config": line["config"],
                         "clocks": line["clocks"]}
            for k in ("mpsm", "fragment_latency_ms", "plain", "batched_over_plain"):
                if k in line:
                    out[name][k] = line[k]
        except Exception as ex:  # a secondary must not hide the headline
            out[name] = {"error": str(ex)[:300]}
        torch.cuda.empty_cache()
    return out


def main():
    args = parse()
    if args.algo is None:
        args.algo = "auto" if args.workload == "join-small" else "radix"
    if args.impl == "reference":
        main_reference(args)
    elif args.workload != "join":
        main_workload(args)
    elif dist_env()[1] > 1 and args.dist_mode == "shuffle":
        main_dist(args)
    else:
        main_gpu(args)


if __name__ == "__main__":
    main()
