#!/usr/bin/env python
"""Benchmark: batched exact pi(x) queries on B200.

Workload (one step): 4096 queries x = floor(10^e), e ~ U[9, 14] drawn from
numpy default_rng(0), all answered by one call of the public batch API
(cudapix_b200.pi_batch -> cpx_pi_batch), every answer exact.  Synthetic
inputs; the reference publishes no dataset or numbers for this path.

  value            queries/s over the device timeline of the batch kernels
                   (CUDA events on the context stream; query list already
                   planned, tables resident)
  e2e              queries/s through the C ABI with host buffers: planning,
                   host->device copy of the queries, kernels, device->host read
  plain            the same queries one pi_deleglise_rivat call (one launch
                   sequence) each, with p50/p99 latency
  cpu_baseline     the oracle's OpenMP restatement of the term pipeline on
                   the host cores, on a bounded sample of the same queries;
                   beside it (reference_terms) the reference's own OpenMP host
                   term code, Gourdon's A and C, restated and timed the same way

`--impl reference` times that CPU restatement alone (the reference itself
cannot be built: its CUDASieve / CUDA-uint128 dependencies are not vendored).
Multi-GPU (`torchrun ... --gpus N`): independent replicas, each GPU answers
its own 4096-query batch; barrier + max over ranks; value = all queries / max time.
"""
import argparse
import gc
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "pi(x) queries/sec (batched, exact)"
UNIT = "queries/s"


def workload(n, seed=0, lo=9.0, hi=14.0):
    e = np.random.default_rng(seed).uniform(lo, hi, n)
    return [int(10.0**v) for v in e]


class Clocks:
    """nvidia-smi sampler running during the timed region."""

    def __init__(self, dev):
        self.dev = dev
        self.proc = None
        self.path = os.path.join(tempfile.gettempdir(), f"cudapix_clocks_{os.getpid()}.csv")

    def __enter__(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.dev}",
                 "--query-gpu=index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        rows = []
        for line in open(self.path):
            p = [s.strip() for s in line.split(",")]
            if len(p) < 9:
                continue
            try:
                rows.append((float(p[1]), float(p[2]), p[5:9]))
            except ValueError:
                continue
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for _, _, r in rows for i, v in enumerate(r) if v.lower() == "active"})
        return {"sm_mhz": statistics.median(r[0] for r in rows), "sm_max_mhz": max(r[1] for r in rows),
                "reasons": reasons, "samples": len(rows)}


TUNING = os.path.join(ROOT, "cudapix_b200", "tuning", "b200.json")


def tuned_context(cpx, device):
    """A context with the committed B200 tuning table (cpx_autotune output),
    when present; results are the same with or without it."""
    ctx = cpx.Context(device)
    if os.path.exists(TUNING):
        ctx.tune_load(TUNING)
    return ctx


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            m = json.load(f)
        return m["hbm_gbs"], "measured"
    except Exception:
        return 6650.0, "fallback"


PROFILES = {k: os.path.join(ROOT, "profiles", f"{k}_batch4096.json") for k in ("k_hard_shared", "k_easy")}


def source_sha(files):
    """sha256 over the kernel's source files, as the ncu summary records it."""
    import hashlib

    h = hashlib.sha256()
    for f in files:
        with open(os.path.join(ROOT, f), "rb") as fh:
            h.update(fh.read())
    return h.hexdigest()[:16]


def kernel_profile(name):
    """Per-launch counters of one of the batch's two dominant kernels on this
    workload from its committed ncu capture (profiles/<kernel>_batch4096.json),
    and whether the capture was taken of the current kernel source."""
    try:
        with open(PROFILES[name]) as f:
            pr = json.load(f)
        pr["matches_source"] = source_sha(pr["source_files"]) == pr["source_sha"]
        return pr
    except Exception:
        return None


def golden_answers(name, xs):
    """The oracle's answers for a workload (tests/golden/make_config_golden.py),
    when the committed fixture holds exactly these queries."""
    try:
        with open(os.path.join(ROOT, "tests", "golden", name)) as f:
            g = json.load(f)
    except Exception:
        return None
    return g["pi"] if g["x"] == xs else None


SMEM_BYTES_PER_CLK = 128  # shared-memory bandwidth of one SM per clock (32 banks x 4 B)
ISSUE_PER_CLK = 4  # warp instructions an SM issues per clock (4 schedulers)


def roofline(kern, hard_ms, hard_bytes, dev_ms, clocks, ctx):
    """Roofline of the batch's dominant kernel (k_easy or k_hard_shared,
    whichever took longer in the timed steps), both bound by the integer ALU
    pipe; the other one beside it.

    achieved = ALU-pipe warp instructions of one launch (ncu, the committed
    capture of this workload; `profile_matches_source` says whether it was
    taken of the current kernel source) / the launch's duration, measured
    live with CUDA events on the context stream; peak = the ALU pipe's issue
    rate per SM per clock (2, ncu's peak_sustained) x SMs x the median SM
    clock sampled during the timed steps.  Beside it: all issued
    instructions against 4 per SM per clock, and for the phi sieve the S2
    rate (segment-bitmap bytes it passes over, one pass per level per
    segment, / duration of the hard-leaf kernels) against the shared-memory
    bandwidth 128 B per SM per clock."""
    mhz = clocks.get("sm_mhz") or 1965.0
    sms = ctx.sm_count()

    def one(name, what):
        ks = statistics.median(k.get(name, 0.0) for k in kern) / 1000.0
        pr = kernel_profile(name)
        r = {"bound": "alu", "kernel": f"{name} ({what})", "unit": "Ginst/s", "achieved": None, "peak": None,
             "frac": None, "kernel_ms": ks * 1000.0, "traffic": None,
             "peak_kind": f"derived: ALU-pipe warp instructions per SM per clock (ncu peak_sustained) x {sms} SMs "
                          f"x {mhz:.0f} MHz (median sampled SM clock), of measured clocks",
             "profile": os.path.relpath(PROFILES[name], ROOT), "profile_matches_source": None}
        if pr and ks:
            r["achieved"] = pr["alu_warp_inst_per_launch"] / ks / 1e9
            r["peak"] = pr["alu_peak_warp_inst_per_sm_clk"] * sms * mhz * 1e6 / 1e9
            r["frac"] = r["achieved"] / r["peak"]
            r["traffic"] = pr["dram_bytes_per_launch"]
            r["profile_matches_source"] = pr["matches_source"]
            issue_peak = ISSUE_PER_CLK * sms * mhz * 1e6 / 1e9
            r["issue_view"] = {"achieved": pr["warp_inst_per_launch"] / ks / 1e9, "peak": issue_peak,
                               "unit": "Ginst/s", "frac": pr["warp_inst_per_launch"] / ks / 1e9 / issue_peak}
        return r

    rows = {"k_hard_shared": one("k_hard_shared", "batch-shared special-leaf phi sieve"),
            "k_easy": one("k_easy", "easy special leaves, one quotient and one pi-table gather each")}
    hs = statistics.median(hard_ms) / 1000.0
    hb = hard_bytes[-1]
    smem_peak = sms * SMEM_BYTES_PER_CLK * mhz * 1e6 / 1e9
    s2 = (hb / hs) / 1e9 if hs else None
    rows["k_hard_shared"]["smem_view"] = {
        "achieved": s2, "peak": smem_peak, "unit": "GB/s", "frac": s2 / smem_peak if s2 else None,
        "peak_kind": f"derived: {SMEM_BYTES_PER_CLK} B per SM per clock x {sms} SMs x {mhz:.0f} MHz",
        "what": "S2 bytes (one pass over the segment bitmap per level per segment) / hard-leaf kernels' time; "
                "the kernel keeps chunk counters instead of sweeping, so this counts work it does not do"}
    main = max(rows, key=lambda n: rows[n]["kernel_ms"])
    roof = dict(rows[main])
    roof["other"] = rows["k_easy" if main == "k_hard_shared" else "k_hard_shared"]
    tot = statistics.median(dev_ms)
    names = sorted({n for k in kern for n in k})
    shares = {n: {"ms": statistics.median(k.get(n, 0.0) for k in kern),
                  "share": statistics.median(k.get(n, 0.0) for k in kern) / tot} for n in names}
    return roof, shares


def cpu_baseline(xs, budget_s):
    import oracle

    nthreads = os.cpu_count() or 1
    done, t0 = 0, time.perf_counter()
    for x in xs:
        y = oracle.default_y(x, *alpha_frac(x))
        oracle.pi_dr(x, y, 6, nthreads)
        done += 1
        if time.perf_counter() - t0 > budget_s:
            break
    dt = time.perf_counter() - t0
    return {"value": done / dt, "unit": UNIT, "cores": nthreads, "kind": "port",
            "sample": f"first {done} of the {len(xs)} workload queries (x log-uniform in [1e9, 1e14]), "
                      f"oracle/oracle.c orc_pi_dr, OpenMP {nthreads} threads, {dt:.1f} s",
            "reference_terms": reference_terms_baseline(xs, budget_s / 3)}


def reference_terms_baseline(xs, budget_s):
    """The reference's only CPU term code, Gourdon's sums A and C
    (src/Gourdon/A2_cpu.cpp:20-134, src/Gourdon/C_cpu.cpp:20-78, restated in
    oracle/oracle.c with the same OpenMP loops), on a bounded sample of the
    workload with the reference alpha.  Two terms per query, not pi(x): the
    reference's pi(x) through these terms is unfinished
    (src/Gourdon/gourdonvariant.cpp:37-75 returns 0)."""
    import oracle

    nthreads = os.cpu_count() or 1
    done, t0 = 0, time.perf_counter()
    for x in xs:
        y = oracle.default_y(x, *alpha_frac(x))
        oracle.gourdon_A(x, y, nthreads)
        oracle.gourdon_C(x, y, nthreads)
        done += 1
        if time.perf_counter() - t0 > budget_s:
            break
    dt = time.perf_counter() - t0
    return {"value": done / dt, "unit": "queries/s (terms A and C only)", "cores": nthreads, "kind": "port",
            "terms": "Gourdon A (src/Gourdon/A2_cpu.cpp:20-134) + C (src/Gourdon/C_cpu.cpp:20-78)",
            "sample": f"first {done} of the {len(xs)} workload queries, oracle/oracle.c orc_gourdon_A + "
                      f"orc_gourdon_C, OpenMP {nthreads} threads, {dt:.1f} s"}


def alpha_frac(x):
    # the reference's alpha(x) (src/main.cpp:128-194) from the oracle, as num/den;
    # the CPU arms load no product library
    import oracle

    return oracle.alpha_milli(x), 1000


def target_ratio(cpx, ctx, args):
    """Batched vs plain queries/s for x log-uniform in [1e10, 1e15] (1024
    queries, numpy default_rng(0)); the plain path on the first 128."""
    xs = workload(1024, seed=0, lo=10.0, hi=15.0)
    ref = cpx.pi_batch(xs, ctx=ctx)
    want = golden_answers("batch_1e10_1e15.json", xs)
    assert want is None or ref == want, "batch answers differ from the oracle's"
    dev = []
    for _ in range(3):
        ctx.flush_l2()
        ctx.timer_start()
        assert cpx.pi_batch(xs, ctx=ctx) == ref
        dev.append(ctx.timer_stop())
    for x in xs[:128]:  # warm: buffers sized for lone queries
        cpx.pi_deleglise_rivat(x, 0, 6, ctx=ctx)
    lat = []
    for x, r in zip(xs[:128], ref):
        ctx.timer_start()
        assert cpx.pi_deleglise_rivat(x, 0, 6, ctx=ctx) == r
        lat.append(ctx.timer_stop())
    b = len(xs) / (statistics.median(dev) / 1000.0)
    p = len(lat) / (sum(lat) / 1000.0)
    return {"workload": "1024 x = floor(10^e), e ~ U[10,15], default_rng(0); plain on the first 128",
            "checked_against_oracle": want is not None, "batch_e2e_qps": b, "plain_qps": p, "ratio": b / p}


def serve_sweep(cpx, ctx, args):
    """Continuous batching (cpx_serve_*) under Poisson arrivals: x = floor(10^e),
    e ~ U[10, 17], gaps ~ Exp(1/lambda), both from numpy default_rng(1).  Per
    rate: p50/p99 latency from arrival to result and completed queries/s; the
    plain path's service rate on the same x mix beside it.  Every answer is
    checked against the same x answered alone."""
    rng = np.random.default_rng(1)
    pool = [int(10.0**e) for e in rng.uniform(10, 17, 400)]
    truth = dict(zip(pool, cpx.pi_batch(pool, ctx=ctx)))
    # plain per-query path on the same distribution (one warm pass first)
    for x in pool[:48]:
        cpx.pi_deleglise_rivat(x, 0, 6, ctx=ctx)
    lat = []
    for x in pool[:48]:
        ctx.timer_start()
        assert cpx.pi_deleglise_rivat(x, 0, 6, ctx=ctx) == truth[x]
        lat.append(ctx.timer_stop())
    lat.sort()
    plain = {"qps": len(lat) / (sum(lat) / 1000.0), "p50_ms": lat[len(lat) // 2], "p99_ms": lat[-1],
             "queries": len(lat)}
    rows = []
    own = tuned_context(cpx, ctx.device)
    with cpx.Server(own, lanes=args.serve_lanes, reserve_x=10**17) as srv:
        for lam in (10.0, 100.0, 1000.0, 10000.0):
            n = int(min(len(pool), max(30, 3 * lam)))
            gaps = rng.exponential(1.0 / lam, n)
            xs = pool[:n]
            t0 = time.perf_counter()
            got, ls = srv.replay(xs, np.cumsum(gaps).tolist())
            wall = time.perf_counter() - t0
            assert got == [truth[x] for x in xs], "served answer differs from the standalone answer"
            ls = sorted(ls)
            rows.append({"lambda": lam, "requests": n, "p50_ms": ls[len(ls) // 2],
                         "p99_ms": ls[min(len(ls) - 1, int(0.99 * len(ls)))], "qps": n / wall})
        st = srv.stats()
    own.close()
    return {"workload": "x = floor(10^e), e ~ U[10,17]; Poisson arrivals; default_rng(1)",
            "lanes": args.serve_lanes, "rates": rows, "plain": plain,
            "batches": st["batches"], "max_batch_seen": st["max_batch_seen"]}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    return world, rank, local


def allmax(v, world):
    if world == 1:
        return v
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(v)], device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def arm_config(args, world):
    """The workload both arms report (the reference arm runs it on the host cores)."""
    return {"workload": "batch4096: x = floor(10^e), e ~ U[9,14], numpy default_rng(0)",
            "queries": args.queries, "c": 6,
            "alpha": "tuning table: 0.094 of the reference alpha(x) (y >= icbrt x) for queries with 16 or more "
                     "others within half a decade of x, else the decade's tuned alpha",
            "l2": "flushed before every timed step (256 MiB write)",
            "tuning": os.path.relpath(TUNING, ROOT) if os.path.exists(TUNING) else None,
            "parallelism": f"replicas x{world}"}


def run_reference(args, world, rank):
    if rank != 0:
        return
    xs = workload(args.queries)
    nthreads = os.cpu_count() or 1
    import oracle

    per_step = []
    sample = None
    # each step a bounded sample of the workload: the whole run stays within a
    # few minutes whatever --steps / --warmup ask for
    step_s = args.ref_step_s or max(2.0, min(20.0, 150.0 / (args.warmup + args.steps)))
    for k in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        done = 0
        for x in xs:
            oracle.pi_dr(x, oracle.default_y(x, *alpha_frac(x)), 6, nthreads)
            done += 1
            if time.perf_counter() - t0 > step_s:
                break
        dt = time.perf_counter() - t0
        if k >= args.warmup:
            per_step.append((done, dt))
        sample = (f"per step the first {done} of the {len(xs)} workload queries ({step_s:.1f} s), "
                  f"oracle/oracle.c orc_pi_dr, OpenMP {nthreads} threads")
    q = sum(d for d, _ in per_step)
    t = sum(s for _, s in per_step)
    v = q / t
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000 * t / len(per_step), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int64/int128", "data": "synthetic",
            "config": arm_config(args, world),
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": nthreads, "kind": "port", "sample": sample,
                             "reference_terms": reference_terms_baseline(xs, step_s)},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_single(args, world, rank, local):
    """One query of size --single (e.g. 1e15 or 1e17) with y = alpha * icbrt(x):
    latency per query through the plain API, term by term timing of the hard leaves."""
    import cudapix_b200 as cpx

    ctx = tuned_context(cpx, local)
    ctx.set_timing(True)
    x = int(float(args.single)) if "e" in args.single.lower() else int(args.single)
    y = cpx.default_y(x, args.alpha) if args.alpha else 0
    ref = None
    for _ in range(args.warmup):
        t = cpx.pi_terms(x, y, 6, ctx=ctx)
        ref = ref or t
        assert t == ref
    lat, hard = [], []
    with Clocks(local) as clk:
        for _ in range(args.steps):
            ctx.flush_l2()
            ctx.timer_start()
            t = cpx.pi_terms(x, y, 6, ctx=ctx)
            lat.append(ctx.timer_stop())
            hard.append(ctx.last_hard_stats())
            assert ref is None or t == ref
    if rank != 0:
        return
    ms = statistics.median(lat)
    hm, hb = hard[-1]
    leaves = cpx.leaf_counts(x, t["y"], 6, ctx=ctx)
    print(json.dumps({"metric": "pi(x) single-query latency", "value": ms, "unit": "ms", "n_gpus": world,
                      "steps": args.steps, "warmup": args.warmup, "higher_is_better": False,
                      "config": {"workload": f"single x={x} y={t['y']} z={t['z']} c=6", "alpha": args.alpha},
                      "pi": t["pi"], "terms": {k: t[k] for k in ("P2", "ordinary", "trivial", "easy", "hard")},
                      "hard_ms": hm, "s2_gbs": (hb / (hm / 1000)) / 1e9 if hm else None,
                      "leaves": leaves, "hard_leaves_per_s": leaves["hard"] / (hm / 1000) if hm else None,
                      "batch_device_ms": ctx.last_batch_ms(), "clocks": clk.summary()}), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--single", default=None, help="time one query of this size instead of the batch")
    ap.add_argument("--alpha", type=float, default=0.0, help="y = alpha * icbrt(x) for --single (0: reference alpha)")
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--queries", type=int, default=4096)
    ap.add_argument("--plain", type=int, default=256, help="queries timed through the plain per-query path")
    ap.add_argument("--cpu-budget", type=float, default=15.0)
    ap.add_argument("--ref-step-s", type=float, default=0.0,
                    help="seconds of CPU work per reference step (0: 150 s over all steps, 2..20 s each)")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--graph", type=int, default=1, help="also time the batch as one CUDA graph launch")
    ap.add_argument("--serve", type=int, default=1, help="serving sweep and the [1e10,1e15] target check")
    ap.add_argument("--serve-lanes", type=int, default=1)
    args = ap.parse_args()
    world, rank, local = dist_setup()
    # no collector passes inside the timed host-driven launch sequences (a
    # pass over the workload's integer lists would land in a CUDA-event interval)
    gc.collect()
    gc.disable()
    if args.impl == "reference":
        run_reference(args, world, rank)
        return
    if args.single:
        run_single(args, world, rank, local)
        return

    import cudapix_b200 as cpx

    ctx = tuned_context(cpx, local)
    ctx.set_timing(True)
    xs = workload(args.queries, seed=0)
    ref = golden_answers("batch_seed0.json", xs)  # the oracle's answers, when committed for these queries
    checked = ref is not None
    for _ in range(max(args.warmup, 3)):
        out = cpx.pi_batch(xs, ctx=ctx)
        if ref is None:
            ref = out
        assert out == ref, "batch answers differ from the oracle's" if checked else "batch results changed between runs"

    # plain path: one full launch sequence per query, on a fixed subsample (before the
    # clock sampler of the timed batches starts polling the driver)
    plain = None
    if args.plain and rank == 0:
        sub = xs[: args.plain]
        for x in sub:  # warm: buffers sized for lone queries
            cpx.pi_deleglise_rivat(x, 0, 6, ctx=ctx)
        lat = []
        for x in sub:
            ctx.timer_start()
            p = cpx.pi_deleglise_rivat(x, 0, 6, ctx=ctx)
            lat.append(ctx.timer_stop())
            assert p == ref[xs.index(x)]
        lat.sort()
        plain = {"value": len(sub) / (sum(lat) / 1000.0), "unit": UNIT, "queries": len(sub),
                 "p50_ms": lat[len(lat) // 2], "p99_ms": lat[min(len(lat) - 1, int(len(lat) * 0.99))]}

    launches0 = ctx.launches
    dev_ms, e2e_ms, hard_ms, hard_bytes, host_stats, kern = [], [], [], [], [], []
    barrier(world)
    with Clocks(local) as clk:
        for _ in range(args.steps):
            ctx.flush_l2()
            ctx.timer_start()
            out = cpx.pi_batch(xs, ctx=ctx)
            e2e_ms.append(ctx.timer_stop())
            dev_ms.append(ctx.last_batch_ms())
            hm, hb = ctx.last_hard_stats()
            hard_ms.append(hm)
            hard_bytes.append(hb)
            host_stats.append(ctx.last_batch_stats())
            kern.append(ctx.last_kernel_ms())
            assert out == ref
    barrier(world)
    import ctypes

    h2d, d2h = ctypes.c_uint64(), ctypes.c_uint64()
    ctx.call("cpx_last_batch_io", ctypes.byref(h2d), ctypes.byref(d2h))
    io = (h2d.value, d2h.value)
    launches = (ctx.launches - launches0) // args.steps
    t_dev = allmax(sum(dev_ms) / 1000.0, world)
    t_e2e = allmax(sum(e2e_ms) / 1000.0, world)
    nq = world * args.queries * args.steps
    value = nq / t_dev

    # the same batch as one CUDA graph launch (CPX_BATCH_GRAPH), e2e through the C ABI
    graph = None
    if args.graph:
        for _ in range(2):
            assert cpx.pi_batch(xs, ctx=ctx, graph=True) == ref
        g_e2e, g_dev = [], []
        for _ in range(args.steps):
            ctx.flush_l2()
            ctx.timer_start()
            out = cpx.pi_batch(xs, ctx=ctx, graph=True)
            g_e2e.append(ctx.timer_stop())
            g_dev.append(ctx.last_batch_ms())
            assert out == ref
        gt_dev = allmax(sum(g_dev) / 1000.0, world)
        gt_e2e = allmax(sum(g_e2e) / 1000.0, world)
        graph = {"value": nq / gt_dev, "e2e": nq / gt_e2e, "unit": UNIT}

    target = None
    serving = None
    if rank == 0 and args.serve:
        target = target_ratio(cpx, ctx, args)
        serving = serve_sweep(cpx, ctx, args)
    if rank != 0:
        return
    clocks = clk.summary()
    roof, shares = roofline(kern, hard_ms, hard_bytes, dev_ms, clocks, ctx)
    cpu = None if args.no_cpu else cpu_baseline(xs, args.cpu_budget)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": max(args.warmup, 3), "ms_per_step": 1000 * t_dev / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int64/int128", "data": "synthetic",
        "config": arm_config(args, world),
        "checked_against_oracle": checked,
        "e2e": {"value": nq / t_e2e, "unit": UNIT, "h2d_bytes_per_step": io[0], "d2h_bytes_per_step": io[1]},
        "gpu_launches": int(launches),
        "host_ms": {k: round(statistics.median(h[k] for h in host_stats), 3)
                    for k in ("roots_ms", "tables_ms", "plan_ms", "launch_ms", "wait_ms")},
        "graph": graph,
        "target_1e10_1e15": target,
        "serving": serving,
        "plain": plain,
        "batched_over_plain": (value / plain["value"]) if plain else None,
        "e2e_over_plain": ((nq / t_e2e) / plain["value"]) if plain else None,
        "s2_gbs": (hard_bytes[-1] / (statistics.median(hard_ms) / 1000.0)) / 1e9 if statistics.median(hard_ms) else None,
        "kernel_ms": shares,
        "roofline": roof,
        "cpu_baseline": cpu,
        "clocks": clocks,
    }
    print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


if __name__ == "__main__":
    main()
