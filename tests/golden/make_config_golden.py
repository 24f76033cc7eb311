"""Exact answers for the benchmark workloads and the per-term values of the
single-query sweeps, from the CPU oracle (oracle/oracle.c).

Writes beside this script:
  batch_seed0.json       the 4096 queries x = floor(10^e), e ~ U[9, 14] from
                         numpy default_rng(0) (the batch benchmark), and pi(x)
  batch_1e10_1e15.json   the 1024 queries x = floor(10^e), e ~ U[10, 15] from
                         default_rng(0) (the batched-vs-plain workload), and pi(x)
  terms_sweep.json       P2, ordinary, trivial, easy, hard, pi(y) and pi(x) of
                         x = 10^15 with y = alpha icbrt(x), alpha in {8, 16, 24, 32},
                         and x = 10^17 with alpha in {8, 32}

pi(x) of the workloads comes from the oracle's Deleglise-Rivat restatement
(orc_pi_dr, one thread per query over a process pool); a random subsample of
each workload is recomputed by the oracle's independent Lehmer count
(orc_pi_lehmer) and must agree.  The sweep's totals must equal the published
pi(10^15) and pi(10^17) (OEIS A006880).  About 15 minutes on 8 cores.

Usage: python tests/golden/make_config_golden.py [batch|sweep|all]
"""
import json
import multiprocessing as mp
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

PI_POW10 = {15: 29844570422669, 17: 2623557157654233}


def workload(n, seed, lo, hi):
    """x = floor(10^e), e ~ U[lo, hi) from numpy default_rng(seed)."""
    e = np.random.default_rng(seed).uniform(lo, hi, n)
    return [int(10.0**v) for v in e]


def _pi_one(x):
    import oracle

    return oracle.pi_dr(x, oracle.icbrt(x), 6, 1)["pi"]


def batch_file(name, n, lo, hi, check=48):
    import oracle

    xs = workload(n, 0, lo, hi)
    t = time.time()
    order = sorted(range(n), key=lambda i: -xs[i])  # largest first: even finish
    with mp.get_context("spawn").Pool(os.cpu_count()) as pool:
        vals = pool.map(_pi_one, [xs[i] for i in order], chunksize=1)
    pis = [0] * n
    for i, v in zip(order, vals):
        pis[i] = v
    rng = np.random.default_rng(12345)
    sub = sorted(rng.choice(n, check, replace=False).tolist())
    for i in sub:
        assert oracle.pi_lehmer(xs[i]) == pis[i], (i, xs[i])
    out = {"workload": f"x = floor(10^e), e ~ U[{lo:g}, {hi:g}), numpy default_rng(0), {n} queries",
           "method": "oracle orc_pi_dr (y = icbrt x, c = 6); Lehmer cross-check of the listed indices",
           "lehmer_checked": sub, "x": xs, "pi": pis, "seconds": round(time.time() - t, 1)}
    with open(os.path.join(HERE, name), "w") as f:
        json.dump(out, f, separators=(",", ":"))
    print(name, out["seconds"], "s", flush=True)


def sweep_file():
    import oracle

    cases = [(15, a) for a in (8, 16, 24, 32)] + [(17, a) for a in (8, 32)]
    rows = []
    for k, a in cases:
        x = 10**k
        y = oracle.default_y(x, a, 1)
        t = time.time()
        d = oracle.pi_dr(x, y, 6)
        assert d["pi"] == PI_POW10[k], (k, a, d["pi"])
        row = {"x": str(x), "alpha": a, "y": y, "c": 6}
        row.update({n: str(v) for n, v in d.items()})
        row["seconds"] = round(time.time() - t, 1)
        rows.append(row)
        print(row, flush=True)
    with open(os.path.join(HERE, "terms_sweep.json"), "w") as f:
        json.dump({"method": "oracle orc_pi_dr, y = alpha icbrt(x), c = 6; pi(x) equal to OEIS A006880",
                   "cases": rows}, f, indent=1)


def main():
    what = sys.argv[1] if len(sys.argv) > 1 else "all"
    if what in ("batch", "all"):
        batch_file("batch_seed0.json", 4096, 9.0, 14.0)
        batch_file("batch_1e10_1e15.json", 1024, 10.0, 15.0)
    if what in ("sweep", "all"):
        sweep_file()


if __name__ == "__main__":
    main()
