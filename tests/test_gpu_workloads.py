"""The benchmark workloads and the single-query sweeps, checked against
committed oracle answers (tests/golden/make_config_golden.py):

* the 4096-query batch (x = floor(10^e), e ~ U[9, 14], numpy default_rng(0))
  with the committed B200 tuning table, which runs it at 1/8 of the
  reference alpha(x) on the shared sieve, launched directly and as one CUDA
  graph: every answer equal to the oracle's;
* the 1024-query batch (e ~ U[10, 15]), batched (direct and graph) and, on a
  subsample, one plain query per launch sequence;
* x = 10^15 with y = alpha icbrt(x), alpha in {8, 16, 24, 32}, and x = 10^17
  with alpha in {8, 32}: P2, ordinary, trivial, easy, hard and pi(y) term by
  term, the total against the published pi(10^k).

All exact integer results: tolerance zero."""
import json
import os

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
TUNING = os.path.join(ROOT, "cudapix_b200", "tuning", "b200.json")


def _load(name):
    with open(os.path.join(HERE, "golden", name)) as f:
        return json.load(f)


def _workload(n, lo, hi):
    import numpy as np

    e = np.random.default_rng(0).uniform(lo, hi, n)
    return [int(10.0**v) for v in e]


@pytest.mark.parametrize("name,n,lo,hi", [("batch_seed0.json", 4096, 9.0, 14.0),
                                           ("batch_1e10_1e15.json", 1024, 10.0, 15.0)])
def test_fixture_inputs_are_the_bench_workload(name, n, lo, hi):
    """The committed queries are the ones bench.py draws (same generator)."""
    g = _load(name)
    assert g["x"] == _workload(n, lo, hi)
    assert len(g["pi"]) == n


@pytest.fixture(scope="module")
def tuned(cpx):
    ctx = cpx.Context(0)
    ctx.tune_load(TUNING)
    yield ctx
    ctx.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["batch_seed0.json", "batch_1e10_1e15.json"])
def test_batch_workload_equals_oracle(cpx, tuned, name):
    g = _load(name)
    xs, want = g["x"], g["pi"]
    got = cpx.pi_batch(xs, ctx=tuned)
    bad = [(x, a, b) for x, a, b in zip(xs, got, want) if a != b]
    assert not bad, bad[:5]
    assert tuned.last_batch_stats()["shared_groups"] >= 1  # the shared sieve ran
    for _ in range(2):  # the graph is built, then updated in place
        assert cpx.pi_batch(xs, ctx=tuned, graph=True) == want


@pytest.mark.gpu
def test_plain_path_on_workload_subsample(cpx, tuned):
    g = _load("batch_1e10_1e15.json")
    for x, p in list(zip(g["x"], g["pi"]))[:48]:
        assert cpx.pi_deleglise_rivat(x, 0, 6, ctx=tuned) == p, x


SWEEP = _load("terms_sweep.json")["cases"] if os.path.exists(os.path.join(HERE, "golden", "terms_sweep.json")) else []


@pytest.mark.gpu
@pytest.mark.parametrize("case", SWEEP, ids=[f"1e{len(c['x']) - 1}-a{c['alpha']}" for c in SWEEP])
def test_sweep_terms_equal_oracle(cpx, ctx, golden, case):
    x, y = int(case["x"]), case["y"]
    assert y == cpx.default_y(x, case["alpha"])
    t = cpx.pi_terms(x, y, 6, ctx=ctx)
    for k in ("P2", "ordinary", "trivial", "easy", "hard", "pi_y", "pi"):
        assert t[k] == int(case[k]), (k, t[k], case[k])
    assert t["pi"] == golden["pi_pow10"][str(len(case["x"]) - 1)]
