"""The batch-shared hard-leaf sieve (one counting sweep for the carries, then
one sieve per group of up to 32 queries) against the oracle and against the
one-sieve-per-query path: bit-exact in every mode, segment size, block size,
offload threshold and group size."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CASES = [(10**9, 10**4), (10**10, 30000), (10**11, 46415 * 2), (10**12, 10**5), (999_999_999_989, 123457),
         (2**40 + 15, 10**5 + 3), (10**13, 172354)]


_HARD = {}


def oracle_hard(orc, x, y):
    if (x, y) not in _HARD:
        _HARD[(x, y)] = orc.hard(x, y, 6)
    return _HARD[(x, y)]


@pytest.fixture
def own(cpx):
    c = cpx.Context(0)
    yield c
    c.close()


@pytest.mark.parametrize("x,y", CASES)
def test_shared_single_query_vs_oracle(own, cpx, orc, x, y):
    """Mode 2 shares the sieve even for one query: carries from the counting
    sweep, leaves answered in the group kernel."""
    own.set_hard_shared(2)
    assert cpx.S2hard(x, y, 6, ctx=own) == orc.hard(x, y, 6), x
    t = cpx.pi_terms(x, y, 6, ctx=own)
    assert t["pi"] == orc.pi_dr(x, y, 6)["pi"], x


def test_shared_batch_terms_vs_oracle(own, cpx, orc):
    xs = [x for x, _ in CASES] + [10**11 + 3, 3 * 10**11, 7 * 10**10 + 1, 5 * 10**12]
    ys = [y for _, y in CASES] + [0, 0, 0, 0]
    got = cpx.terms_batch(xs, ys, ctx=own)
    assert own.last_batch_stats()["shared_groups"] >= 1
    for x, y, t in zip(xs, ys, got):
        yy = t["y"]
        assert t["hard"] == orc.hard(x, yy, 6), (x, yy)
        assert t["pi"] == orc.pi_dr(x, yy, 6)["pi"], x


def test_shared_equals_per_query_log_uniform(own, cpx):
    rng = np.random.default_rng(21)
    xs = [int(10**e) for e in rng.uniform(8, 13.5, 700)]
    own.set_hard_shared(0)
    ref = cpx.terms_batch(xs, ctx=own)
    assert own.last_batch_stats()["shared_groups"] == 0
    own.set_hard_shared(1)
    got = cpx.terms_batch(xs, ctx=own)
    assert own.last_batch_stats()["shared_groups"] > 1
    assert got == ref


@pytest.mark.parametrize("lbits,threads", [(15, 128), (16, 256), (18, 256), (18, 512), (20, 512), (17, 1024),
                                           (20, 1024)])
def test_shared_segment_sizes(own, cpx, lbits, threads):
    rng = np.random.default_rng(lbits * 1000 + threads)
    xs = [int(10**e) for e in rng.uniform(9, 12.5, 150)]
    own.set_hard_shared(0)
    ref = cpx.pi_batch(xs, ctx=own)
    own.set_hard_shared(2)
    assert cpx.pi_batch(xs, hard_log2_bits=lbits, hard_threads=threads, ctx=own) == ref


@pytest.mark.parametrize("off", [0, 1, 64, 1024])
def test_shared_offload_thresholds(own, cpx, orc, off):
    """Leaf sets sent to k_hard_leaves share one snapshot per (sub-segment,
    level); threshold 1 sends nearly every set there, 0 none."""
    xs = [10**10, 10**11, 2 * 10**11 + 7, 10**12, 10**12 + 39, 3 * 10**12, 10**11 + 1, 4 * 10**10 + 3, 10**13]
    own.set_hard_shared(2)
    own.set_hard_offload(off)
    for th in (128, 256, 512, 1024):
        got = cpx.terms_batch(xs, hard_threads=th, ctx=own)
        for x, t in zip(xs, got):
            assert t["hard"] == oracle_hard(orc, x, t["y"]), (off, th, x)


def test_shared_wide_kernels(own, cpx, orc):
    xs = [10**11, 2**40 + 15, 10**12, 3 * 10**13 + 7, 10**10 + 19, 10**12 + 39, 999_999_999_989, 5 * 10**11]
    own.set_hard_shared(2)
    got = cpx.terms_batch(xs, wide=True, ctx=own)
    for x, t in zip(xs, got):
        assert t["hard"] == oracle_hard(orc, x, t["y"]), x
    own.set_hard_shared(0)
    assert cpx.terms_batch(xs, wide=True, ctx=own) == got


@pytest.mark.parametrize("n", [1, 2, 31, 32, 33, 65])
def test_shared_group_sizes(own, cpx, n):
    """Partial and several groups, and batches small enough that the groups
    shrink below 32 queries."""
    rng = np.random.default_rng(n)
    xs = [int(10**e) for e in rng.uniform(10, 12.8, n)]
    own.set_hard_shared(0)
    ref = cpx.pi_batch(xs, ctx=own)
    own.set_hard_shared(2)
    assert cpx.pi_batch(xs, ctx=own) == ref
    assert cpx.pi_batch(xs, graph=True, ctx=own) == ref


def test_shared_pi_pow10(own, cpx, golden):
    own.set_hard_shared(2)
    xs = [10**k for k in range(1, 16)]
    assert cpx.pi_batch(xs, ctx=own) == [golden["pi_pow10"][str(k)] for k in range(1, 16)]


def test_1024_threads_outside_the_shared_sieve(own, cpx, orc):
    """A batch that does not share the sieve runs 1024-thread requests as 512."""
    own.set_hard_shared(0)
    xs = [10**11, 10**12 + 39]
    got = cpx.terms_batch(xs, hard_threads=1024, ctx=own)
    for x, t in zip(xs, got):
        assert t["hard"] == oracle_hard(orc, x, t["y"]), x


def test_shared_mode_argument(own, cpx):
    with pytest.raises(cpx.CpxError):
        own.set_hard_shared(3)


def test_batch_alpha_only_for_queries_with_companions(own, cpx):
    """Under the batch tuning a query with few neighbours in x (here one at
    1e16 among forty in [1e10, 1e11]) keeps its decade's tuned alpha, so it
    does not sieve a long interval alone; the results are the same as with
    one sieve per query."""
    import os

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    own.tune_load(os.path.join(root, "cudapix_b200", "tuning", "b200.json"))
    xs = [int(10**e) for e in np.random.default_rng(4).uniform(10, 11, 40)] + [10**16 + 1]
    got = cpx.terms_batch(xs, ctx=own)
    alone = cpx.terms_batch([10**16 + 1], ctx=own)[0]  # plain path: the decade's tuning
    assert got[-1]["y"] == alone["y"] and got[-1]["pi"] == alone["pi"]
    own.set_hard_shared(0)
    assert cpx.terms_batch(xs, ctx=own) == got


def test_shared_sieve_over_budget_replans_without_batch_alpha(own, cpx, tmp_path):
    """Seventeen queries near 1e18 have companions, but with 1024-thread
    blocks over 2^20-bit segments the batch alpha would give the shared
    sieve's counting sweep 22.5 GB of carry rows, above the 16 GiB budget: the
    batch is planned again with each decade's alpha (y as for the query alone;
    6.6 GB of rows, so the sieve is still shared) and the answers are exact."""
    import json
    import os

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    with open(os.path.join(root, "cudapix_b200", "tuning", "b200.json")) as f:
        tune = json.load(f)
    for e in tune["entries"]:
        if e["decade"] == 99:
            e["threads"], e["log2_bits"] = 1024, 20
    path = tmp_path / "tune.json"
    path.write_text(json.dumps(tune))
    own.tune_load(str(path))
    xs = [10**18 + k * 3 * 10**16 + 1 for k in range(17)]
    got = cpx.terms_batch(xs, ctx=own)
    assert own.last_batch_stats()["shared_groups"] >= 1
    for x, t in list(zip(xs, got))[::8]:
        alone = cpx.terms_batch([x], ctx=own)[0]
        assert t["y"] == alone["y"] and t["pi"] == alone["pi"], x


@pytest.mark.parametrize("c", [1, 2, 3, 5, 7, 8])
def test_shared_other_c(own, cpx, orc, c):
    """Pre-sieving p_2..p_c and sieving from level c+1 in the shared sieve,
    for every c the library takes: equal to one sieve per query, and to the
    oracle's hard leaves."""
    xs = [10**10 + 7, 3 * 10**10, 10**11, 2 * 10**11 + 1, 10**12, 7 * 10**11, 10**12 + 39, 4 * 10**11 + 3, 10**13]
    own.set_hard_shared(2)
    got = cpx.terms_batch(xs, c=c, ctx=own)
    own.set_hard_shared(0)
    assert cpx.terms_batch(xs, c=c, ctx=own) == got
    for x, t in list(zip(xs, got))[:3]:
        assert t["hard"] == orc.hard(x, t["y"], c), (c, x)
