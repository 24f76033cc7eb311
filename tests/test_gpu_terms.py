"""GPU parity of every Deleglise-Rivat term against the CPU oracle (bit-exact),
and of pi(x) against published pi(10^k) (OEIS A006880)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CASES = [
    (10**7, 400), (10**8, 2000), (10**9, 10**4), (10**10, 30000), (10**11, 46415 * 2),
    (10**12, 10**5), (999_999_999_989, 123457), (2**40 + 15, 10**5 + 3), (10**13, 172354),
]


@pytest.mark.parametrize("x,y", CASES)
def test_terms_vs_oracle(ctx, cpx, orc, x, y):
    t = cpx.pi_terms(x, y, 6, ctx=ctx)
    o = orc.pi_dr(x, y, 6)
    for k in ("P2", "ordinary", "trivial", "easy", "hard", "pi_y", "pi"):
        assert t[k] == o[k], (k, x, y, t[k], o[k])


@pytest.mark.parametrize("x,y", CASES[:6])
def test_single_term_entry_points(ctx, cpx, orc, x, y):
    assert cpx.P2(x, y, ctx=ctx) == orc.P2(x, y)
    assert cpx.S2_trivial(x, y, ctx=ctx) == orc.trivial(x, y)
    assert cpx.Ordinary(x, y, 6, ctx=ctx) == orc.ordinary(x, y, 6)
    assert cpx.S2_easy(x, y, ctx=ctx) == orc.easy(x, y)
    assert cpx.S2hard(x, y, 6, ctx=ctx) == orc.hard(x, y, 6)
    assert cpx.S2hard(x, y, 6, ctx=ctx, maxPrime=orc.iroot4(x)) == orc.hard(x, y, 6)


@pytest.mark.parametrize("c", [1, 2, 3, 4, 5, 7, 8])
def test_other_c(ctx, cpx, orc, c):
    x, y = 10**11, 10**4 * 5
    assert cpx.Ordinary(x, y, c, ctx=ctx) == orc.ordinary(x, y, c)
    assert cpx.S2hard(x, y, c, ctx=ctx) == orc.hard(x, y, c)
    assert cpx.S2_easy(x, y, c, ctx=ctx) == orc.easy(x, y, c)
    assert cpx.pi_deleglise_rivat(x, y, c, ctx=ctx) == 4118054813


def test_pi_pow10(ctx, cpx, golden):
    for k in range(1, 16):
        assert cpx.pi(10**k, ctx=ctx) == golden["pi_pow10"][str(k)], k


@pytest.mark.parametrize("alpha", [8, 16, 24, 32])
def test_pi_1e15_alpha_sweep(ctx, cpx, golden, alpha):
    y = cpx.default_y(10**15, alpha)
    assert cpx.pi_deleglise_rivat(10**15, y, 6, ctx=ctx) == golden["pi_pow10"]["15"]


def test_pi_random_small(ctx, cpx, golden):
    for x, p in golden["pi_random"]:
        assert cpx.pi(x, ctx=ctx) == p, x


def test_segment_params_do_not_change_results(ctx, cpx, orc):
    x, y = 10**12, 10**5
    ref = orc.hard(x, y)
    for lb, th in [(15, 128), (15, 256), (16, 512), (17, 256), (18, 256), (19, 512), (20, 256)]:
        ctx.set_hard_params(lb, th)
        assert cpx.S2hard(x, y, 6, ctx=ctx) == ref, (lb, th)
    ctx.set_hard_params(18, 256)


@pytest.mark.parametrize("x,y", [(10**9, 10**4), (10**10, 30000), (10**11, 92830), (10**12, 10**5)])
def test_hard_offload_threshold_does_not_change_results(ctx, cpx, orc, x, y):
    """Leaf sets answered by k_hard_leaves from snapshots (threshold 1 sends
    nearly every level there, 0 keeps every leaf in the sieve) give the same
    hard sum, for every block size."""
    ref = orc.hard(x, y)
    try:
        for off in (0, 1, 64, 1024):
            ctx.set_hard_offload(off)
            for th in (128, 256, 512):
                ctx.set_hard_params(18, th)
                assert cpx.S2hard(x, y, 6, ctx=ctx) == ref, (off, th)
    finally:
        ctx.set_hard_offload(1024)
        ctx.set_hard_params(18, 256)


def test_edge_y_bounds(ctx, cpx, orc):
    """y at the ends of the domain: y = icbrt(x) and y = isqrt(x) - 1."""
    for x in (10**10 + 1, 3 * 10**11, 2**36 - 1):
        s, c, _ = cpx.iroots(x)
        for y in (c, c + 1, s // 3, s - 1):
            t = cpx.pi_terms(x, y, 6, ctx=ctx)
            assert t["pi"] == orc.pi_sieve(x) if x < 10**11 else t["pi"] == orc.pi_dr(x, y)["pi"], (x, y)


def test_random_x_log_uniform(ctx, cpx, orc):
    rng = np.random.default_rng(5)
    for e in rng.uniform(7, 12.5, 20):
        x = int(10**e)
        y = cpx.default_y(x, 4)
        t = cpx.pi_terms(x, y, 6, ctx=ctx)
        o = orc.pi_dr(x, y, 6)
        assert t == {**o, "x": x, "y": y, "z": x // y, "c": 6}, x


def test_batch_equals_single(ctx, cpx, orc):
    rng = np.random.default_rng(0)
    xs = [int(10**e) for e in rng.uniform(3, 12, 300)] + [1, 2, 3, 10, 999_983, 10**6]
    got = cpx.pi_batch(xs, alpha=4, ctx=ctx)
    for x, g in zip(xs, got):
        if x <= 2 * 10**8:
            assert g == orc.pi_sieve(x), x
    # a few against single-query launches
    for x, g in list(zip(xs, got))[:40]:
        assert g == cpx.pi_deleglise_rivat(x, cpx.default_y(x, 4) if x >= 10**6 else 0, 6, ctx=ctx), x


def test_invalid_arguments(ctx, cpx):
    with pytest.raises(cpx.CpxError):
        cpx.Ordinary(10**12, 10**5, 9, ctx=ctx)
    with pytest.raises(cpx.CpxError):
        cpx.pi_deleglise_rivat(10**12, 10**3, 6, ctx=ctx)  # y below cbrt(x)
    with pytest.raises(cpx.CpxError):
        ctx.set_hard_params(21, 256)


def test_wide_kernels_match_oracle(ctx, cpx, orc):
    """The 128-bit kernels (u128 quotients, 128-bit accumulators) on x < 2^64,
    every term against the oracle, in one batch with per-query y."""
    cases = CASES + [(10**14, 600000), (3 * 10**13 + 7, 250001)]
    got = cpx.terms_batch([x for x, _ in cases], [y for _, y in cases], wide=True, ctx=ctx)
    for (x, y), t in zip(cases, got):
        o = orc.pi_dr(x, y, 6)
        for k in ("P2", "ordinary", "trivial", "easy", "hard", "pi_y", "pi"):
            assert t[k] == o[k], (k, x, y, t[k], o[k])


def test_wide_batch_equals_narrow(ctx, cpx):
    rng = np.random.default_rng(11)
    xs = [int(10**e) for e in rng.uniform(6, 13, 200)]
    assert cpx.pi_batch(xs, ctx=ctx, wide=True) == cpx.pi_batch(xs, ctx=ctx)


def test_terms_batch_equals_single(ctx, cpx):
    xs = [10**9 + 7, 10**11, 2**40 + 15, 10**12]
    ys = [0, 46415 * 2, 10**5 + 3, 0]
    got = cpx.terms_batch(xs, ys, ctx=ctx)
    for x, y, t in zip(xs, ys, got):
        assert t == cpx.pi_terms(x, y, 6, ctx=ctx), x


def test_graph_batches_equal_direct_launches(ctx, cpx, golden):
    """CUDA-graph batches: the first builds the graph, later ones of other
    sizes update it in place; every result equals the direct launches'."""
    rng = np.random.default_rng(3)
    for n, hi in ((300, 12), (57, 13.5), (300, 11), (1, 9)):
        xs = [int(10**e) for e in rng.uniform(6, hi, n)]
        assert cpx.pi_batch(xs, ctx=ctx, graph=True) == cpx.pi_batch(xs, ctx=ctx), (n, hi)
    pw = [10**k for k in range(1, 16)]
    assert cpx.pi_batch(pw, ctx=ctx, graph=True) == [golden["pi_pow10"][str(k)] for k in range(1, 16)]


@pytest.mark.parametrize("x,y", [(10**12, 10**5), (10**13, 172354), (2**40 + 15, 10**5 + 3)])
def test_p2_by_table_windows(cpx, orc, x, y):
    """P2 summed over pi-table windows (forced by a small resident-table bound:
    many windows of 2^20 integers) equals the oracle, and so does pi(x)."""
    own = cpx.Context(0)
    own.set_p2_window(1 << 20)
    t = cpx.pi_terms(x, y, 6, ctx=own)
    o = orc.pi_dr(x, y, 6)
    assert t["P2"] == o["P2"] and t["pi"] == o["pi"], (x, t["P2"], o["P2"])
    xs = [10**11, 10**12 + 39, 3 * 10**12]
    assert cpx.pi_batch(xs, ctx=own) == [orc.pi_dr(v, cpx.default_y(v), 6)["pi"] for v in xs]
    own.close()


@pytest.mark.parametrize("x,y,c", [(10**9, 10**4, 6), (10**10, 30000, 6), (10**12, 10**5, 6),
                                   (2**40 + 15, 10**5 + 3, 6), (10**11, 50000, 3)])
def test_leaf_counts(ctx, cpx, orc, x, y, c):
    """Exact leaf counts by class against the oracle's brute force; the four
    classes partition the special leaves."""
    assert cpx.leaf_counts(x, y, c, ctx=ctx) == orc.leaf_counts(x, y, c)
