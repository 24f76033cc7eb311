"""GPU parity of the sieves and tables against the oracle and golden vectors.
Bit-exact (integer work)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_mu_lpf_golden(ctx, cpx, golden):
    for key in ("mu_lpf_window", "mu_lpf_low"):
        g = golden[key]
        assert cpx.gen_h_mu(g["lo"], g["hi"], ctx=ctx).tolist() == g["mu"]
        assert cpx.gen_h_lpf(g["lo"], g["hi"], ctx=ctx).tolist() == g["lpf"]


@pytest.mark.parametrize("lo,hi", [(0, 2), (0, 10), (0, 1 << 20), (123456, 123456 + 50000),
                                   (1 << 31, (1 << 31) + 40000), (4294967296 - 20000, 4294967296)])
def test_mu_lpf_vs_oracle(ctx, cpx, orc, lo, hi):
    mu_o, lpf_o = orc.mu_lpf(lo, hi)
    assert np.array_equal(cpx.gen_h_mu(lo, hi, ctx=ctx), mu_o)
    assert np.array_equal(cpx.gen_h_lpf(lo, hi, ctx=ctx), lpf_o)
    d = cpx.gen_d_mu(lo, hi, ctx=ctx)
    assert np.array_equal(d.to_host(), mu_o)


def test_lpf64_above_2_32(ctx, cpx):
    lo, hi = (1 << 40), (1 << 40) + 4096
    lpf = cpx.gen_d_lpf(lo, hi, wide=True, ctx=ctx).to_host()
    mu, lpf2 = cpx.gen_d_mu_lpf(lo, hi, ctx=ctx)
    lpf2 = lpf2.to_host()
    mu = mu.to_host()
    assert np.array_equal(lpf, lpf2)
    for i in range(0, 2048, 37):
        n = lo + 2 * i + 1
        p = int(lpf[i])
        assert n % p == 0
        for d in range(3, min(p, 2000), 2):
            assert n % d != 0
    # mu by trial factorisation for a few entries
    for i in range(0, 2048, 97):
        n, m, f, sq = lo + 2 * i + 1, 1, 3, False
        k = n
        while f * f <= k:
            if k % f == 0:
                k //= f
                if k % f == 0:
                    sq = True
                    break
                m = -m
            f += 2
        if not sq and k > 1:
            m = -m
        assert int(mu[i]) == (0 if sq else m), n


def test_mutest(ctx, cpx, golden, orc):
    for top, m in golden["mertens"]:
        assert cpx.mutest(top, ctx=ctx) == m
    for top in (10**6, 10**7 + 3):
        assert cpx.mutest(top, ctx=ctx) == orc.mertens(top)


def test_dense_pitable(ctx, cpx, orc):
    for hi in (2, 3, 100, 65536, 10**6 + 2):
        t = cpx.get_d_piTable(hi, ctx=ctx).to_host()
        assert np.array_equal(t, orc.pitable_dense(hi))


@pytest.mark.parametrize("base,rng", [(0, 1000), (2, 100), (10**6, 10**5), (10**12, 1 << 20), (1 << 40, 5000)])
def test_window_pitable(ctx, cpx, orc, base, rng):
    pt = cpx.PiTable(base, 0, rng, ctx=ctx)
    t = pt.getCurrent().to_host()
    if base < 10**9:
        to, pb = orc.pitable_window(base, rng)
        assert pt.pi_base == pb
        assert np.array_equal(t, to)
    else:
        # relative counts against oracle prime lists
        ps = orc.primes(base, base + rng + 4)
        for k in (1, 3, 999, rng // 2 + 1):
            n = base + 2 * k - 1
            assert int(t[k]) == int(np.sum(ps <= n))


def test_pitable_walk(ctx, cpx, orc):
    pt = cpx.PiTable(2_000_000, 1_000_000, 200_000, ctx=ctx)
    pt.getCurrent()
    b0 = pt.get_base()
    t = pt.getNextDown().to_host()
    assert pt.get_base() == b0 - 200_000
    assert pt.pi_base == orc.pi_sieve(pt.get_base() - 1)
    assert t[5] + pt.pi_base == orc.pi_sieve(pt.get_base() + 9)
    t = pt.getNextUp().to_host()
    assert pt.get_base() == b0
    assert t[77] + pt.pi_base == orc.pi_sieve(b0 + 153)


def test_pitable_pi_base_and_buffers(ctx, cpx, orc):
    pt = cpx.PiTable(2_000_000, 1_000_000, 100_000, ctx=ctx)
    want = orc.pi_sieve(1_999_999)
    assert pt.get_pi_base() == want  # counted before any window is filled
    pt.set_pi_base(want)  # a caller's value is kept for this base
    assert pt.get_pi_base() == want
    pt.set_base(1_500_000)
    assert pt.get_pi_base() == orc.pi_sieve(1_499_999)  # a new base is counted again
    buf = pt._buf.ptr
    pt.allocate()
    assert pt._buf.ptr == buf  # allocate() keeps an existing buffer
    pt.reallocate()
    t = pt.getCurrent().to_host()
    assert pt.pi_base == orc.pi_sieve(1_499_999)
    assert t[7] + pt.pi_base == orc.pi_sieve(1_500_013)


@pytest.mark.parametrize("lo,hi", [(0, 100), (0, 2), (2, 3), (90, 97), (10**9, 10**9 + 10**6), (10**13, 10**13 + 10**5)])
def test_primes_and_counts(ctx, cpx, orc, lo, hi):
    p = cpx.get_device_primes(lo, hi, ctx=ctx).to_host()
    assert np.array_equal(p, orc.primes(lo, hi))
    assert cpx.count_primes(lo, hi, ctx=ctx) == len(p)


def test_count_primes_golden(ctx, cpx, golden):
    for x, p in golden["pi_random"]:
        assert cpx.count_primes(0, x + 1, ctx=ctx) == p
    for k in range(1, 11):
        assert cpx.count_primes(0, 10**k + 1, ctx=ctx) == golden["pi_pow10"][str(k)]


def test_phi_golden(ctx, cpx, golden):
    ph = cpx.Phi(10**6, ctx=ctx)
    for x, a, v in golden["phi"]:
        assert ph.phi_std(x, a) == v, (x, a)


def test_phi_large(ctx, cpx, orc):
    ph = cpx.Phi(0, ctx=ctx)
    for x, a in [(10**9, 10), (10**9 + 7, 100), (3 * 10**8, 1000), (2**32 + 5, 5)]:
        assert ph.phi_std(x, a) == orc.phi(x, a)
    # reference index convention: phi(x, a) excludes the first a + 1 primes
    assert ph.phi(10**6, 0) == orc.phi(10**6, 1)


def test_phi_range(ctx, cpx, orc):
    ph = cpx.Phi(0, ctx=ctx)
    t = ph.generateRange(100000, 5).to_host()  # a = 5 -> first 6 primes
    for i in (0, 1, 2, 10, 49999):
        assert int(t[i]) == orc.phi(2 * i + 1, 6)


def test_phi_getters_and_phisieve_set_a(ctx, cpx, orc):
    ph = cpx.Phi(10**6, ctx=ctx)
    _, lpf_o = orc.mu_lpf(0, 10**6)
    assert np.array_equal(ph.get_d_lpf().to_host(), lpf_o)
    pl = ph.get_h_primeList()  # primes 41 .. isqrt(10^6), after the 12 small primes
    assert pl[0] == 41 and pl[-1] == 997 and ph.get_primeListLength() == 168 - 12
    assert np.array_equal(ph.get_d_primeList().to_host(), pl)
    ph.makeModCache(8)
    assert ph.phi(10**5, 5) == orc.phi(10**5, 6)
    ps = cpx.Phisieve(1000, 1 << 16, ctx=ctx)
    ps.firstSieve(6)
    ps.set_a_current(6)  # as it was: the next markNext crosses off p_7 = 17
    ps.markNext()
    ps.updateCount()
    assert np.array_equal(ps.getCountHost(), orc.phisieve_counts(7, 1 << 16))
    ps.set_a_current(3)
    assert ps.get_a_current() == 3


def test_phisieve(ctx, cpx, orc):
    ps = cpx.Phisieve(1000, 1 << 16, ctx=ctx)
    ps.firstSieve(6)
    cnt = ps.getCountHost()
    assert np.array_equal(cnt, orc.phisieve_counts(6, 1 << 16))
    for _ in range(3):
        ps.markNext()
    ps.updateCount()
    assert ps.get_a_current() == 9
    assert np.array_equal(ps.getCountHost(), orc.phisieve_counts(9, 1 << 16))
