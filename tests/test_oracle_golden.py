"""Pins the CPU oracle (the checker) to independent known answers:
published pi(10^k) (OEIS A006880) and sympy-generated vectors
(tests/golden/make_golden.py).  CPU only."""
import numpy as np
import pytest


def test_pi_sieve_pow10(orc, golden):
    for k in range(1, 10):
        assert orc.pi_sieve(10**k) == golden["pi_pow10"][str(k)]


def test_pi_sieve_random(orc, golden):
    for x, p in golden["pi_random"]:
        assert orc.pi_sieve(x) == p, x


def test_lehmer_pow10(orc, golden):
    for k in range(5, 13):
        assert orc.pi_lehmer(10**k) == golden["pi_pow10"][str(k)]


def test_lehmer_random(orc, golden):
    for x, p in golden["pi_random"][:20]:
        assert orc.pi_lehmer(x) == p


@pytest.mark.parametrize("k", range(6, 15))
def test_dr_identity_pow10(orc, golden, k):
    x = 10**k
    for alpha in (1, 4, 10):
        y = orc.default_y(x, alpha)
        t = orc.pi_dr(x, y)
        assert t["pi"] == golden["pi_pow10"][str(k)], (k, alpha, t)


def test_dr_identity_random(orc):
    rng = np.random.default_rng(7)
    for e in rng.uniform(6, 11, 12):
        x = int(10**e)
        y = orc.default_y(x, 3)
        assert orc.pi_dr(x, y)["pi"] == orc.pi_sieve(x)


def test_per_term_functions_match_dr(orc):
    x, y = 10**12, 10**5
    t = orc.pi_dr(x, y)
    assert orc.P2(x, y) == t["P2"]
    assert orc.trivial(x, y) == t["trivial"]
    assert orc.ordinary(x, y) == t["ordinary"]
    assert orc.easy(x, y) == t["easy"]
    assert orc.hard(x, y) == t["hard"]


def test_mertens(orc, golden):
    for top, m in golden["mertens"]:
        assert orc.mertens(top) == m, top


def test_mu_lpf_windows(orc, golden):
    for key in ("mu_lpf_window", "mu_lpf_low"):
        g = golden[key]
        mu, lpf = orc.mu_lpf(g["lo"], g["hi"])
        assert mu.tolist() == g["mu"]
        assert lpf.tolist() == g["lpf"]


def test_phi(orc, golden):
    for x, a, v in golden["phi"]:
        assert orc.phi(x, a) == v, (x, a)


def test_phisieve_counts(orc):
    for a in (1, 2, 6, 9):
        cnt = orc.phisieve_counts(a, 5000)
        for i in (1, 2, 17, 100, 4999):
            assert cnt[i] == orc.phi(2 * i - 1, a)


def test_pitable_dense(orc):
    t = orc.pitable_dense(20000)
    for k in (1, 2, 3, 100, 9999):
        assert t[k] == orc.pi_sieve(2 * k - 1)
    assert t[0] == 0


def test_pitable_window(orc):
    base, rng = 1_000_000, 10_000
    t, pb = orc.pitable_window(base, rng)
    assert pb == orc.pi_sieve(base - 1)
    for k in (1, 7, 500, rng // 2 + 1):
        assert t[k] + pb == orc.pi_sieve(base + 2 * k - 1)


def test_roots(orc):
    rng = np.random.default_rng(3)
    for _ in range(200):
        x = int(rng.integers(1, 2**62)) * int(rng.integers(1, 2**60))
        s, c, q = orc.isqrt(x), orc.icbrt(x), orc.iroot4(x)
        assert s * s <= x < (s + 1) ** 2
        assert c**3 <= x < (c + 1) ** 3
        assert q**4 <= x < (q + 1) ** 4
