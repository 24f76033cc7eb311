"""Gourdon's decomposition in the oracle.  The restatement of the reference's
OpenMP host terms (Gourdon's A and C, src/Gourdon/A2_cpu.cpp:20-134 and
src/Gourdon/C_cpu.cpp:20-78), which bench.py times as the reference's CPU path
for those terms, against the sums written out from their definitions over a
plain Python prime list; and pi(x) through the whole decomposition
A - B + C + D + Phi0 + Sigma against published and sympy values, a second
split of the leaves beside the Deleglise-Rivat one.  CPU only."""
import bisect
import math

import pytest


def _primes_upto(n):
    s = bytearray([1]) * (n + 1)
    s[0:2] = b"\x00\x00"
    for p in range(2, math.isqrt(n) + 1):
        if s[p]:
            s[p * p :: p] = bytes(len(range(p * p, n + 1, p)))
    return [i for i in range(n + 1) if s[i]]


def _icbrt(x):
    r = round(x ** (1 / 3))
    while r**3 > x:
        r -= 1
    while (r + 1) ** 3 <= x:
        r += 1
    return r


def _brute(x, y):
    """A and C from their definitions (p, q prime):
    A = sum_{x^(1/4) < p <= x^(1/3)} sum_{p < q <= sqrt(x/p)} chi(x/pq) pi(x/pq), chi = 2 below y;
    C = sum_{sqrt(y) < p <= x^(1/4)} sum_{x/p^3 < q <= y} [pi(x/pq) - pi(p) + 2]."""
    r4 = math.isqrt(math.isqrt(x))
    P = _primes_upto(max(math.isqrt(x), y) + 1)

    def pi(n):
        return bisect.bisect_right(P, n)

    A = 0
    for p in P[pi(r4) : pi(_icbrt(x))]:
        for q in P[pi(p) : pi(math.isqrt(x // p))]:
            u = x // (p * q)
            A += (2 if u < y else 1) * pi(u)
    C = 0
    for p in P[pi(math.isqrt(y)) : pi(r4)]:
        for q in P[pi(x // p**3) : pi(y)]:
            C += pi(x // (p * q)) - pi(p) + 2
    return A, C


CASES = [(10**6, 1), (10**8, 1), (10**8, 10), (123456789, 3), (10**10, 1), (10**10, 10),
         (30000000007, 7), (99999999977, 2)]


@pytest.mark.parametrize("x,alpha", CASES)
def test_gourdon_terms_match_definitions(orc, x, alpha):
    y = orc.default_y(x, alpha)
    A, C = _brute(x, y)
    assert orc.gourdon_A(x, y) == A, (x, y)
    assert orc.gourdon_C(x, y) == C, (x, y)


def test_gourdon_terms_thread_count(orc):
    x = 10**13 + 37
    y = orc.default_y(x, 5)
    assert orc.gourdon_A(x, y, 1) == orc.gourdon_A(x, y, 4)
    assert orc.gourdon_C(x, y, 1) == orc.gourdon_C(x, y, 4)


def test_gourdon_y_at_sqrt_edge(orc):
    # y close to sqrt(x): the C range (sqrt y, x^(1/4)] is nearly empty, A counts chi = 2 often
    x = 10**9 + 7
    y = math.isqrt(x) - 1
    A, C = _brute(x, y)
    assert orc.gourdon_A(x, y) == A
    assert orc.gourdon_C(x, y) == C


@pytest.mark.parametrize("k", range(6, 16))
def test_gourdon_pi_pow10(orc, golden, k):
    # alpha 1 puts x/y^2 above x^(1/4) (x* = x/y^2), alpha 30 below it
    x = 10**k
    for alpha in (1, 4, 30):
        y = orc.default_y(x, alpha)
        assert orc.pi_gourdon(x, y)["pi"] == golden["pi_pow10"][str(k)], (k, alpha)


def test_gourdon_pi_random(orc, golden):
    for i, (x, p) in enumerate(golden["pi_random"]):
        if x < 10**6:
            continue
        y = orc.default_y(x, (1, 3, 17)[i % 3])
        assert orc.pi_gourdon(x, y)["pi"] == p, x


def test_gourdon_terms_against_dr(orc):
    # y >= x^(3/8): x* = x^(1/4), the reference's own setting
    x = 10**12 + 39
    y = orc.default_y(x, 20)
    assert x // (y * y) <= math.isqrt(math.isqrt(x))
    g = orc.pi_gourdon(x, y)
    t = orc.pi_dr(x, y)
    assert g["D"] == t["hard"] and g["phi0"] == t["ordinary"]
    assert g["A"] == orc.gourdon_A(x, y)
    assert g["pi"] == t["pi"]


def test_gourdon_y_range_edges(orc):
    # y = floor(cbrt x) below the real cube root (x* stops at cbrt x, sqrt z lies above it)
    # and y just under sqrt x
    for x in (387452, 7164126, 13091049675, 10**11 + 3):
        p = orc.pi_lehmer(x)
        for y in (orc.icbrt(x), orc.icbrt(x) + 1, orc.isqrt(x) - 1):
            assert orc.pi_gourdon(x, y)["pi"] == p, (x, y)
