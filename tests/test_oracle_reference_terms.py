"""The restatement of the reference's OpenMP host terms (Gourdon's A and C,
src/Gourdon/A2_cpu.cpp:20-134 and src/Gourdon/C_cpu.cpp:20-78), which bench.py
times as the reference's CPU path for those terms, against the sums written
out from their definitions over a plain Python prime list.  CPU only."""
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
