"""Generate tests/golden/golden.json.

Independent known-answer vectors for the oracle and the CUDA library:
  * pi(10^k), k = 1..20 -- published values, OEIS A006880;
  * pi(x) at seeded random x <= 2e8           -- sympy.primepi;
  * Mertens sums M(top - 1) at several tops     -- sympy.mobius, summed here;
  * mu(n) and lpf(n) for the odd n of a window  -- sympy.factorint;
  * phi(x, a) for small x                        -- brute force from sympy's primes.
The reference (curtisseizert/CUDApix) ships no golden vectors of its own, so
these are the pins.  Run:  python tests/golden/make_golden.py
"""
import json
import os
import random

import sympy

OEIS_A006880 = {
    1: 4,
    2: 25,
    3: 168,
    4: 1229,
    5: 9592,
    6: 78498,
    7: 664579,
    8: 5761455,
    9: 50847534,
    10: 455052511,
    11: 4118054813,
    12: 37607912018,
    13: 346065536839,
    14: 3204941750802,
    15: 29844570422669,
    16: 279238341033925,
    17: 2623557157654233,
    18: 24739954287740860,
    19: 234057667276344607,
    20: 2220819602560918840,
}


def lpf(n):
    if n == 1:
        return 0xFFFFFFFF
    return min(sympy.factorint(n))


def mu(n):
    return int(sympy.mobius(n))


def main():
    rng = random.Random(20161208)
    out = {"source": "tests/golden/make_golden.py", "sympy": sympy.__version__}
    out["pi_pow10"] = {str(k): v for k, v in OEIS_A006880.items()}
    xs = sorted({rng.randrange(2, 200_000_000) for _ in range(40)} | {2, 3, 4, 5, 100, 65535, 65536, 65537})
    out["pi_random"] = [[x, int(sympy.primepi(x))] for x in xs]
    # Mertens: sum_{1 <= n < top} mu(n)  (src/mutest.cu:6-19 semantics)
    tops = [1, 2, 10, 100, 1000, 10_000, 65_537, 100_000, 250_000]
    mus = [0] + [mu(n) for n in range(1, max(tops))]
    acc, pref = 0, [0]
    for n in range(1, max(tops)):
        acc += mus[n]
        pref.append(acc)
    out["mertens"] = [[t, pref[t - 1] if t >= 1 else 0] for t in tops]
    # mu / lpf of odd n = lo + 2i + 1 over a window
    lo = 1_000_000_000
    win = [lo + 2 * i + 1 for i in range(2048)]
    out["mu_lpf_window"] = {"lo": lo, "hi": lo + 4096, "mu": [mu(n) for n in win], "lpf": [lpf(n) for n in win]}
    lo0 = 0
    win0 = [lo0 + 2 * i + 1 for i in range(4096)]
    out["mu_lpf_low"] = {"lo": lo0, "hi": lo0 + 8192, "mu": [mu(n) for n in win0], "lpf": [lpf(n) for n in win0]}
    # phi(x, a) by brute force
    P = list(sympy.primerange(2, 200))
    phis = []
    for _ in range(60):
        x = rng.randrange(0, 300_000)
        a = rng.randrange(0, 30)
        bad = P[:a]
        cnt = sum(1 for n in range(1, x + 1) if all(n % p for p in bad))
        phis.append([x, a, cnt])
    out["phi"] = phis
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden.json")
    with open(path, "w") as f:
        json.dump(out, f, separators=(",", ":"))
    print("wrote", path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
