"""ctypes front end for the CPU oracle (oracle/oracle.c).

Test infrastructure only: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, as the checker.  The product library never
imports it.
"""
import ctypes
import os
import subprocess

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "liboracle.so")
_lib = None

U64 = ctypes.c_uint64
MASK64 = (1 << 64) - 1


def build():
    """Compile liboracle.so with the committed Makefile (gcc + OpenMP)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB) or os.path.getmtime(_LIB) < os.path.getmtime(
            os.path.join(_HERE, "oracle.c")
        ):
            build()
        L = ctypes.CDLL(_LIB)
        for name in ("orc_isqrt", "orc_icbrt", "orc_iroot4"):
            getattr(L, name).restype = U64
            getattr(L, name).argtypes = [U64, U64]
        L.orc_alpha_milli.restype = ctypes.c_uint32
        L.orc_alpha_milli.argtypes = [U64, U64]
        L.orc_pi_sieve.restype = U64
        L.orc_pi_sieve.argtypes = [U64]
        L.orc_pi_lehmer.restype = U64
        L.orc_pi_lehmer.argtypes = [U64]
        L.orc_primes.restype = U64
        L.orc_primes.argtypes = [U64, U64, ctypes.c_void_p, U64]
        L.orc_mu_lpf.restype = None
        L.orc_mu_lpf.argtypes = [U64, U64, ctypes.c_void_p, ctypes.c_void_p]
        L.orc_mertens.restype = ctypes.c_int64
        L.orc_mertens.argtypes = [U64]
        L.orc_pitable_dense.restype = None
        L.orc_pitable_dense.argtypes = [U64, ctypes.c_void_p]
        L.orc_pitable_window.restype = None
        L.orc_pitable_window.argtypes = [U64, U64, ctypes.c_void_p, ctypes.POINTER(U64)]
        L.orc_phi.restype = U64
        L.orc_phi.argtypes = [U64, ctypes.c_uint32]
        L.orc_phisieve_counts.restype = None
        L.orc_phisieve_counts.argtypes = [ctypes.c_uint32, U64, ctypes.c_void_p]
        for name in ("orc_P2", "orc_P2_windowed", "orc_trivial"):
            getattr(L, name).restype = None
            getattr(L, name).argtypes = [U64, U64, U64, ctypes.c_void_p]
        for name in ("orc_ordinary", "orc_hard", "orc_easy"):
            getattr(L, name).restype = None
            getattr(L, name).argtypes = [U64, U64, U64, ctypes.c_uint32, ctypes.c_void_p]
        L.orc_leaf_counts.restype = None
        L.orc_leaf_counts.argtypes = [U64, U64, U64, ctypes.c_uint32, ctypes.c_void_p]
        L.orc_pi_dr.restype = None
        L.orc_pi_dr.argtypes = [U64, U64, U64, ctypes.c_uint32, ctypes.c_int, ctypes.c_void_p]
        L.orc_pi_gourdon.restype = None
        L.orc_pi_gourdon.argtypes = [U64, U64, ctypes.c_uint32, ctypes.c_int, ctypes.c_void_p]
        for name in ("orc_gourdon_A", "orc_gourdon_C"):
            getattr(L, name).restype = None
            getattr(L, name).argtypes = [U64, U64, ctypes.c_int, ctypes.c_void_p]
        _lib = L
    return _lib


def _split(x):
    return x & MASK64, x >> 64


def _s128(lo, hi):
    v = (hi << 64) | lo
    return v - (1 << 128) if v >> 127 else v


def _call128(fn, *args):
    out = (U64 * 2)()
    fn(*args, out)
    return _s128(out[0], out[1])


def isqrt(x):
    return lib().orc_isqrt(*_split(x))


def icbrt(x):
    return lib().orc_icbrt(*_split(x))


def iroot4(x):
    return lib().orc_iroot4(*_split(x))


def alpha_milli(x):
    """The reference's alpha(x) (src/main.cpp:128-194) in per mille."""
    return lib().orc_alpha_milli(*_split(x))


def pi_sieve(x):
    return lib().orc_pi_sieve(x)


def pi_lehmer(x):
    return lib().orc_pi_lehmer(x)


def primes(lo, hi):
    import numpy as np

    cap = int(max(16, (hi - lo) // 2 + 16)) if hi - lo < 1 << 26 else 1 << 26
    out = np.zeros(cap, dtype=np.uint64)
    n = lib().orc_primes(lo, hi, out.ctypes.data, cap)
    assert n <= cap
    return out[:n]


def mu_lpf(lo, hi):
    import numpy as np

    n = (hi - lo) // 2
    mu = np.zeros(n, dtype=np.int8)
    lpf = np.zeros(n, dtype=np.uint32)
    lib().orc_mu_lpf(lo, hi, mu.ctypes.data, lpf.ctypes.data)
    return mu, lpf


def mertens(top):
    return lib().orc_mertens(top)


def pitable_dense(hi):
    import numpy as np

    out = np.zeros(hi // 2, dtype=np.uint32)
    lib().orc_pitable_dense(hi, out.ctypes.data)
    return out


def pitable_window(base, rng):
    import numpy as np

    out = np.zeros(rng // 2 + 2, dtype=np.uint32)
    pb = U64(0)
    lib().orc_pitable_window(base, rng, out.ctypes.data, ctypes.byref(pb))
    return out, pb.value


def phi(x, a):
    return lib().orc_phi(x, a)


def phisieve_counts(a, nbits):
    import numpy as np

    out = np.zeros(nbits, dtype=np.uint32)
    lib().orc_phisieve_counts(a, nbits, out.ctypes.data)
    return out


def P2(x, y):
    return _call128(lib().orc_P2, *_split(x), y)


def P2_windowed(x, y):
    """P2 with pi(x/p) from windows of 2^31 integers (no table to z); used
    for z beyond host memory and checked against P2 where both fit."""
    return _call128(lib().orc_P2_windowed, *_split(x), y)


def trivial(x, y):
    return _call128(lib().orc_trivial, *_split(x), y)


def ordinary(x, y, c=6):
    return _call128(lib().orc_ordinary, *_split(x), y, c)


def easy(x, y, c=6):
    return _call128(lib().orc_easy, *_split(x), y, c)


def hard(x, y, c=6):
    return _call128(lib().orc_hard, *_split(x), y, c)


TERM_NAMES = ("P2", "ordinary", "trivial", "easy", "hard", "pi_y", "pi")


def pi_dr(x, y, c=6, nthreads=0):
    """All DR terms for (x, y, c) as a dict; 'pi' is pi(x) by the term identity."""
    out = (U64 * 14)()
    lib().orc_pi_dr(*_split(x), y, c, nthreads, out)
    return {k: _s128(out[2 * i], out[2 * i + 1]) for i, k in enumerate(TERM_NAMES)}


def gourdon_A(x, y, nthreads=0):
    """Gourdon's A as the reference's OpenMP host code sums it
    (src/Gourdon/A2_cpu.cpp:20-134): over primes x^(1/4) < p <= x^(1/3) and
    p < q <= sqrt(x/p), chi(x/(pq)) pi(x/(pq)) with chi = 2 below y, else 1."""
    assert 0 < x < 1 << 64
    return _call128(lib().orc_gourdon_A, x, y, nthreads)


def gourdon_C(x, y, nthreads=0):
    """Gourdon's C as the reference's OpenMP host code sums it
    (src/Gourdon/C_cpu.cpp:20-78): over primes sqrt(y) < p <= x^(1/4) and
    x/p^3 < q <= y, pi(x/(pq)) - pi(p) + 2."""
    assert 0 < x < 1 << 64
    return _call128(lib().orc_gourdon_C, x, y, nthreads)


GOURDON_NAMES = ("A", "B", "C", "D", "phi0", "sigma", "pi")


def pi_gourdon(x, y, c=6, nthreads=0):
    """pi(x) through Gourdon's decomposition A - B + C + D + Phi0 + Sigma (the
    term names of src/Gourdon/gourdonvariant.hpp:7-56), with
    x* = max(x^(1/4), x/y^2); a second split of the leaves that the
    Deleglise-Rivat identity sums.  x < 2^64."""
    assert 0 < x < 1 << 64
    out = (U64 * 14)()
    lib().orc_pi_gourdon(x, y, c, nthreads, out)
    return {k: _s128(out[2 * i], out[2 * i + 1]) for i, k in enumerate(GOURDON_NAMES)}


def default_y(x, alpha_num=1, alpha_den=1):
    """y = floor(alpha * icbrt(x)) for a rational alpha (the rule of
    src/main.cpp:59-64), clamped to [icbrt(x), isqrt(x) - 1], the range the
    term identity needs."""
    cb = icbrt(x)
    y = cb * alpha_num // alpha_den
    lo, hi = cb, isqrt(x)
    return max(lo, min(y, hi - 1 if hi > lo else hi))


def leaf_counts(x, y, c=6):
    """Special-leaf counts by class (hard, easy_composite, easy_prime, trivial), brute force."""
    out = (ctypes.c_uint64 * 4)()
    lib().orc_leaf_counts(*_split(x), y, c, out)
    return dict(zip(("hard", "easy_composite", "easy_prime", "trivial"), (int(v) for v in out)))
