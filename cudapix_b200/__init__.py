"""cudapix_b200 -- exact pi(x) by Deleglise-Rivat on B200 (sm_100a).

Python mirror of the reference's term entry points (curtisseizert/CUDApix),
over the C ABI in include/cpx.h.  Names and argument meanings follow the
reference:

    P2(x, y)                      include/P2.cuh:16-17
    S2_trivial(x, y)              include/trivial.cuh:8,12
    Ordinary(x, y, c)             include/ordinary.cuh:6-7
    S2hard(x, y, c)               include/sieve/S2_hard_host.cuh:35-36
    pi_deleglise_rivat(x, y, c)   include/Deleglise-Rivat/deleglise-rivat.hpp:28,64
    mutest(top)                   include/mutest.cuh:3
    gen_d_mu / gen_d_lpf / gen_h_mu / gen_h_lpf / gen_d_mu_lpf
                                  include/sieve/lpf_mu.cuh:12-24
    get_d_piTable(hi), PiTable    include/pitable.cuh:7,12-51
    Phi                           include/phi.cuh:17-36
    Phisieve                      include/sieve/phisieve_host.cuh:6-40
    get_device_primes / count_primes   CUDASieve (external dependency)

Errors raise CpxError (the reference checked none).  Every value is an exact
Python int; 64- and 128-bit overloads are chosen by the size of x.
"""
import ctypes
import math
import os

import numpy as np

from ._lib import (BatchStats, CpxError, ExtensionMissing, GourdonTerms, LeafCounts, Params, ServeConfig, ServeCounters,  # noqa: F401
                   Terms, TuneEntry,
                   U128,
                   header_symbols, load)

__all__ = [
    "Context", "context", "P2", "S2_trivial", "Ordinary", "S2_easy", "S2hard", "pi_deleglise_rivat",
    "pi_terms", "pi", "pi_batch", "mutest", "gen_d_mu", "gen_d_lpf", "gen_h_mu", "gen_h_lpf", "gen_d_mu_lpf",
    "get_d_piTable", "PiTable", "Phi", "Phisieve", "get_device_primes", "count_primes", "DeviceArray",
    "default_y", "iroots", "CpxError", "ExtensionMissing",
]

_U64 = (1 << 64) - 1


class DeviceArray:
    """A cudaMalloc'd buffer returned by the library (caller-owned, like the
    reference's gen_d_* / get_d_piTable pointers)."""

    def __init__(self, ptr, n, ctype, owned=True):
        self.ptr, self.n, self.ctype, self.owned = ptr, n, ctype, owned

    def to_host(self):
        import numpy as np

        dt = np.dtype(self.ctype)
        out = np.empty(self.n, dtype=dt)
        if self.n:
            _check(None, load().cpx_copy_to_host(out.ctypes.data, self.ptr, self.n * dt.itemsize))
        return out

    def free(self):
        if self.owned and self.ptr:
            load().cpx_free(self.ptr)
        self.ptr = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def _check(ctx, rc):
    if rc != 0:
        msg = load().cpx_last_error(ctx.h).decode() if ctx is not None else "device copy failed"
        raise CpxError(rc, msg)


class Context:
    """Owns a CUDA stream and the resident tables on one device."""

    def __init__(self, device=0):
        L = load()
        h = ctypes.c_void_p()
        rc = L.cpx_create(device, ctypes.byref(h))
        if rc != 0:
            raise CpxError(rc, f"cannot create a context on device {device}")
        self.h = h
        self.L = L
        self.device = device

    def close(self):
        if getattr(self, "h", None):
            self.L.cpx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def call(self, name, *args):
        _check(self, getattr(self.L, name)(self.h, *args))

    @property
    def stream(self):
        return self.L.cpx_stream(self.h)

    @property
    def launches(self):
        return self.L.cpx_launch_count(self.h)

    def set_hard_params(self, log2_bits, threads):
        self.call("cpx_set_hard_params", log2_bits, threads)

    def set_hard_offload(self, min_candidates):
        self.call("cpx_set_hard_offload", min_candidates)

    def set_hard_shared(self, mode):
        """0: one hard-leaf sieve per query; 1: batches share a sieve
        (default); 2: always share (single queries too)."""
        self.call("cpx_set_hard_shared", mode)

    def autotune(self, decade_lo=9, decade_hi=17, seconds=0.0):
        """Tunes the plain path per decade of x (lone queries at 10^e and 10^(e+1/2))."""
        self.call("cpx_autotune", decade_lo, decade_hi, float(seconds))

    def autotune_batch(self, xs):
        """Tunes the entry used by batches of more than four queries on this sample batch."""
        self.call("cpx_autotune_batch", _u128_array(xs), len(xs))

    def tune_save(self, path):
        self.call("cpx_tune_save", os.fsencode(path))

    def tune_load(self, path):
        self.call("cpx_tune_load", os.fsencode(path))

    def tune_get(self, decade):
        """Entry of a decade of x (99: the batch entry); threads = 0 means untuned."""
        t = TuneEntry()
        self.call("cpx_tune_get", decade, ctypes.byref(t))
        return {k: getattr(t, k) for k, _ in t._fields_}

    def tune_clear(self):
        self.call("cpx_tune_clear")

    def set_p2_window(self, limit):
        """z above `limit`: P2 over pi-table windows (resident table to sqrt x)."""
        self.call("cpx_set_p2_window", limit)

    def set_timing(self, on=True):
        self.call("cpx_set_timing", 1 if on else 0)

    def last_hard_stats(self):
        ms, by = ctypes.c_float(), ctypes.c_double()
        self.call("cpx_last_hard_stats", ctypes.byref(ms), ctypes.byref(by))
        return ms.value, by.value

    def sm_count(self):
        return self.L.cpx_sm_count(self.h)

    def last_kernel_ms(self):
        """{kernel: device ms} of the timed kernel launches of the last batch
        (timing on, not a graph); launches of the same kernel are summed."""
        out = {}
        i = 0
        while True:
            name, ms = ctypes.c_char_p(), ctypes.c_float()
            if self.L.cpx_last_kernel_span(self.h, i, ctypes.byref(name), ctypes.byref(ms)) != 0:
                break
            k = name.value.decode()
            out[k] = out.get(k, 0.0) + ms.value
            i += 1
        return out

    def last_batch_ms(self):
        ms = ctypes.c_float()
        self.call("cpx_last_batch_ms", ctypes.byref(ms))
        return ms.value

    def last_batch_stats(self):
        """Host phases (ms) and hard-leaf work shape of the last batch."""
        st = BatchStats()
        self.call("cpx_last_batch_stats", ctypes.byref(st))
        return st.as_dict()

    def timer_start(self):
        self.call("cpx_timer_start")

    def timer_stop(self):
        ms = ctypes.c_float()
        self.call("cpx_timer_stop", ctypes.byref(ms))
        return ms.value

    def flush_l2(self):
        self.call("cpx_flush_l2")

    def mem_info(self):
        f, t = ctypes.c_uint64(), ctypes.c_uint64()
        self.call("cpx_mem_info", ctypes.byref(f), ctypes.byref(t))
        return f.value, t.value


_default = {}


def context(device=0):
    if device not in _default:
        _default[device] = Context(device)
    return _default[device]


def _wide(x):
    return x > _U64


def iroots(x):
    s, c, q = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
    load().cpx_iroots(U128.of(x), ctypes.byref(s), ctypes.byref(c), ctypes.byref(q))
    return s.value, c.value, q.value


def default_y(x, alpha=None):
    """y = floor(alpha * icbrt(x)) (src/main.cpp:59-64), alpha an int or
    Fraction; None = the reference's alpha(x) (src/main.cpp:128-194)."""
    from fractions import Fraction

    if alpha is None:
        num, den = 0, 0
    else:
        f = Fraction(alpha).limit_denominator(1000)
        num, den = f.numerator, f.denominator
    y = ctypes.c_uint64()
    load().cpx_default_y(U128.of(x), num, den, ctypes.byref(y))
    return y.value


# ---------------------------------------------------------------- terms

def P2(x, y, ctx=None):
    ctx = ctx or context()
    if _wide(x):
        o = U128()
        ctx.call("cpx_P2_u128", U128.of(x), y, ctypes.byref(o))
        return o.value(signed=True)
    o = ctypes.c_uint64()
    ctx.call("cpx_P2_u64", x, y, ctypes.byref(o))
    return o.value


def S2_trivial(x, y, ctx=None):
    ctx = ctx or context()
    if _wide(x):
        o = U128()
        ctx.call("cpx_trivial_u128", U128.of(x), y, ctypes.byref(o))
        return o.value(signed=True)
    o = ctypes.c_uint64()
    ctx.call("cpx_trivial_u64", x, y, ctypes.byref(o))
    return o.value


def Ordinary(x, y, c=6, ctx=None):
    ctx = ctx or context()
    if _wide(x):
        o = U128()
        ctx.call("cpx_ordinary_u128", U128.of(x), y, c, ctypes.byref(o))
        return o.value(signed=True)
    o = ctypes.c_int64()
    ctx.call("cpx_ordinary_u64", x, y, c, ctypes.byref(o))
    return o.value


def S2_easy(x, y, c=6, ctx=None):
    ctx = ctx or context()
    if _wide(x):
        o = U128()
        ctx.call("cpx_S2_easy_u128", U128.of(x), y, c, ctypes.byref(o))
        return o.value(signed=True)
    o = ctypes.c_int64()
    ctx.call("cpx_S2_easy_u64", x, y, c, ctypes.byref(o))
    return o.value


def S2hard(x, y, c=6, ctx=None, maxPrime=None):
    """Hard leaves of the exact split (x/(p_b m) >= p_b^2, so p_b <= x^(1/4)).
    maxPrime caps the sieving primes (include/sieve/S2_hard_host.cuh:36); as
    hard leaves stop at x^(1/4), any cap >= x^(1/4) gives all of them and a
    smaller one raises ValueError."""
    if maxPrime is not None and maxPrime < math.isqrt(math.isqrt(x)):
        raise ValueError("S2hard with maxPrime below x^(1/4) is not supported")
    ctx = ctx or context()
    if _wide(x):
        o = U128()
        ctx.call("cpx_S2_hard_u128", U128.of(x), y, c, ctypes.byref(o))
        return o.value(signed=True)
    o = ctypes.c_int64()
    ctx.call("cpx_S2_hard_u64", x, y, c, ctypes.byref(o))
    return o.value


def pi_terms(x, y=0, c=6, ctx=None):
    """Every term of pi(x) as a dict (P2, ordinary, trivial, easy, hard, pi_y, pi, x, y, z, c)."""
    ctx = ctx or context()
    t = Terms()
    if _wide(x):
        o = U128()
        ctx.call("cpx_pi_u128", U128.of(x), y, c, ctypes.byref(o), ctypes.byref(t))
    else:
        o = ctypes.c_uint64()
        ctx.call("cpx_pi_u64", x, y, c, ctypes.byref(o), ctypes.byref(t))
    return t.as_dict()


def pi_gourdon(x, y=0, c=6, ctx=None):
    """pi(x) through Gourdon's decomposition, every term as a dict (A, B, C,
    D, phi0, sigma, pi, x, y): the terms of the reference's GourdonVariant64
    (include/Gourdon/gourdonvariant.hpp:7-56).  x < 2^64."""
    ctx = ctx or context()
    if _wide(x):
        raise ValueError("Gourdon's decomposition here takes x < 2^64 (as GourdonVariant64)")
    t = GourdonTerms()
    ctx.call("cpx_gourdon_u64", x, y, c, ctypes.byref(t))
    return t.as_dict()


def leaf_counts(x, y=0, c=6, ctx=None):
    """Exact special-leaf counts of pi(x) by class: hard, easy_composite,
    easy_prime, trivial (src/leafcount.cpp:12-202 estimates them)."""
    ctx = ctx or context()
    o = LeafCounts()
    ctx.call("cpx_leaf_count", U128.of(x), y, c, ctypes.byref(o))
    return {k: getattr(o, k) for k, _ in o._fields_}


def pi_deleglise_rivat(x, y=0, c=6, ctx=None):
    return pi_terms(x, y, c, ctx)["pi"]


def pi(x, ctx=None):
    return pi_deleglise_rivat(x, 0, 6, ctx)


BATCH_WIDE = 1   # 128-bit kernels for every query (CPX_BATCH_WIDE)
BATCH_GRAPH = 2  # the batch's kernels as one CUDA graph launch (CPX_BATCH_GRAPH)


def _params(alpha, c, hard_log2_bits, hard_threads, wide, graph):
    from fractions import Fraction

    p = Params()
    if alpha is not None:
        f = Fraction(alpha).limit_denominator(1000)
        p.alpha_num, p.alpha_den = f.numerator, f.denominator
    p.c = c
    p.flags = (BATCH_WIDE if wide else 0) | (BATCH_GRAPH if graph else 0)
    p.hard_log2_bits = hard_log2_bits
    p.hard_threads = hard_threads
    return p


_M64 = (1 << 64) - 1


def _u128_array(xs):
    """A ctypes array of 128-bit values (low word first), filled through a
    numpy view (a per-element struct loop costs milliseconds per batch)."""
    n = len(xs)
    arr = (U128 * max(n, 1))()
    if n:
        w = np.frombuffer(arr, dtype=np.uint64).reshape(-1, 2)
        a = np.asarray(xs) if isinstance(xs, (list, tuple, np.ndarray)) else None
        if a is not None and a.ndim == 1 and a.dtype.kind in "iu" and (a.dtype.kind == "u" or a.min() >= 0):
            w[:n, 0] = a.astype(np.uint64)  # integers below 2^64: one conversion, high words stay 0
        else:
            ints = [int(x) for x in xs]
            w[:n, 0] = [x & _M64 for x in ints]
            w[:n, 1] = [(x >> 64) & _M64 for x in ints]
    return arr


def _u128_values(arr, n):
    w = np.frombuffer(arr, dtype=np.uint64).reshape(-1, 2)[:n]
    return [lo | (hi << 64) if hi else lo for lo, hi in zip(w[:, 0].tolist(), w[:, 1].tolist())]


def pi_batch(xs, alpha=None, c=6, hard_log2_bits=0, hard_threads=0, wide=False, graph=False, ctx=None):
    """pi(x) for every x in xs in one batched device pass."""
    ctx = ctx or context()
    n = len(xs)
    arr = _u128_array(xs)
    out = (U128 * max(n, 1))()
    p = _params(alpha, c, hard_log2_bits, hard_threads, wide, graph)
    ctx.call("cpx_pi_batch", arr, n, ctypes.byref(p), out)
    return _u128_values(out, n)


class Server:
    """Continuous batching of pi(x) requests (cpx_serve_*): `lanes` worker
    streams share the context's resident tables; while the server exists the
    context answers no other call."""

    def __init__(self, ctx, lanes=4, max_batch=4096, admit_fraction=0.5, reserve_x=0, alpha=None, c=6,
                 hard_log2_bits=0, hard_threads=0, graph=False, fill_target=0, window_us=0):
        self.ctx = ctx
        self.L = ctx.L
        cfg = ServeConfig()
        cfg.lanes = lanes
        cfg.max_batch = max_batch
        cfg.admit_fraction = admit_fraction
        cfg.reserve_x = U128.of(reserve_x)
        cfg.params = _params(alpha, c, hard_log2_bits, hard_threads, False, graph)
        cfg.fill_target = fill_target
        cfg.window_us = window_us
        h = ctypes.c_void_p()
        rc = self.L.cpx_serve_create(ctx.h, ctypes.byref(cfg), ctypes.byref(h))
        if rc != 0:
            raise CpxError(rc, self.L.cpx_last_error(ctx.h).decode())
        self.h = h

    def _check(self, rc):
        if rc != 0:
            raise CpxError(rc, self.L.cpx_serve_last_error(self.h).decode())

    def submit(self, x):
        t = ctypes.c_uint64()
        self._check(self.L.cpx_serve_submit(self.h, U128.of(x), ctypes.byref(t)))
        return t.value

    def wait(self, ticket):
        """(pi, latency_ms) of a submitted request."""
        o, ms = U128(), ctypes.c_double()
        self._check(self.L.cpx_serve_wait(self.h, ticket, ctypes.byref(o), ctypes.byref(ms)))
        return o.value(), ms.value

    def replay(self, xs, arrival_s):
        """Submits xs[i] at arrival_s[i] seconds from now; returns (pis, latencies_ms)."""
        n = len(xs)
        arr = _u128_array(xs)
        ts = (ctypes.c_double * max(n, 1))(*arrival_s)
        out = (U128 * max(n, 1))()
        lat = (ctypes.c_double * max(n, 1))()
        self._check(self.L.cpx_serve_replay(self.h, arr, ts, n, out, lat))
        return [out[i].value() for i in range(n)], [lat[i] for i in range(n)]

    def stats(self):
        st = ServeCounters()
        self._check(self.L.cpx_serve_stats(self.h, ctypes.byref(st)))
        return st.as_dict()

    def close(self):
        if getattr(self, "h", None):
            self.L.cpx_serve_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def terms_batch(xs, ys=None, alpha=None, c=6, hard_log2_bits=0, hard_threads=0, wide=False, graph=False,
                ctx=None):
    """Every term (as pi_terms) for each x in xs, in one batched pass; ys[i] = 0
    or ys = None selects the y rule (alpha)."""
    ctx = ctx or context()
    n = len(xs)
    arr = _u128_array(xs)
    yarr = (ctypes.c_uint64 * max(n, 1))(*(ys or [0] * n))
    out = (Terms * max(n, 1))()
    p = _params(alpha, c, hard_log2_bits, hard_threads, wide, graph)
    ctx.call("cpx_terms_batch", arr, yarr, n, ctypes.byref(p), out)
    return [out[i].as_dict() for i in range(n)]


# ---------------------------------------------------------- sieves / tables

def mutest(top, ctx=None):
    ctx = ctx or context()
    o = ctypes.c_int64()
    ctx.call("cpx_mutest", top, ctypes.byref(o))
    return o.value


def gen_d_mu(bottom, top, ctx=None):
    ctx = ctx or context()
    p = ctypes.c_void_p()
    ctx.call("cpx_gen_d_mu", bottom, top, ctypes.byref(p))
    return DeviceArray(p.value, (top - bottom) // 2, "int8")


def gen_d_lpf(bottom, top, wide=False, ctx=None):
    ctx = ctx or context()
    p = ctypes.c_void_p()
    if wide or top > (1 << 32):
        ctx.call("cpx_gen_d_lpf64", bottom, top, ctypes.byref(p))
        return DeviceArray(p.value, (top - bottom) // 2, "uint64")
    ctx.call("cpx_gen_d_lpf32", bottom, top, ctypes.byref(p))
    return DeviceArray(p.value, (top - bottom) // 2, "uint32")


def gen_d_mu_lpf(bottom, top, ctx=None):
    """Returns (mu int8, lpf uint64) device arrays (src/sieve/lpf_mu.cu:282-302)."""
    ctx = ctx or context()
    n = (top - bottom) // 2
    L = load()
    pm, pl = ctypes.c_void_p(), ctypes.c_void_p()
    _check(None, L.cpx_device_alloc(max(n, 1), ctypes.byref(pm)))
    _check(None, L.cpx_device_alloc(max(n, 1) * 8, ctypes.byref(pl)))
    ctx.call("cpx_gen_d_mu_lpf", bottom, top, pm, pl)
    return DeviceArray(pm.value, n, "int8"), DeviceArray(pl.value, n, "uint64")


def gen_h_mu(bottom, top, ctx=None):
    import numpy as np

    ctx = ctx or context()
    out = np.zeros((top - bottom) // 2, dtype=np.int8)
    ctx.call("cpx_gen_h_mu", bottom, top, out.ctypes.data)
    return out


def gen_h_lpf(bottom, top, ctx=None):
    import numpy as np

    ctx = ctx or context()
    out = np.zeros((top - bottom) // 2, dtype=np.uint32)
    ctx.call("cpx_gen_h_lpf32", bottom, top, out.ctypes.data)
    return out


def get_d_piTable(hi, ctx=None):
    """Dense table t[k] = pi(2k - 1), k < hi/2 (src/pitable.cu:10-25)."""
    ctx = ctx or context()
    p = ctypes.c_void_p()
    ctx.call("cpx_pitable", hi, ctypes.byref(p))
    return DeviceArray(p.value, hi // 2, "uint32")


def get_device_primes(bottom, top, ctx=None):
    """Primes in [bottom, top) (CudaSieve::getDevicePrimes)."""
    ctx = ctx or context()
    p, n = ctypes.c_void_p(), ctypes.c_uint64()
    ctx.call("cpx_primes", bottom, top, ctypes.byref(p), ctypes.byref(n))
    return DeviceArray(p.value, n.value, "uint64")


def count_primes(bottom, top, ctx=None):
    """Number of primes in [bottom, top) (CudaSieve::countPrimes)."""
    ctx = ctx or context()
    n = ctypes.c_uint64()
    ctx.call("cpx_count_primes", bottom, top, ctypes.byref(n))
    return n.value


class PiTable:
    """Windowed pi table (src/pitable.cu:27-218): table[k] = pi(base + 2k - 1) - pi_base
    for k < range/2 + 2, walked up or down in windows of `range`."""

    def __init__(self, *args, ctx=None):
        self.ctx = ctx or context()
        if len(args) == 1:
            self.base, self.bottom, self.range = 0, 0, int(args[0])
        elif len(args) in (2, 3):
            self.base, self.bottom = int(args[0]), int(args[1])
            rng = int(args[2]) if len(args) == 3 else 0
            self.range = rng if rng else min(self.getMaxRange(), self.base - self.bottom)
        else:
            raise TypeError("PiTable(range) or PiTable(base, bottom, range=0)")
        self._buf = None
        self._alloc()
        self.pi_base = None
        self._pi_base_at = None  # the base that pi_base belongs to

    def _alloc(self):
        L = load()
        p = ctypes.c_void_p()
        _check(None, L.cpx_device_alloc((self.range // 2 + 2) * 4, ctypes.byref(p)))
        if self._buf is not None:
            self._buf.free()
        self._buf = DeviceArray(p.value, self.range // 2 + 2, "uint32")

    def getMaxRange(self):
        free, _ = self.ctx.mem_info()
        return int(free / 2.5)

    def get_base(self):
        return self.base

    def get_range(self):
        return self.range

    def get_bottom(self):
        return self.bottom

    def get_pi_base(self):
        """pi(base - 1), counted on first use after the base changes
        (src/pitable.cu:154-166)."""
        if self.base == 0:
            return 0
        if self._pi_base_at != self.base:
            self.pi_base = count_primes(0, self.base, ctx=self.ctx)
            self._pi_base_at = self.base
        return self.pi_base

    def set_pi_base(self, pi_base):
        """A caller's pi(base - 1) (src/pitable.cu:175-179), kept until the base
        changes; the next window fill replaces it by the exact count."""
        self.pi_base = int(pi_base)
        self._pi_base_at = self.base

    def set_base(self, base):
        self.base = int(base)

    def set_range(self, rng):
        """Unlike the reference (src/pitable.cu:181-186), the buffer follows
        the new range."""
        self.range = int(rng)
        self._alloc()

    def allocate(self):
        """Keeps an existing buffer (src/pitable.cu:63-68); contents are
        written by the next getCurrent / getNextUp / getNextDown."""
        if self._buf is None or not self._buf.ptr:
            self._alloc()

    def reallocate(self):
        """A new buffer for the current range (src/pitable.cu:70-75)."""
        self._alloc()

    def setMaxRange(self):
        """range = getMaxRange(), then reallocate (src/pitable.cu:56-61)."""
        self.range = self.getMaxRange()
        self._alloc()
        return self.range

    def set_bottom(self, bottom):
        self.bottom = int(bottom)

    def _fill(self):
        pb = ctypes.c_uint64()
        self.ctx.call("cpx_pitable_window", self.base, self.range, self._buf.ptr, ctypes.byref(pb))
        self.pi_base = pb.value
        self._pi_base_at = self.base
        return self._buf

    def getCurrent(self):
        return self._fill()

    def getNextUp(self):
        self.base += self.range
        return self._fill()

    def getNextDown(self):
        if self.bottom < self.base - self.range:
            self.base -= self.range
        else:
            self.range = self.base - self.bottom
            self.base = self.bottom
        return self._fill()

    def getNextBaseUp(self):
        return self.base + self.range

    def getNextBaseDown(self):
        return max(self.bottom, self.base - self.range)


class Phi:
    """phi(x, a) and phi prefix ranges (src/phi.cu:14-109).

    Index convention of the reference: phi(x, a) excludes the primes up to
    smallPrimes[a] / h_primeList[a - 12] (0-based), i.e. the first a + 1
    primes; phi_std(x, a) is the textbook phi with the first a primes."""

    def __init__(self, max_, p_max=None, ctx=None):
        self.ctx = ctx or context()
        self.max = int(max_)
        self.p_max = p_max
        self._lpf = None
        self._primes = None

    def get_d_lpf(self):
        """lpf of the odd n in [0, max) (src/phi.cu:16), built on first use."""
        if self._lpf is None:
            self._lpf = gen_d_lpf(0, self.max, ctx=self.ctx)
        return self._lpf

    def get_h_primeList(self):
        """The sieving primes after the 12 small primes 2 .. 37, up to p_max
        (default isqrt(max)), as PrimeList::getSievingPrimes gives them
        (src/phi.cu:20,30)."""
        if self._primes is None:
            top = self.p_max if self.p_max is not None else math.isqrt(self.max)
            self._primes = get_device_primes(41, top + 1, ctx=self.ctx).to_host().astype(np.uint32)
        return self._primes

    def get_d_primeList(self):
        h = self.get_h_primeList()
        p = ctypes.c_void_p()
        _check(None, load().cpx_device_alloc(max(1, h.size) * 4, ctypes.byref(p)))
        arr = DeviceArray(p.value, h.size, "uint32")
        if h.size:
            _check(None, load().cpx_copy_to_device(p.value, h.ctypes.data, h.size * 4))
        return arr

    def get_primeListLength(self):
        return int(self.get_h_primeList().size)

    def makeModCache(self, pi_max):
        """The reference fills a private cache that phi() never reads
        (src/phi.cu:58-73); phi() here is exact without it."""

    def phi(self, x, a):
        return self.phi_std(x, a + 1)

    def phi_std(self, x, a):
        o = ctypes.c_uint64()
        self.ctx.call("cpx_phi", x, a, ctypes.byref(o))
        return o.value

    def generateRange(self, num, a):
        """t[i] = phi(2i + 1, a + 1) (inclusive count), i < num/2."""
        p = ctypes.c_void_p()
        self.ctx.call("cpx_phi_range", num, a + 1, ctypes.byref(p))
        return DeviceArray(p.value, num // 2, "uint32")


class Phisieve:
    """Odd-only bit sieve with a count table counts[i] = phi(2i - 1, a)
    (src/sieve/phisieve_host.cu:12-89)."""

    def __init__(self, maxPrime, blockSize=1 << 28, ctx=None):
        self.ctx = ctx or context()
        self.blockSize = int(blockSize)
        h = ctypes.c_void_p()
        self.ctx.call("cpx_phisieve_create", maxPrime, self.blockSize, ctypes.byref(h))
        self.h = h

    def _c(self, name, *args):
        rc = getattr(load(), name)(self.h, *args)
        if rc != 0:
            raise CpxError(rc, load().cpx_last_error(self.ctx.h).decode())

    def firstSieve(self, c):
        self._c("cpx_phisieve_first", c)

    def markNext(self):
        self._c("cpx_phisieve_mark_next")

    def updateCount(self):
        self._c("cpx_phisieve_update")

    def get_a_current(self):
        a = ctypes.c_uint32()
        self._c("cpx_phisieve_counts", None, ctypes.byref(a))
        return a.value

    def set_a_current(self, a):
        """The next markNext crosses off p_(a+1); the bitmap is left as it is
        (include/sieve/phisieve_host.cuh:37)."""
        self._c("cpx_phisieve_set_a", a)

    def getCountDevice(self):
        p, a = ctypes.c_void_p(), ctypes.c_uint32()
        self._c("cpx_phisieve_counts", ctypes.byref(p), ctypes.byref(a))
        return DeviceArray(p.value, self.blockSize, "uint32", owned=False)

    def getCountHost(self):
        return self.getCountDevice().to_host()

    def close(self):
        if getattr(self, "h", None):
            load().cpx_phisieve_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
