"""The C-ABI library: loads, exports every symbol declared in include/cpx.h,
and its host-side logic (exact roots, y rule, error paths) works without a
GPU.  CPU only."""
import ctypes

import numpy as np
import pytest


def test_exports_every_declared_symbol():
    from cudapix_b200 import _lib

    L = _lib.load()
    names = _lib.header_symbols()
    assert len(names) > 40
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    # and every declared symbol has a Python signature
    assert not [n for n in names if n not in _lib._SIGS], [n for n in names if n not in _lib._SIGS]


def test_version_string():
    from cudapix_b200 import _lib

    assert b"sm_100a" in _lib.load().cpx_version()


def test_roots_exact(orc):
    import cudapix_b200 as cpx

    rng = np.random.default_rng(11)
    vals = [0, 1, 2, 3, 7, 8, 15, 16, 17, 10**12, 10**20, 2**64 - 1, 2**64, 2**100 + 12345]
    vals += [int(rng.integers(1, 2**63)) * int(rng.integers(1, 2**62)) for _ in range(300)]
    for x in vals:
        s, c, q = cpx.iroots(x)
        assert s == orc.isqrt(x) and c == orc.icbrt(x) and q == orc.iroot4(x), x


def test_default_y_rule(orc):
    import cudapix_b200 as cpx

    for x, a in [(10**12, 10), (10**15, 8), (10**17, 32), (10**20, 16), (10**9, 1)]:
        assert cpx.default_y(x, a) == orc.default_y(x, a)
    # the documented configs
    assert cpx.default_y(10**12, 10) == 10**5
    assert cpx.default_y(10**20, 16) == 74265408


def test_reference_alpha_is_positive():
    from cudapix_b200 import _lib

    L = _lib.load()
    prev = 0
    for e in (6, 9, 12, 15, 18, 20):
        a = L.cpx_alpha_milli(_lib.U128.of(10**e))
        assert 1000 <= a < 100000 and a >= prev
        prev = a


def test_no_gpu_error_path():
    """Without a device, creating a context fails with a status, not a crash."""
    from cudapix_b200 import _lib

    L = _lib.load()
    if L.cpx_device_count() > 0:
        return
    h = ctypes.c_void_p()
    rc = L.cpx_create(0, ctypes.byref(h))
    assert rc != 0 and not h.value


def test_null_context_rejected():
    from cudapix_b200 import _lib

    L = _lib.load()
    out = ctypes.c_uint64()
    assert L.cpx_P2_u64(None, 10**12, 10**5, ctypes.byref(out)) == _lib.CPX_EINVAL
    assert L.cpx_destroy(None) == _lib.CPX_EINVAL


def test_s2hard_max_prime_below_quarter_root_refused():
    import cudapix_b200 as cpx

    with pytest.raises(ValueError):
        cpx.S2hard(10**12, 10**5, 6, maxPrime=999)
