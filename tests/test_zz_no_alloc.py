"""cpx_mutest_noalloc, the Mertens self-test for callers that cannot call
cudaMalloc (their device memory belongs to another allocator, or an
allocation would synchronise a latency-critical path).  It keeps its scratch
in a static device array instead of allocating.

Checked through the C ABI on two calls in a row against the CPU oracle's
Mertens sum (orc_mertens), the sympy Mertens vectors of golden.json and the
allocating entry point cpx_mutest.  All are integer counts, so the tolerance
is zero.  This file is collected last so that a run stopping at the first
failure has already run every other test; it also passes alone in a fresh
process."""
import ctypes

import pytest

pytestmark = pytest.mark.gpu

MAX_TOP = 1 << 25


def _mutest(L, h, name, top):
    out = ctypes.c_int64()
    rc = getattr(L, name)(h, top, ctypes.byref(out))
    assert rc == 0, (name, rc, L.cpx_last_error(h))
    return out.value


@pytest.fixture(scope="module")
def lib_ctx():
    from cudapix_b200 import _lib

    L = _lib.load()
    h = ctypes.c_void_p()
    assert L.cpx_create(0, ctypes.byref(h)) == 0
    yield L, h
    L.cpx_destroy(h)


@pytest.mark.parametrize("top", [1, 2, 100, 10**6 + 7, 12_345_679, MAX_TOP])
def test_noalloc_matches_oracle_and_allocating_entry_point_twice(lib_ctx, orc, top):
    L, h = lib_ctx
    want = orc.mertens(top)
    first = _mutest(L, h, "cpx_mutest_noalloc", top)
    second = _mutest(L, h, "cpx_mutest_noalloc", top)
    assert first == want
    assert second == want
    assert _mutest(L, h, "cpx_mutest", top) == want


def test_noalloc_matches_sympy_mertens(lib_ctx, golden):
    # golden["mertens"]: [top, sum of mu(n) over 1 <= n < top] from sympy
    L, h = lib_ctx
    for top, m in golden["mertens"]:
        assert _mutest(L, h, "cpx_mutest_noalloc", top) == m, top


def test_noalloc_after_a_larger_call(lib_ctx, orc):
    # the static array keeps the previous call's contents; a smaller call must not read them
    L, h = lib_ctx
    _mutest(L, h, "cpx_mutest_noalloc", MAX_TOP)
    assert _mutest(L, h, "cpx_mutest_noalloc", 1000) == orc.mertens(1000) == _mutest(L, h, "cpx_mutest", 1000)


def test_noalloc_rejects_sizes_beyond_its_scratch(lib_ctx):
    L, h = lib_ctx
    out = ctypes.c_int64()
    from cudapix_b200 import _lib

    assert L.cpx_mutest_noalloc(h, MAX_TOP + 1, ctypes.byref(out)) == _lib.CPX_ERANGE
    assert b"33554432" in L.cpx_last_error(h)
