"""pi(10^21) in the 128-bit path, y = 16 icbrt(x): the per-(segment, level)
hard-leaf records of one sieve would take about 160 GB, so the hard leaves
run in windows of segments merged in order and device memory stays near
20 GB.  The total against OEIS A006880.  About a minute on one B200."""
import pytest

pytestmark = [pytest.mark.gpu, pytest.mark.slow]

PI_1E21 = 21127269486018731928


def test_pi_1e21(cpx):
    own = cpx.Context(0)
    try:
        t = cpx.pi_terms(10**21, cpx.default_y(10**21, 16), 6, ctx=own)
        free, total = own.mem_info()
    finally:
        own.close()
    assert t["pi"] == PI_1E21
    assert total - free < 160 * 10**9
