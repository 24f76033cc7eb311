"""pi(10^20) in the 128-bit path: x above 2^64, y = 16 icbrt(x), u128
quotients x/(p m), 128-bit partial sums, P2 over pi-table windows.  P2,
ordinary, trivial and pi(y) against the CPU oracle's values
(golden/terms_1e20.json, made by golden/make_terms_1e20.py); the total
against OEIS A006880.  About ten seconds on one B200."""
import json
import os

import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


def test_pi_1e20_terms(cpx, golden):
    with open(os.path.join(HERE, "golden", "terms_1e20.json")) as f:
        ref = json.load(f)
    x = 10**20
    y = ref["y"]
    assert y == cpx.default_y(x, 16) == 74265408
    own = cpx.Context(0)
    t = cpx.pi_terms(x, y, 6, ctx=own)
    free, total = own.mem_info()
    own.close()
    for k in ("P2", "ordinary", "trivial", "pi_y"):
        assert t[k] == int(ref[k]), (k, t[k], ref[k])
    assert t["pi"] == golden["pi_pow10"]["20"] == 2220819602560918840
    assert total - free < 160 * 10**9
