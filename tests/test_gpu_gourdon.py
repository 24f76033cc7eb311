"""pi(x) through Gourdon's decomposition on the GPU (cpx_gourdon_u64, the
terms of the reference's GourdonVariant64, include/Gourdon/gourdonvariant.hpp:7-56):
A, B, C, D, Phi0 and Sigma each equal to the CPU oracle's (orc_pi_gourdon,
which is checked against the Deleglise-Rivat identity on the CPU), and the
total equal to the published pi(10^k) and to the Deleglise-Rivat path.
Exact integers: tolerance zero."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TERMS = ("A", "B", "C", "D", "phi0", "sigma", "pi")


def _cases():
    out = [(10**12, 10**5), (10**9, 1000), (10**10, 2154), (10**11, 4641 * 3), (10**13, 23208 * 2),
           (10**14, 46415 * 8), (2**40 + 15, 10**5 + 3)]
    rng = np.random.default_rng(7)
    for e in rng.uniform(8, 14, 6):
        x = int(10.0**e)
        cb = round(x ** (1 / 3))
        sq = int(x**0.5)
        out.append((x, cb + 1))            # y at the bottom of the domain
        out.append((x, min(sq - 2, cb * 20)))
    return out


@pytest.mark.parametrize("x,y", _cases())
def test_gourdon_terms_equal_oracle(ctx, cpx, orc, x, y):
    y = max(y, orc.icbrt(x))
    g = cpx.pi_gourdon(x, y, 6, ctx=ctx)
    o = orc.pi_gourdon(x, y, 6)
    for k in TERMS:
        assert g[k] == o[k], (k, x, y, g[k], o[k])
    assert g["pi"] == cpx.pi_deleglise_rivat(x, y, 6, ctx=ctx)


@pytest.mark.parametrize("k", range(7, 19))
def test_gourdon_pi_pow10(ctx, cpx, golden, k):
    assert cpx.pi_gourdon(10**k, 0, 6, ctx=ctx)["pi"] == golden["pi_pow10"][str(k)]


def test_gourdon_rejects_wide_x(ctx, cpx):
    with pytest.raises(ValueError):
        cpx.pi_gourdon(2**64 + 1, 0, 6, ctx=ctx)
