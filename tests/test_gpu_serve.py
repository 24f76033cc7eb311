"""Serving (cpx_serve_*): continuous batching over resident tables.

Every answer of a served request must equal the same query answered alone
(an exact integer: tolerance zero) and, where the oracle's sieve reaches, the
oracle's count.  The servers here own private contexts so that the shared
test context stays usable."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _xs(seed, n, lo, hi):
    return [int(10.0**e) for e in np.random.default_rng(seed).uniform(lo, hi, n)]


def test_mix_equals_standalone(cpx, ctx, orc):
    xs = _xs(7, 240, 6, 13) + [10**14, 2**40 + 15, 999_983, 1, 2, 10**6]
    alone = [cpx.pi(x, ctx=ctx) for x in xs]
    own = cpx.Context(0)
    with cpx.Server(own, lanes=3, max_batch=64) as srv:
        tickets = [srv.submit(x) for x in xs]
        got = [srv.wait(t)[0] for t in tickets]
        st = srv.stats()
    assert got == alone
    for x, g in zip(xs, got):
        if x <= 10**8:
            assert g == orc.pi_sieve(x), x
    assert st["completed"] == len(xs) and st["failed"] == 0
    assert st["batches"] >= 2 and st["max_batch_seen"] <= 64


def test_replay_poisson_trace(cpx, ctx):
    rng = np.random.default_rng(1)
    n = 150
    gaps = rng.exponential(1.0 / 2000.0, n)
    xs = [int(10.0**e) for e in rng.uniform(10, 14, n)]
    arrivals = np.cumsum(gaps).tolist()
    alone = cpx.pi_batch(xs, ctx=ctx)
    own = cpx.Context(0)
    with cpx.Server(own, lanes=4, reserve_x=10**14, graph=True) as srv:
        got, lat = srv.replay(xs, arrivals)
        st = srv.stats()
    assert got == alone
    assert all(v > 0 for v in lat)
    assert st["completed"] == n and st["table_growths"] == 0


def test_tuned_lanes_cover_every_alpha(cpx, ctx, tmp_path):
    """Lanes of a tuned context run large batches with the batch alpha, the
    decade's own batch alpha (the committed table has them for 10^16 and
    10^17) or, without a batch alpha, the untuned one; the admission bounds
    cover each, so no request fails on table coverage."""
    import json
    import os

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    src = os.path.join(root, "cudapix_b200", "tuning", "b200.json")
    t = json.load(open(src))
    off = dict(t, entries=[dict(e, alpha_scale_milli=0) if e["decade"] == 99 else e for e in t["entries"]])
    path_off = tmp_path / "no_batch_alpha.json"
    path_off.write_text(json.dumps(off))  # one line: every entry is read all the same
    xs = _xs(11, 96, 10, 16.4) + [10**16 + 61, 2 * 10**16 + 3]
    alone = cpx.pi_batch(xs, ctx=ctx)
    for path in (src, str(path_off)):
        own = cpx.Context(0)
        own.tune_load(path)
        with cpx.Server(own, lanes=2, reserve_x=10**12) as srv:
            tickets = [srv.submit(x) for x in xs]
            got = [srv.wait(t)[0] for t in tickets]
            st = srv.stats()
        own.close()
        assert got == alone, path
        assert st["failed"] == 0 and st["completed"] == len(xs)


def test_tables_grow_on_demand(cpx, ctx):
    own = cpx.Context(0)
    with cpx.Server(own, lanes=2) as srv:
        small = [10**9 + 7, 123456789012]
        r1 = [srv.wait(srv.submit(x))[0] for x in small]
        big = [10**15, 3 * 10**14 + 11]
        r2 = [srv.wait(srv.submit(x))[0] for x in big]
        st = srv.stats()
    assert r1 == [cpx.pi(x, ctx=ctx) for x in small]
    assert r2 == [cpx.pi(x, ctx=ctx) for x in big]
    assert st["table_growths"] >= 1


def test_context_is_locked_while_serving(cpx):
    own = cpx.Context(0)
    srv = cpx.Server(own, lanes=1)
    with pytest.raises(cpx.CpxError):
        cpx.pi(10**12, ctx=own)
    assert srv.wait(srv.submit(10**12))[0] == 37607912018
    srv.close()
    assert cpx.pi(10**12, ctx=own) == 37607912018


def test_invalid_server_config(cpx):
    own = cpx.Context(0)
    with pytest.raises(cpx.CpxError):
        cpx.Server(own, lanes=17)
    with pytest.raises(cpx.CpxError):
        cpx.Server(own, admit_fraction=0.99)
    with cpx.Server(own, lanes=1) as srv:
        with pytest.raises(cpx.CpxError):
            cpx.Server(own, lanes=1)  # one server per context
        with pytest.raises(cpx.CpxError):
            srv.wait(12345)  # never issued
