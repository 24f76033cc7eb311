"""Autotuner (cpx_autotune, cpx_autotune_batch, cpx_tune_*): settings
measured on the device, per decade for the plain path and one entry for
larger batches.  Every answer is identical with and without tuning, and the
table round trips through its JSON file."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_autotune_keeps_results_and_round_trips(cpx, ctx, tmp_path):
    own = cpx.Context(0)
    xs = [int(10.0**e) for e in np.random.default_rng(2).uniform(9, 11, 300)]
    singles = [10**9 + 7, 3 * 10**10 + 1]
    want = cpx.pi_batch(xs, ctx=ctx)
    want1 = [cpx.pi(x, ctx=ctx) for x in singles]
    own.autotune(9, 10)
    own.autotune_batch(xs[:64])
    e9, e10, eb = own.tune_get(9), own.tune_get(10), own.tune_get(99)
    for e in (e9, e10, eb):
        assert e["threads"] in (128, 256, 512, 1024) and e["ms"] > 0
        assert e["log2_bits"] == 0 or 15 <= e["log2_bits"] <= 20
    assert own.tune_get(11)["threads"] == 0  # not tuned
    assert cpx.pi_batch(xs, ctx=own) == want
    assert [cpx.pi(x, ctx=own) for x in singles] == want1
    path = tmp_path / "tune.json"
    own.tune_save(str(path))
    own.tune_clear()
    assert own.tune_get(9)["threads"] == 0 and own.tune_get(99)["threads"] == 0
    own.tune_load(str(path))
    assert own.tune_get(9) == e9 and own.tune_get(10) == e10 and own.tune_get(99) == eb
    assert cpx.pi_batch(xs, ctx=own) == want
    bad = tmp_path / "bad.json"
    bad.write_text('{"format": "cudapix_b200 tuning 1", "entries": [\n {"decade": 9, "threads": 7}\n]}\n')
    with pytest.raises(cpx.CpxError):
        own.tune_load(str(bad))
    with pytest.raises(cpx.CpxError):
        own.autotune_batch(xs[:3])
    own.close()


def test_tuning_file_layout_does_not_matter(cpx, tmp_path):
    """The committed table read from its own file and from the same JSON on one
    line gives the same entries (per decade, batch, per-decade batch alpha)."""
    import json
    import os

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    src = os.path.join(root, "cudapix_b200", "tuning", "b200.json")
    one = tmp_path / "one_line.json"
    one.write_text(json.dumps(json.load(open(src))))
    a, b = cpx.Context(0), cpx.Context(0)
    a.tune_load(src)
    b.tune_load(str(one))
    decades = [e["decade"] for e in json.load(open(src))["entries"]]
    assert len(decades) >= 10
    for d in decades:
        assert a.tune_get(d) == b.tune_get(d), d
    a.close()
    b.close()
