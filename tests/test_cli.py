"""cpx-pi, the command-line front end (cudapix_b200/cli/cpx_pi.cpp): exact
128-bit parsing of x without a GPU, and one query on the GPU."""
import json
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "cudapix_b200", "bin", "cpx-pi")


@pytest.fixture(scope="module")
def cli():
    if not os.path.exists(CLI):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "cudapix_b200")], check=True)
    return CLI


@pytest.mark.parametrize("expr,val", [
    ("1e20", 10**20), ("2^64+13", 2**64 + 13), ("3*(10^12 - 5) + 2e3", 3 * (10**12 - 5) + 2000),
    ("1_000_000", 10**6), ("2^127 - 1 + 2^127", 2**128 - 1), ("10^38", 10**38),
])
def test_parse(cli, expr, val):
    out = subprocess.run([cli, "--parse", expr], capture_output=True, text=True, check=True).stdout
    assert int(out) == val


@pytest.mark.parametrize("expr", ["2^128", "5-6", "1e", "(1+2", "abc", "2^^3"])
def test_parse_rejects(cli, expr):
    r = subprocess.run([cli, "--parse", expr], capture_output=True, text=True)
    assert r.returncode == 1 and r.stderr.startswith("cpx-pi:")


@pytest.mark.gpu
def test_cli_pi_json(cli, golden, tmp_path):
    r = subprocess.run([cli, "1e12", "--alpha", "10", "--terms", "--json"], capture_output=True, text=True, check=True)
    d = json.loads(r.stdout)
    assert int(d["pi"]) == golden["pi_pow10"]["12"] and d["y"] == 100000
    f = tmp_path / "xs.txt"
    f.write_text("# comment\n1e9\n2^40+15\n\n10^13\n")
    r = subprocess.run([cli, "--batch", str(f), "--json"], capture_output=True, text=True, check=True)
    rows = [json.loads(l) for l in r.stdout.splitlines()]
    assert [int(v["x"]) for v in rows] == [10**9, 2**40 + 15, 10**13]
    assert int(rows[0]["pi"]) == golden["pi_pow10"]["9"] and int(rows[2]["pi"]) == golden["pi_pow10"]["13"]
