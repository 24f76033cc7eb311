"""The C++ drop-in header (include/cudapix_compat.hpp): a program written
against the reference's call shapes compiles and links against the library
(CPU), and on the GPU a program calling the reference's signatures prints
values that equal the CPU oracle's (P2, S2_trivial, Ordinary, S2hard with
and without maxPrime, pi_deleglise_rivat, mutest, the dense and windowed pi
tables, Phi and Phisieve; and the 128-bit overloads at x = 10^20)."""
import json
import os
import subprocess
import tempfile

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PROGRAM = r"""
#include "cudapix_compat.hpp"
int main() {
  uint64_t a = P2((uint64_t)1000000000000ull, 100000);
  uint128_t b = P2((uint128_t)1 << 70, 100000);
  uint64_t t = S2_trivial((uint64_t)1000000000000ull, 100000);
  uint64_t o = Ordinary((uint64_t)1000000000000ull, 100000, 6);
  uint128_t o2 = Ordinary((uint128_t)1 << 70, 100000, 6);
  int8_t *mu = gen_d_mu<uint32_t>(0u, 1000u);
  uint32_t *lpf = gen_d_lpf<uint32_t>(0u, 1000u);
  uint32_t *pt = get_d_piTable(1000);
  PiTable w(1000000, 0, 4096); w.getCurrent(); w.getNextDown();
  w.set_pi_base(w.get_pi_base()); w.allocate(); w.reallocate(); (void)w.getNextBaseDown();
  PiTable big(1 << 20); (void)big.setMaxRange();
  Phi f(1000); uint64_t ph = f.phi(100000, 5);
  f.makeModCache(8); uint32_t *fl = f.get_d_lpf(); uint32_t np = f.get_primeListLength();
  uint32_t *hp = f.get_h_primeList(); uint32_t *dp = f.get_d_primeList();
  Phi g(1 << 20, 2000); (void)g.get_h_primeList();
  Phisieve s(1000, 1 << 16); s.firstSieve(6); s.markNext(); s.updateCount();
  s.set_a_current(s.get_a_current()); s.markNext();
  (void)fl; (void)np; (void)hp; (void)dp;
  uint64_t h = S2hardHost::S2hard(1000000000000ull, 100000, 6);
  uint64_t h4 = S2hardHost::S2hard(1000000000000ull, 100000, 6, 1000);
  uint64_t p = deleglise_rivat64::pi_deleglise_rivat(1000000000000ull, 100000, 6);
  uint64_t gp = GourdonVariant64::piGourdon(1000000000000ull, 100000, 6);
  GourdonVariant64 gv(1000000000000ull, 100000, 6);
  int64_t gs = gv.sigma() + (int64_t)gv.A() + (int64_t)gv.B() + (int64_t)gv.C() + (int64_t)gv.D() + (int64_t)gv.phi_0();
  uint128_t q = deleglise_rivat128::pi_deleglise_rivat((uint128_t)1 << 70, 0, 6);
  cpx_free(mu); cpx_free(lpf); cpx_free(pt);
  return (int)(a + (uint64_t)b + t + o + (uint64_t)o2 + ph + h + h4 + p + (uint64_t)q + mutest(100) + gp + (uint64_t)gs);
}
"""


def test_compat_header_compiles_and_links():
    with tempfile.TemporaryDirectory() as d:
        src = os.path.join(d, "t.cpp")
        with open(src, "w") as f:
            f.write(PROGRAM)
        out = os.path.join(d, "t")
        r = subprocess.run(
            ["g++", "-std=c++17", "-O1", "-Wall", "-I", os.path.join(ROOT, "include"), src,
             "-L", os.path.join(ROOT, "cudapix_b200", "lib"), "-lcudapix_b200", "-o", out],
            capture_output=True, text=True)
        assert r.returncode == 0, r.stderr


RUN_PROGRAM = r"""
#include <cinttypes>
#include <string>
#include "cudapix_compat.hpp"

static std::string dec(uint128_t v)
{
  if (!v) return "0";
  std::string s;
  while (v) { s.insert(s.begin(), char('0' + (int)(v % 10))); v /= 10; }
  return s;
}
static std::string sdec(uint128_t v)
{
  return (v >> 127) ? "-" + dec(~v + 1) : dec(v);
}
static uint64_t sum_dev(const uint32_t *d, size_t n)
{
  std::vector<uint32_t> h(n);
  if (cpx_copy_to_host(h.data(), d, n * 4) != CPX_OK) std::abort();
  uint64_t s = 0;
  for (size_t i = 0; i < n; i++) s += (uint64_t)h[i] * (i % 7 + 1);
  return s;
}

int main(int argc, char **argv)
{
  const uint64_t x = 1000000000000ull, y = 100000;
  std::printf("P2 %" PRIu64 "\n", P2(x, y));
  std::printf("trivial %" PRIu64 "\n", S2_trivial(x, y));
  std::printf("ordinary %" PRId64 "\n", (int64_t)Ordinary(x, y, 6));
  std::printf("hard %" PRId64 "\n", (int64_t)S2hardHost::S2hard(x, y, 6));
  std::printf("hard_maxprime %" PRId64 "\n", (int64_t)S2hardHost::S2hard(x, y, 6, 1000));
  std::printf("pi64 %" PRIu64 "\n", deleglise_rivat64::pi_deleglise_rivat(x, y, 6));
  std::printf("pi64_default_y %" PRIu64 "\n", deleglise_rivat64::pi_deleglise_rivat(x, 0, 6));
  std::printf("mutest %" PRId64 "\n", mutest(1000000));
  GourdonVariant64 gv(x, y, 6);
  std::printf("gA %" PRIu64 "\ngB %" PRIu64 "\ngC %" PRIu64 "\ngD %" PRId64 "\ngphi0 %" PRId64 "\ngsigma %" PRId64 "\n",
              gv.A(), gv.B(), gv.C(), (int64_t)gv.D(), (int64_t)gv.phi_0(), gv.sigma());
  std::printf("gpi %" PRIu64 "\n", GourdonVariant64::piGourdon(x, y, 6));
  uint32_t *pt = get_d_piTable(100000);
  std::printf("dense_sum %" PRIu64 "\n", sum_dev(pt, 50000));
  cpx_free(pt);
  PiTable w(2000000, 1000000, 200000);
  w.getCurrent();
  uint32_t *dn = w.getNextDown();
  std::printf("win_base %" PRIu64 "\n", w.get_base());
  std::printf("win_pi_base %" PRIu64 "\n", w.get_pi_base());
  std::printf("win_sum %" PRIu64 "\n", sum_dev(dn, 100000));
  Phi f(1000000);
  std::printf("phi %" PRIu64 "\n", f.phi(100000, 5));
  Phisieve s(1000, 1 << 16);
  s.firstSieve(6);
  std::printf("phisieve6_sum %" PRIu64 "\n", sum_dev(s.getCountDevice(), 1 << 16));
  s.markNext(); s.markNext(); s.markNext();
  s.updateCount();
  std::printf("phisieve9_sum %" PRIu64 "\n", sum_dev(s.getCountDevice(), 1 << 16));
  if (argc > 1) {
    const uint128_t X = (uint128_t)10000000000ull * 10000000000ull;  // 10^20
    const uint64_t Y = 74265408;
    std::printf("P2_128 %s\n", dec(P2(X, Y)).c_str());
    std::printf("trivial_128 %s\n", dec(S2_trivial(X, Y)).c_str());
    std::printf("ordinary_128 %s\n", sdec(Ordinary(X, Y, 6)).c_str());
    std::printf("pi128 %s\n", dec(deleglise_rivat128::pi_deleglise_rivat(X, Y, 6)).c_str());
  }
  return 0;
}
"""


def _weighted_sum(a):
    a = np.asarray(a, dtype=np.uint64)
    w = (np.arange(len(a), dtype=np.uint64) % 7) + 1
    return int((a * w).sum())


@pytest.mark.gpu
def test_compat_program_runs_and_matches_oracle(orc, golden):
    """The reference's C++ call shapes, run on the GPU through the header."""
    with tempfile.TemporaryDirectory() as d:
        src = os.path.join(d, "r.cpp")
        with open(src, "w") as f:
            f.write(RUN_PROGRAM)
        exe = os.path.join(d, "r")
        libdir = os.path.join(ROOT, "cudapix_b200", "lib")
        r = subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-I", os.path.join(ROOT, "include"), src,
                            "-L", libdir, "-lcudapix_b200", "-Wl,-rpath," + libdir, "-o", exe],
                           capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
        r = subprocess.run([exe, "wide"], capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stderr
    got = dict(line.split(" ", 1) for line in r.stdout.strip().splitlines())
    x, y = 10**12, 10**5
    assert int(got["P2"]) == orc.P2(x, y)
    assert int(got["trivial"]) == orc.trivial(x, y)
    assert int(got["ordinary"]) == orc.ordinary(x, y, 6)
    assert int(got["hard"]) == orc.hard(x, y, 6)
    assert int(got["hard_maxprime"]) == orc.hard(x, y, 6)
    assert int(got["pi64"]) == int(got["pi64_default_y"]) == golden["pi_pow10"]["12"]
    assert int(got["mutest"]) == orc.mertens(10**6)
    g = orc.pi_gourdon(x, y, 6)
    for k in ("A", "B", "C", "D", "phi0", "sigma"):
        assert int(got["g" + k]) == g[k], k
    assert int(got["gpi"]) == g["pi"] == golden["pi_pow10"]["12"]
    assert int(got["dense_sum"]) == _weighted_sum(orc.pitable_dense(100000))
    base = int(got["win_base"])
    assert base == 1_800_000
    t, pb = orc.pitable_window(base, 200_000)
    assert int(got["win_pi_base"]) == pb == orc.pi_sieve(base - 1)
    assert int(got["win_sum"]) == _weighted_sum(t[:100_000])
    assert int(got["phi"]) == orc.phi(10**5, 6)  # the reference's a excludes the first a + 1 primes
    assert int(got["phisieve6_sum"]) == _weighted_sum(orc.phisieve_counts(6, 1 << 16))
    assert int(got["phisieve9_sum"]) == _weighted_sum(orc.phisieve_counts(9, 1 << 16))
    with open(os.path.join(ROOT, "tests", "golden", "terms_1e20.json")) as f:
        t20 = json.load(f)
    assert int(got["P2_128"]) == int(t20["P2"])
    assert int(got["trivial_128"]) == int(t20["trivial"])
    assert int(got["ordinary_128"]) == int(t20["ordinary"])
    assert int(got["pi128"]) == golden["pi_pow10"]["20"]
