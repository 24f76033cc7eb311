"""The C++ drop-in header (include/cudapix_compat.hpp) compiles with the
reference's call shapes and links against the library.  CPU only (the
program is built, not run)."""
import os
import subprocess
import tempfile

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
  uint128_t q = deleglise_rivat128::pi_deleglise_rivat((uint128_t)1 << 70, 0, 6);
  cpx_free(mu); cpx_free(lpf); cpx_free(pt);
  return (int)(a + (uint64_t)b + t + o + (uint64_t)o2 + ph + h + h4 + p + (uint64_t)q + mutest(100));
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
