"""cpx_udiv_2by1 (cudapix_b200/csrc/cpx_int.cuh), the 128-by-64-bit division
of the 128-bit path (x / p, x / n and x / (p m) for x >= 2^64): its host form
against the compiler's unsigned __int128 division on 10^8 random operands of
every size and on edge operands.  The device form performs the same
IEEE-rounded steps (its GPU check is the pi(10^20) test).  CPU only."""
import os
import subprocess
import tempfile

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

HARNESS = r"""
#include <cstdio>
#include <cstdlib>
#include <initializer_list>
#define __align__(n) alignas(n)
#include "cpx_int.cuh"

static uint64_t s[2] = {0x9E3779B97F4A7C15ull, 0xD1B54A32D192ED03ull};
static uint64_t rnd()  // xorshift128+
{
    uint64_t a = s[0], b = s[1];
    s[0] = b;
    a ^= a << 23;
    s[1] = a ^ b ^ (a >> 17) ^ (b >> 26);
    return s[1] + b;
}
static long bad = 0;
static void check(u128 n, uint64_t d)
{
    if (!d || (uint64_t)(n >> 64) >= d) return;
    const uint64_t want = (uint64_t)(n / d), got = cpx_udiv_2by1(n, d);
    if (got != want && bad++ < 5)
        std::printf("MISMATCH n=%016llx%016llx d=%llu got=%llu want=%llu\n", (unsigned long long)(n >> 64),
                    (unsigned long long)n, (unsigned long long)d, (unsigned long long)got, (unsigned long long)want);
}
int main(int argc, char **argv)
{
    const long N = atol(argv[1]);
    for (long i = 0; i < N; i++) {
        const int bd = 1 + (int)(rnd() % 64);  // divisor bit length
        uint64_t d = rnd() >> (64 - bd);
        d |= 1ull << (bd - 1);
        const uint64_t q = rnd() >> (rnd() % 64), r = d > 1 ? rnd() % d : 0;
        check((u128)q * d + r, d);  // quotient and remainder of every size
        check(((u128)(rnd() % d) << 64) | rnd(), d);
    }
    const uint64_t ds[] = {1, 2, 3, 7, 0xFFFFFFFFull, 0x100000000ull, 0x100000001ull, 1ull << 52, (1ull << 53) + 1,
                           1ull << 63, (1ull << 63) + 1, ~0ull, ~0ull - 1, 1000000007ull, 74265408ull};
    for (uint64_t d : ds)
        for (uint64_t q : {0ull, 1ull, 2ull, (1ull << 53) - 1, 1ull << 53, (1ull << 63), ~0ull - 1, ~0ull})
            for (uint64_t r : {(uint64_t)0, (uint64_t)1, d / 2, d - 1}) {
                if (r >= d) continue;
                const u128 n = (u128)q * d + r;
                check(n, d);
                if (n) check(n - 1, d);
            }
    std::printf("bad %ld\n", bad);
    return bad != 0;
}
"""


def test_udiv_2by1_matches_int128_division():
    with tempfile.TemporaryDirectory() as t:
        src = os.path.join(t, "h.cpp")
        with open(src, "w") as f:
            f.write(HARNESS)
        exe = os.path.join(t, "h")
        r = subprocess.run(["g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "cudapix_b200", "csrc"), src, "-o", exe],
                           capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
        r = subprocess.run([exe, str(5 * 10**7)], capture_output=True, text=True, timeout=600)
        assert r.returncode == 0 and "bad 0" in r.stdout, r.stdout
