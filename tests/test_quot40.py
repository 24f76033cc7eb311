"""cpx_quot40_core and cpx_quot40_small (cudapix_b200/csrc/cpx_int.cuh), the
quotient floor(n / d) for n < 2^53, d < 2^32 and a quotient below 2^41 (d <
2^31 for the form corrected in 32 bits) of the leaves and of P2: their host
forms, given every reciprocal estimate the hardware approximation may return
(the correctly rounded reciprocal of float(d) and the floats one ulp either
side of it), against integer division on 5 x 10^7 random operands and on edge
operands (exact multiples and their neighbours, divisors that do not fit a
float, dividends near 2^40 and 2^53).  The host form rounds the product up
exactly, as the device's __dmul_ru does; the device form is checked through
the leaf and P2 terms of the GPU tests.  CPU only."""
import os
import subprocess
import tempfile

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

HARNESS = r"""
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <initializer_list>
#define __align__(n) alignas(n)
#include "cpx_int.cuh"

static uint64_t s[2] = {0x243F6A8885A308D3ull, 0x13198A2E03707344ull};
static uint64_t rnd()  // xorshift128+
{
    uint64_t a = s[0], b = s[1];
    s[0] = b;
    a ^= a << 23;
    s[1] = a ^ b ^ (a >> 17) ^ (b >> 26);
    return s[1] + b;
}
static long bad = 0, checked = 0;
static void check(uint64_t n, uint64_t d)
{
    if (!d || d >> 32 || n >> 53 || (n / d) >> 41) return;
    const uint64_t want = n / d;
    const float rn = 1.0f / (float)d;
    for (int k = -1; k <= 1; k++) {
        const float r0 = k < 0 ? std::nextafterf(rn, 0.0f) : (k > 0 ? std::nextafterf(rn, 1.0f) : rn);
        if (std::fabs((double)d * (double)r0 - 1.0) >= 0x1p-22) {
            if (bad++ < 5) std::printf("ESTIMATE d=%llu k=%d outside the documented bound\n", (unsigned long long)d, k);
            continue;
        }
        const uint64_t got = cpx_quot40_core<uint64_t>(n, (double)n, (uint32_t)d, r0);
        if (got != want && bad++ < 5)
            std::printf("MISMATCH n=%llu d=%llu k=%d got=%llu want=%llu\n", (unsigned long long)n,
                        (unsigned long long)d, k, (unsigned long long)got, (unsigned long long)want);
        if (d < (1ull << 31) && want < 0x7FFFFFFEull) {
            const uint32_t gs = cpx_quot40_small(n, (double)n, (uint32_t)d, r0);
            if (gs != want && bad++ < 5)
                std::printf("MISMATCHS n=%llu d=%llu k=%d got=%u\n", (unsigned long long)n, (unsigned long long)d, k, gs);
        }
        if (want < 0xFFFFFFFEull) {
            const uint32_t g32 = cpx_quot40_core<uint32_t>(n, (double)n, (uint32_t)d, r0);
            if (g32 != want && bad++ < 5)
                std::printf("MISMATCH32 n=%llu d=%llu k=%d got=%u\n", (unsigned long long)n, (unsigned long long)d,
                            k, g32);
        }
        checked++;
    }
}
int main(int argc, char **argv)
{
    const long N = atol(argv[1]);
    for (long i = 0; i < N; i++) {
        const int bd = 1 + (int)(rnd() % 32);  // divisor bit length
        uint64_t d = (rnd() >> (64 - bd)) | (1ull << (bd - 1));
        const int bq = (int)(rnd() % 41);  // quotient bit length
        const uint64_t q = bq ? (rnd() >> (64 - bq)) : 0, r = rnd() % d;
        check(q * d + r, d);
        check(q * d, d);
        if (q) check(q * d - 1, d);
        check(rnd() >> 24, d);
        check(rnd() >> 11, d);                                  // n < 2^53 (quotient < 2^41 only)
        const uint64_t q2 = rnd() >> (64 - 1 - (int)(rnd() % 41));  // quotient < 2^41
        if (q2 && d < (1ull << 53) / q2) check(q2 * d + rnd() % d, d);
    }
    const uint64_t ds[] = {1, 2, 3, 7, 127, 65535, (1ull << 24) - 1, 1ull << 24, (1ull << 24) + 1, (1ull << 24) + 3,
                           1000003, 2147483647ull, 2147483648ull, 0xFFFFFFFBull, 0xFFFFFFFFull};
    for (uint64_t d : ds)
        for (uint64_t n : {0ull, 1ull, (1ull << 40) - 1, (1ull << 40) - 2, (1ull << 39), 1099511627689ull,
                           (1ull << 53) - 1, (1ull << 53) - 2, 9007199254740881ull})
            for (int64_t o = -2; o <= 2; o++) {
                check(n + o, d);
                const uint64_t m = (n / d) * d;
                check(m + o, d);
            }
    std::printf("bad %ld checked %ld\n", bad, checked);
    return bad != 0;
}
"""


def test_quot40_matches_integer_division():
    with tempfile.TemporaryDirectory() as t:
        src = os.path.join(t, "q.cpp")
        with open(src, "w") as f:
            f.write(HARNESS)
        exe = os.path.join(t, "q")
        r = subprocess.run(["g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "cudapix_b200", "csrc"), src, "-o", exe],
                           capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
        r = subprocess.run([exe, str(10**7)], capture_output=True, text=True, timeout=600)
        assert r.returncode == 0 and "bad 0" in r.stdout, r.stdout
