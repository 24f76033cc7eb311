/*
 * oracle.h -- CPU restatement of the Deleglise-Rivat term pipeline of
 * curtisseizert/CUDApix, used ONLY as test infrastructure (the checker).
 *
 * Nothing in the product library links, loads or calls this code.  Only the
 * tests, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it.
 *
 * Parity status: the reference ships no tests, fixtures or golden vectors and
 * cannot be built here (CUDASieve and CUDA-uint128 are not vendored), so the
 * oracle is pinned against published values of pi(10^k) (OEIS A006880) and
 * against vectors generated with sympy (tests/golden/make_golden.py), not
 * against outputs of the reference itself.
 *
 * 128-bit quantities cross the C ABI as (lo, hi) pairs of uint64_t; signed
 * results are two's-complement 128-bit values split the same way.
 */
#ifndef CPX_ORACLE_H
#define CPX_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* exact integer roots of the 128-bit value (hi:lo) */
uint64_t orc_isqrt(uint64_t lo, uint64_t hi);
uint64_t orc_icbrt(uint64_t lo, uint64_t hi);
uint64_t orc_iroot4(uint64_t lo, uint64_t hi);
/* alpha(x) of src/main.cpp:128-194 in per mille (chooses y only). */
uint32_t orc_alpha_milli(uint64_t lo, uint64_t hi);

/* pi(x) by an OpenMP segmented sieve of Eratosthenes (independent count). */
uint64_t orc_pi_sieve(uint64_t x);
/* pi(x) by Lehmer's formula with a sieve-built pi table to x^(3/4). */
uint64_t orc_pi_lehmer(uint64_t x);
/* primes in [lo, hi) written to out (capacity cap); returns the count found. */
uint64_t orc_primes(uint64_t lo, uint64_t hi, uint64_t *out, uint64_t cap);

/* mu(n), lpf(n) for odd n = lo + 2i + 1, i < (hi - lo)/2, lo even.
 * lpf(1) = 0xFFFFFFFF (src/sieve/lpf_mu.cu:54); lpf(p) = p for primes. */
void orc_mu_lpf(uint64_t lo, uint64_t hi, int8_t *mu, uint32_t *lpf);
/* Mertens sum over 1 <= n < top (src/mutest.cu:6-19 semantics). */
int64_t orc_mertens(uint64_t top);
/* dense pi table, get_d_piTable layout: out[k] = pi(2k - 1), k < hi/2. */
void orc_pitable_dense(uint64_t hi, uint32_t *out);
/* windowed pi table: out[k] = pi(base + 2k - 1) - pi(base - 1), k < range/2 + 2. */
void orc_pitable_window(uint64_t base, uint64_t range, uint32_t *out, uint64_t *pi_base);
/* phi(x, a): #{1 <= n <= x : n has no prime factor among the first a primes}. */
uint64_t orc_phi(uint64_t x, uint32_t a);
/* Phisieve counts: out[i] = phi(2i - 1, a) for i < nbits (exclusive scan of
 * the odd-only bit sieve of the first a primes, src/sieve/phisieve_host.cu:88-96). */
void orc_phisieve_counts(uint32_t a, uint64_t nbits, uint32_t *out);

/* Terms.  x = (x_hi:x_lo).  out[0..1] = signed 128-bit result (lo, hi). */
void orc_P2(uint64_t x_lo, uint64_t x_hi, uint64_t y, uint64_t *out);
void orc_P2_windowed(uint64_t x_lo, uint64_t x_hi, uint64_t y, uint64_t *out);
void orc_leaf_counts(uint64_t x_lo, uint64_t x_hi, uint64_t y, uint32_t c, uint64_t *out);
void orc_trivial(uint64_t x_lo, uint64_t x_hi, uint64_t y, uint64_t *out);
void orc_ordinary(uint64_t x_lo, uint64_t x_hi, uint64_t y, uint32_t c, uint64_t *out);
void orc_easy(uint64_t x_lo, uint64_t x_hi, uint64_t y, uint32_t c, uint64_t *out);
void orc_hard(uint64_t x_lo, uint64_t x_hi, uint64_t y, uint32_t c, uint64_t *out);

/* Full pi(x) through the term identity
 *   pi(x) = ordinary + trivial + easy + hard + pi(y) - 1 - P2
 * (src/Deleglise-Rivat/deleglise-rivat.cpp:77).  terms[2k..2k+1] receives
 * P2, ordinary, trivial, easy, hard, pi(y), pi(x) as signed 128-bit pairs.
 * nthreads <= 0 uses every host thread. */
void orc_pi_dr(uint64_t x_lo, uint64_t x_hi, uint64_t y, uint32_t c, int nthreads,
               uint64_t *terms);

/* The reference's OpenMP host terms (Gourdon's A and C, src/Gourdon/A2_cpu.cpp,
 * src/Gourdon/C_cpu.cpp), restated for the timed CPU baseline; x < 2^64.
 * out[0..1] = the 128-bit sum (lo, hi).  nthreads <= 0 uses every host thread. */
void orc_gourdon_A(uint64_t x, uint64_t y, int nthreads, uint64_t *out);
void orc_gourdon_C(uint64_t x, uint64_t y, int nthreads, uint64_t *out);

/* pi(x) through Gourdon's decomposition pi(x) = A - B + C + D + Phi0 + Sigma,
 * a second split of the same leaves (x < 2^64).  terms[2k..2k+1] receives A,
 * B, C, D, Phi0, Sigma, pi(x) as signed 128-bit pairs. */
void orc_pi_gourdon(uint64_t x, uint64_t y, uint32_t c, int nthreads, uint64_t *terms);

#ifdef __cplusplus
}
#endif
#endif
