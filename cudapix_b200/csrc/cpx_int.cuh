// cpx_int.cuh -- exact integer helpers shared by host and device code.
//
// Replaces the CUDA-uint128 dependency of the reference (its uint128_t,
// mul128, _isqrt/_icbrt/_iqrt call sites are listed at
// src/Deleglise-Rivat/deleglise-rivat.cpp:99-102, src/P2.cu:23,
// src/main.cpp:61,165).  Every root here is an exact floor root computed in
// integers; no floating point value ever reaches a count.
#pragma once
#include <cmath>
#include <cstdint>

#if defined(__CUDACC__)
#define CPX_HD __host__ __device__ __forceinline__
#else
#define CPX_HD inline
#endif

typedef unsigned __int128 u128;
typedef __int128 i128;

// ------------------------------------------------------------------ roots
// x < 2^64: a double estimate of the root corrected to the exact floor root
// by integer comparisons (the estimate is within 2 of the root).  Wider x:
// integer Newton iteration from an over-estimate (a power of two above the
// root), which decreases monotonically to the floor root.

CPX_HD int cpx_bitlen128(u128 x)
{
    uint64_t hi = (uint64_t)(x >> 64), lo = (uint64_t)x;
#if defined(__CUDA_ARCH__)
    if (hi) return 128 - __clzll((long long)hi);
    return lo ? 64 - __clzll((long long)lo) : 0;
#else
    if (hi) return 128 - __builtin_clzll(hi);
    return lo ? 64 - __builtin_clzll(lo) : 0;
#endif
}

CPX_HD uint64_t cpx_isqrt(u128 x)
{
    if (x < 2) return (uint64_t)x;
    if (!(x >> 64)) {
        const uint64_t v = (uint64_t)x;
        uint64_t r = (uint64_t)sqrt((double)v);
        while ((u128)r * r > v) r--;
        while ((u128)(r + 1) * (r + 1) <= v) r++;
        return r;
    }
    int b = cpx_bitlen128(x);
    u128 r = (u128)1 << ((b + 1) / 2); // r >= sqrt(x)
    for (;;) {
        u128 n = (r + x / r) >> 1;
        if (n >= r) break;
        r = n;
    }
    return (uint64_t)r;
}

CPX_HD uint64_t cpx_icbrt(u128 x)
{
    if (x < 8) return x ? 1 : 0;
    if (!(x >> 64)) {
        const uint64_t v = (uint64_t)x;
        uint64_t r = (uint64_t)cbrt((double)v);
        while ((u128)r * r * r > v) r--;
        while ((u128)(r + 1) * (r + 1) * (r + 1) <= v) r++;
        return r;
    }
    int b = cpx_bitlen128(x);
    u128 r = (u128)1 << ((b + 2) / 3); // r >= cbrt(x)
    for (;;) {
        u128 n = (2 * r + x / (r * r)) / 3;
        if (n >= r) break;
        r = n;
    }
    return (uint64_t)r;
}

CPX_HD uint64_t cpx_iroot4(u128 x) { return cpx_isqrt((u128)cpx_isqrt(x)); }

// ------------------------------------------------ 128-by-64-bit division
// floor(n / d) for d >= 1 and a quotient below 2^64 (n < d 2^64): the x/p,
// x/n and x/(p m) of x >= 2^64.  Division by Newton-Raphson reciprocal
// refinement with exact integer correction (Brent and Zimmermann, Modern
// Computer Arithmetic, sections 1.4.1 and 3.4.1):
//   r0 = 1/d rounded to float; one Newton step in double,
//   rd = r0 + r0 (1 - d r0), relative error below 2^-46;
//   q0 = trunc(n * rd), within 2^18 of n/d since n/d < 2^64;
//   the remainder r = n - q0 d is exact in 128 bits (|r| < 2^18 d + d);
//   t = floor(r * rd) is within 1 of floor(r/d) (|r/d| < 2^19), and
//   q0 + t corrected by the sign and size of r - t d is the quotient.
// Every step is an IEEE-rounded operation, so the host and device forms
// return the same value; the host form is checked against the compiler's
// 128-bit division on random and edge operands.
CPX_HD uint64_t cpx_udiv_2by1(u128 n, uint64_t d)
{
    const uint64_t nh = (uint64_t)(n >> 64), nl = (uint64_t)n;
    constexpr double k2p64 = 18446744073709551616.0;
#if defined(__CUDA_ARCH__)
    const double dd = __ull2double_rn(d);
    const double r0 = (double)__frcp_rn(__ull2float_rn(d));
    const double rd = __fma_rn(r0, __fma_rn(-dd, r0, 1.0), r0);
    const double qd = __dmul_rn(__fma_rn(__ull2double_rn(nh), k2p64, __ull2double_rn(nl)), rd);
#else
    const double dd = (double)d;
    const double r0 = (double)(1.0f / (float)d);
    const double rd = std::fma(r0, std::fma(-dd, r0, 1.0), r0);
    const double qd = std::fma((double)nh, k2p64, (double)nl) * rd;
#endif
    uint64_t q = qd >= k2p64 ? ~0ull : (uint64_t)qd;  // truncation
    i128 r = (i128)(n - (u128)q * d);
    const double rr = (double)(int64_t)(uint64_t)((u128)r >> 64) * k2p64 + (double)(uint64_t)r;
#if defined(__CUDA_ARCH__)
    const int64_t t = __double2ll_rd(__dmul_rn(rr, rd));
#else
    const int64_t t = (int64_t)std::floor(rr * rd);
#endif
    q += (uint64_t)t;
    r -= (i128)t * (i128)d;
    while (r < 0) {
        q--;
        r += d;
    }
    while (r >= (i128)d) {
        q++;
        r -= d;
    }
    return q;
}

// --------------------------------------------------------- table lookups
// Compressed prime table: entry w covers the odd numbers 128w+1 .. 128w+127,
// .x = bitmap (bit j <-> 128w + 2j + 1 is prime), .y = number of odd primes
// below 128w.  pi(n) = [n >= 2] + .y + popcount(.x & mask(n)).

struct __align__(16) cpx_pient {
    uint64_t bits;
    uint64_t pre;
};

CPX_HD uint64_t cpx_pi_from_entry(cpx_pient e, uint64_t n)
{
    uint32_t j = (uint32_t)(((n - 1) & 127) >> 1);
    uint64_t mask = (2ull << j) - 1; // j == 63 wraps to all ones
#if defined(__CUDA_ARCH__)
    return 1 + e.pre + (uint64_t)__popcll(e.bits & mask);
#else
    return 1 + e.pre + (uint64_t)__builtin_popcountll(e.bits & mask);
#endif
}

#if defined(__CUDACC__)
__device__ __forceinline__ uint64_t cpx_pi_dev(const cpx_pient *__restrict__ T, uint64_t n)
{
    if (n < 2) return 0;
    const ulonglong2 v = __ldg(reinterpret_cast<const ulonglong2 *>(T) + ((n - 1) >> 7));
    cpx_pient e{v.x, v.y};
    return cpx_pi_from_entry(e, n);
}

// ------------------------------------------------ leaf quotients floor(n / d)
// Leaves and level parameters divide 64-bit values by d < 2^32.  The quotient
// is taken from the double product n * (1/d) and made exact in integers,
// instead of the general 64-bit division routine:
//   r0 = 1/d rounded to float, then one Newton-Raphson step in double
//   rd = r0 + r0 (1 - d r0), relative error < 2^-45;
//   q0 = trunc(n * rd) is within 2^-44.9 n/d + 1 of the quotient.
//   n/d < 2^44: q0 is floor(n/d) - 1, floor(n/d) or floor(n/d) + 1, and the
//   sign of n - q0 d settles which.
//   larger n/d (< 2^64): the remainder r = n - q0 d is below 2^52 in
//   magnitude, so r and r * rd are exact enough in double; t = floor(r * rd)
//   corrected by the sign of r - t d gives floor(n/d) = q0 + t.
// d >= 2^32 uses the hardware path.
static __device__ __noinline__ uint64_t cpx_udiv_slow(uint64_t n, uint64_t d) { return n / d; }

__device__ __forceinline__ uint64_t cpx_udiv_leaf(uint64_t n, uint64_t d)
{
    if (d >> 32) return cpx_udiv_slow(n, d);
    const uint32_t d32 = (uint32_t)d;
    const double r = (double)__frcp_rn(__uint2float_rn(d32));
    const double dd = (double)d32;
    const double e = __fma_rn(-dd, r, 1.0);
    const double rd = __fma_rn(r, e, r);
    uint64_t u = __double2ull_rz(__dmul_rn(__ull2double_rn(n), rd));
    const int64_t rem = (int64_t)(n - u * d);
    if ((n >> 44) < d) {
        if (rem < 0) u--;
        else if (rem >= (int64_t)d) u++;
        return u;
    }
    int64_t t = __double2ll_rd(__dmul_rn(__ll2double_rn(rem), rd));
    const int64_t r2 = rem - t * (int64_t)d32;
    if (r2 < 0) t--;
    else if (r2 >= (int64_t)d32) t++;
    return u + (uint64_t)t;
}
__device__ __forceinline__ uint64_t cpx_qdiv(uint64_t n, uint64_t d) { return cpx_udiv_leaf(n, d); }
// 128-bit dividend: x/p is below 2^64 for x < 2^64 p, so most leaf
// quotients of the 128-bit path take the 64-bit route; a wider dividend with
// a quotient below 2^64 takes cpx_udiv_2by1, and only quotients of 2^64 or
// more the compiler's 128-bit division
static __device__ __noinline__ u128 cpx_udiv128_slow(u128 n, uint64_t d) { return n / (u128)d; }
__device__ __forceinline__ u128 cpx_qdiv(u128 n, uint64_t d)
{
    const uint64_t nh = (uint64_t)(n >> 64);
    if (!nh) return (u128)cpx_udiv_leaf((uint64_t)n, d);
    if (nh < d) return (u128)cpx_udiv_2by1(n, d);
    return cpx_udiv128_slow(n, d);
}

#endif  // __CUDACC__

// floor(n / d) for 1 <= d < 2^32 and n < 2^53 (nd = n as a double, exact)
// with a quotient below 2^41 (every n < 2^40 qualifies), from a reciprocal
// estimate r0 with |d r0 - 1| < 2^-22 (the hardware approximation of 1/d
// rounded to float: at most 1 ulp of the approximation plus the rounding of
// d to float).  One Newton-Raphson step with its target raised by 2^-42,
//   rd = r0 + r0 (1 + 2^-42 - d r0) = (1/d) (1 - e^2 + 2^-42 (1 + e)),  e = d r0 - 1,
// lies in (1/d, (1/d)(1 + 2^-41.9)) after the two roundings of the fused
// steps (e^2 < 2^-44), so t = n rd rounded toward +infinity satisfies
// n/d <= t < n/d + (n/d) 2^-41.8 < n/d + 0.6: trunc(t) is floor(n/d) or
// floor(n/d) + 1, and a single comparison of q d with n settles which
// (q d <= n + d < 2^54).
// QT = uint32_t when floor(n/d) < 2^32 - 1.  On the device d becomes a
// double and trunc(t) an integer through the exponent 2^52 (2^52 + d is
// exact; 2^52 + t rounded toward zero is 2^52 + trunc(t) for t < 2^52), on
// the double pipe rather than the conversion unit.  The host form takes r0
// from its caller and rounds the product up exactly (error-free product,
// then the next double up when the rounded-to-nearest product was low).
template <class QT> CPX_HD QT cpx_quot40_est(double nd, uint32_t d, float r0)
{
    const double r = (double)r0;
#if defined(__CUDA_ARCH__)
    const double dd = __hiloint2double(0x43300000, (int)d) - 0x1p52;
    const double rd = fma(r, fma(-dd, r, 1.0 + 0x1p-42), r);
    const double tt = __dadd_rz(__dmul_ru(nd, rd), 0x1p52);
    if constexpr (sizeof(QT) == 4) return (QT)__double2loint(tt);
    else return (QT)(__double_as_longlong(tt) & 0xFFFFFFFFFFFFFull);
#else
    const double rd = fma(r, fma(-(double)d, r, 1.0 + 0x1p-42), r);
    double t = nd * rd;
    if (std::fma(nd, rd, -t) > 0) t = std::nextafter(t, INFINITY);
    return (QT)t;
#endif
}
template <class QT> CPX_HD QT cpx_quot40_core(uint64_t n, double nd, uint32_t d, float r0)
{
    const QT q = cpx_quot40_est<QT>(nd, d, r0);
    return q - (QT)((uint64_t)q * d > n);
}
// The same quotient for d < 2^31 and floor(n/d) < 2^31 - 1, corrected in 32
// bits: n - q d lies in [0, d) or [-d, 0), so its low 32 bits are below d
// or at least 2^32 - d > d.
CPX_HD uint32_t cpx_quot40_small(uint64_t n, double nd, uint32_t d, float r0)
{
    const uint32_t q = cpx_quot40_est<uint32_t>(nd, d, r0);
    return q - (uint32_t)((uint32_t)n - q * d >= d);
}

#if defined(__CUDACC__)
__device__ __forceinline__ float cpx_rcp_approx(uint32_t d)
{
    float rf;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(rf) : "f"(__uint2float_rn(d)));
    return rf;
}
__device__ __forceinline__ uint64_t cpx_quot40(uint64_t n, double nd, uint32_t d)
{
    return cpx_quot40_core<uint64_t>(n, nd, d, cpx_rcp_approx(d));
}

// pi(floor(n / d)) of an easy leaf whose dividend n = x/p is below 2^40, with
// d = q < 2^31 and a quotient u below 2^30 (u < sqrt(x), x < 2^60 when x/p <
// 2^40), by cpx_quot40_small.
// u >= 2; pi(u) = 1 + entry prefix + bits 0..j of the entry's bitmap,
// j = ((u - 1) mod 128) / 2.
__device__ __forceinline__ uint64_t cpx_pi_quot40(const cpx_pient *__restrict__ T, uint64_t n, double nd, uint32_t d)
{
    const uint32_t m = cpx_quot40_small(n, nd, d, cpx_rcp_approx(d)) - 1;
    const ulonglong2 e = __ldg(reinterpret_cast<const ulonglong2 *>(T) + (m >> 7));
    const uint32_t j = (m & 127u) >> 1;
    return 1 + e.y + (uint64_t)__popcll(e.x << (63 - j));
}

// floor(n / d) for n < 2^53 and a quotient below 2^44, d < 2^32, nd = n as a
// double: the reciprocal rounded to nearest (relative error 2^-24) and one
// Newton-Raphson step give an error below 2^-46, so trunc(n rd) is within 1
// of the quotient; the remainder's sign and size fix it without a branch.
// The easy leaves of x >= 2^64 (x/p < 2^53 for p > x^(1/4) when x < 2^106).
__device__ __forceinline__ uint64_t cpx_quot53(uint64_t n, double nd, uint32_t d)
{
    const double r = (double)__frcp_rn(__uint2float_rn(d));
    const double rd = __fma_rn(r, __fma_rn(-(double)d, r, 1.0), r);
    const uint64_t u = __double2ull_rz(__dmul_rn(nd, rd));
    const int64_t rem = (int64_t)(n - u * d);
    return u + (rem >= (int64_t)d) - (rem < 0);
}

// pi(u) for 2 <= u from the compressed table, without the small-u test
__device__ __forceinline__ uint64_t cpx_pi_ge2(const cpx_pient *__restrict__ T, uint64_t u)
{
    const uint64_t m = u - 1;
    const ulonglong2 e = __ldg(reinterpret_cast<const ulonglong2 *>(T) + (m >> 7));
    const uint32_t j = ((uint32_t)m & 127u) >> 1;
    return 1 + e.y + (uint64_t)__popcll(e.x << (63 - j));
}

// ------------------------------------------------ 128-bit atomic accumulate
// Two 64-bit atomics; the carry out of the low word is added to the high word
// by the same thread, which makes the final 128-bit total exact in any order.
__device__ __forceinline__ void cpx_atomic_add_i128(unsigned long long *dst, i128 v)
{
    unsigned long long lo = (unsigned long long)(u128)v;
    unsigned long long hi = (unsigned long long)((u128)v >> 64);
    unsigned long long old = atomicAdd(dst, lo);
    hi += (old + lo < old) ? 1ull : 0ull;
    if (hi) atomicAdd(dst + 1, hi);
}

__device__ __forceinline__ i128 cpx_shfl_down_i128(i128 v, int d)
{
    unsigned long long lo = (unsigned long long)(u128)v, hi = (unsigned long long)((u128)v >> 64);
    lo = __shfl_down_sync(0xffffffffu, lo, d);
    hi = __shfl_down_sync(0xffffffffu, hi, d);
    return (i128)(((u128)hi << 64) | lo);
}

__device__ __forceinline__ i128 cpx_warp_sum_i128(i128 v)
{
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) v += cpx_shfl_down_i128(v, d);
    return v;
}

// Block-wide sum of an i128 held by every thread; result valid in thread 0.
// `sh` needs 32 entries.  All threads of the block must call it.
__device__ __forceinline__ i128 cpx_block_sum_i128(i128 v, i128 *sh)
{
    v = cpx_warp_sum_i128(v);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) sh[w] = v;
    __syncthreads();
    i128 r = 0;
    if (threadIdx.x < 32) {
        r = (threadIdx.x < (blockDim.x >> 5)) ? sh[threadIdx.x] : (i128)0;
        r = cpx_warp_sum_i128(r);
    }
    return r;
}
#endif
