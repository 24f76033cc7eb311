// cudapix_compat.hpp -- the reference's C++ term entry points, header-only,
// over the C ABI of include/cpx.h.  A caller of curtisseizert/CUDApix swaps
// its includes for this header and links libcudapix_b200.so; the calls keep
// their names, argument meanings and return types:
//
//   uint64_t  P2(uint64_t x, uint64_t y)              include/P2.cuh:16
//   uint128_t P2(uint128_t x, uint64_t y)             include/P2.cuh:17
//   uint64_t  S2_trivial(uint64_t x, uint64_t y)      include/trivial.cuh:8
//   uint128_t S2_trivial(uint128_t x, uint64_t y)     include/trivial.cuh:12
//   uint64_t  Ordinary(uint64_t x, uint64_t y, uint16_t c)   include/ordinary.cuh:6
//   uint128_t Ordinary(uint128_t x, uint64_t y, uint16_t c)  include/ordinary.cuh:7
//   int64_t   mutest(uint64_t top)                    include/mutest.cuh:3
//   uint32_t* get_d_piTable(uint32_t hi)              include/pitable.cuh:7
//   class PiTable                                     include/pitable.cuh:12-51
//   class Phi                                         include/phi.cuh:17-36
//   class Phisieve                                    include/sieve/phisieve_host.cuh:6-40
//   gen_d_lpf / gen_h_lpf / gen_d_mu / gen_h_mu / gen_d_mu_lpf
//                                                     include/sieve/lpf_mu.cuh:12-24
//   S2hardHost::S2hard(x, y, c)                       include/sieve/S2_hard_host.cuh:35
//   GourdonVariant64 (piGourdon, pi, A, B, C, sigma, phi_0)
//                                                     include/Gourdon/gourdonvariant.hpp:7-56
//   deleglise_rivat64/128::pi_deleglise_rivat(x, y, c)
//                                                     include/Deleglise-Rivat/deleglise-rivat.hpp:28,64
//
// Differences a caller will notice: uint128_t is the compiler's unsigned
// __int128 (the reference used the CUDA-uint128 class); a failing call prints
// the library's message and aborts (the reference checked no errors at all);
// results are exact (the reference's easy + hard split was off by ~1 ppm).
#pragma once
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstdint>
#include <vector>

#include "cpx.h"

typedef unsigned __int128 uint128_t;

namespace cudapix_compat {

inline cpx_ctx *ctx()
{
    static cpx_ctx *c = [] {
        cpx_ctx *h = nullptr;
        if (cpx_create(0, &h) != CPX_OK) {
            std::fprintf(stderr, "cudapix_b200: cannot create a context on device 0\n");
            std::abort();
        }
        return h;
    }();
    return c;
}

inline void ok(int rc)
{
    if (rc != CPX_OK) {
        std::fprintf(stderr, "cudapix_b200 error %d: %s\n", rc, cpx_last_error(ctx()));
        std::abort();
    }
}

inline cpx_u128 to(uint128_t v) { return cpx_u128{(uint64_t)v, (uint64_t)(v >> 64)}; }
inline uint128_t from(cpx_u128 v) { return ((uint128_t)v.hi << 64) | v.lo; }

}  // namespace cudapix_compat

inline uint64_t P2(uint64_t x, uint64_t y)
{
    uint64_t r;
    cudapix_compat::ok(cpx_P2_u64(cudapix_compat::ctx(), x, y, &r));
    return r;
}
inline uint128_t P2(uint128_t x, uint64_t y)
{
    cpx_u128 r;
    cudapix_compat::ok(cpx_P2_u128(cudapix_compat::ctx(), cudapix_compat::to(x), y, &r));
    return cudapix_compat::from(r);
}
inline uint64_t S2_trivial(uint64_t x, uint64_t y)
{
    uint64_t r;
    cudapix_compat::ok(cpx_trivial_u64(cudapix_compat::ctx(), x, y, &r));
    return r;
}
inline uint128_t S2_trivial(uint128_t x, uint64_t y)
{
    cpx_u128 r;
    cudapix_compat::ok(cpx_trivial_u128(cudapix_compat::ctx(), cudapix_compat::to(x), y, &r));
    return cudapix_compat::from(r);
}
inline uint64_t Ordinary(uint64_t x, uint64_t y, uint16_t c)
{
    int64_t r;
    cudapix_compat::ok(cpx_ordinary_u64(cudapix_compat::ctx(), x, y, c, &r));
    return (uint64_t)r;
}
inline uint128_t Ordinary(uint128_t x, uint64_t y, uint16_t c)
{
    cpx_u128 r;
    cudapix_compat::ok(cpx_ordinary_u128(cudapix_compat::ctx(), cudapix_compat::to(x), y, c, &r));
    return cudapix_compat::from(r);
}
inline int64_t mutest(uint64_t top)
{
    int64_t r;
    cudapix_compat::ok(cpx_mutest(cudapix_compat::ctx(), top, &r));
    return r;
}
inline uint32_t *get_d_piTable(uint32_t hi)
{
    uint32_t *p;
    cudapix_compat::ok(cpx_pitable(cudapix_compat::ctx(), hi, &p));
    return p;
}

template <typename T> T *gen_d_lpf(T bottom, T top);
template <> inline uint32_t *gen_d_lpf<uint32_t>(uint32_t bottom, uint32_t top)
{
    uint32_t *p;
    cudapix_compat::ok(cpx_gen_d_lpf32(cudapix_compat::ctx(), bottom, top, &p));
    return p;
}
template <> inline uint64_t *gen_d_lpf<uint64_t>(uint64_t bottom, uint64_t top)
{
    uint64_t *p;
    cudapix_compat::ok(cpx_gen_d_lpf64(cudapix_compat::ctx(), bottom, top, &p));
    return p;
}
template <typename T> inline int8_t *gen_d_mu(T bottom, T top)
{
    int8_t *p;
    cudapix_compat::ok(cpx_gen_d_mu(cudapix_compat::ctx(), bottom, top, &p));
    return p;
}
template <typename T> inline int8_t *gen_h_mu(T bottom, T top)
{
    int8_t *h = (int8_t *)std::malloc((size_t)(top - bottom) / 2 + 1);
    cudapix_compat::ok(cpx_gen_h_mu(cudapix_compat::ctx(), bottom, top, h));
    return h;
}
template <typename T> inline T *gen_h_lpf(T bottom, T top)
{
    const size_t n = (size_t)(top - bottom) / 2;
    T *h = (T *)std::malloc((n + 1) * sizeof(T));
    if (sizeof(T) == 4) {
        cudapix_compat::ok(cpx_gen_h_lpf32(cudapix_compat::ctx(), bottom, top, (uint32_t *)h));
    } else {
        uint64_t *d = gen_d_lpf<uint64_t>(bottom, top);
        cudapix_compat::ok(cpx_copy_to_host(h, d, n * 8));
        cpx_free(d);
    }
    return h;
}
inline void gen_d_mu_lpf(uint64_t bottom, uint64_t top, int8_t *d_mu, uint64_t *d_lpf)
{
    cudapix_compat::ok(cpx_gen_d_mu_lpf(cudapix_compat::ctx(), bottom, top, d_mu, d_lpf));
}

class PiTable {
    uint64_t base = 0, range = 0, bottom = 0, pi_base = 0;
    bool pi_current = false;  // pi_base belongs to the current base
    uint32_t *d_pitable = nullptr;

    void alloc()
    {
        if (d_pitable) cpx_free(d_pitable);
        void *p = nullptr;
        cudapix_compat::ok(cpx_device_alloc((range / 2 + 2) * 4, &p));
        d_pitable = (uint32_t *)p;
    }
    uint32_t *fill()
    {
        cudapix_compat::ok(cpx_pitable_window(cudapix_compat::ctx(), base, range, d_pitable, &pi_base));
        pi_current = true;
        return d_pitable;
    }

  public:
    PiTable() {}
    explicit PiTable(uint64_t range) : range(range) { alloc(); }
    PiTable(uint64_t base, uint64_t bottom, uint64_t range = 0) : base(base), bottom(bottom)
    {
        this->range = range ? range : std::min<uint64_t>(getMaxRange(), base - bottom);
        alloc();
    }
    ~PiTable()
    {
        if (d_pitable) cpx_free(d_pitable);
    }
    uint64_t get_base() { return base; }
    uint64_t get_range() { return range; }
    uint64_t get_bottom() { return bottom; }
    // pi(base - 1): counted on first use after the base changes (src/pitable.cu:154-166)
    uint64_t get_pi_base()
    {
        if (base == 0) return 0;
        if (!pi_current) {
            cudapix_compat::ok(cpx_count_primes(cudapix_compat::ctx(), 0, base, &pi_base));
            pi_current = true;
        }
        return pi_base;
    }
    // a caller's pi(base - 1), kept until the base changes (src/pitable.cu:175-179); the
    // next window fill replaces it by the exact count
    void set_pi_base(uint64_t v)
    {
        pi_base = v;
        pi_current = true;
    }
    void set_base(uint64_t b)
    {
        base = b;
        pi_current = false;
    }
    // unlike the reference (src/pitable.cu:181-186), the buffer follows the new range
    void set_range(uint64_t r)
    {
        range = r;
        alloc();
    }
    void set_bottom(uint64_t b) { bottom = b; }
    uint64_t getMaxRange()
    {
        uint64_t f = 0, t = 0;
        cudapix_compat::ok(cpx_mem_info(cudapix_compat::ctx(), &f, &t));
        return (uint64_t)(f / 2.5);
    }
    // src/pitable.cu:56-75: allocate() keeps an existing buffer, reallocate() replaces it;
    // the contents are written by the next getCurrent / getNextUp / getNextDown
    void allocate()
    {
        if (!d_pitable) alloc();
    }
    void reallocate() { alloc(); }
    uint64_t setMaxRange()
    {
        range = getMaxRange();
        reallocate();
        return range;
    }
    uint32_t *getCurrent() { return fill(); }
    uint32_t *getNextUp()
    {
        base += range;
        return fill();
    }
    uint32_t *getNextDown()
    {
        if ((int64_t)bottom < (int64_t)base - (int64_t)range) base -= range;
        else {
            range = base - bottom;
            base = bottom;
        }
        return fill();
    }
    uint64_t getNextBaseUp() { return base + range; }
    uint64_t getNextBaseDown() { return std::max<int64_t>((int64_t)bottom, (int64_t)(base - range)); }
};

// phi(x, a) with the reference's prime index: a selects p = smallPrimes[a]
// (0-based: a = 0 -> 2), i.e. the first a + 1 primes are excluded.
class Phi {
    uint32_t max_, p_max_;
    uint32_t *d_lpf = nullptr, *d_primeList = nullptr, *h_primeList = nullptr, primeListLength = 0;

    static uint32_t isqrt32(uint32_t m)
    {
        uint64_t r = (uint64_t)std::sqrt((double)m);
        while (r * r > m) r--;
        while ((r + 1) * (r + 1) <= m) r++;
        return (uint32_t)r;
    }
    // the sieving primes after the 12 small primes 2 .. 37, up to p_max
    // (PrimeList::getSievingPrimes in src/phi.cu:20,30), built on first use
    void primes()
    {
        if (h_primeList) return;
        uint64_t *d = nullptr, n = 0;
        cudapix_compat::ok(cpx_primes(cudapix_compat::ctx(), 41, (uint64_t)p_max_ + 1, &d, &n));
        std::vector<uint64_t> h(n);
        if (n) cudapix_compat::ok(cpx_copy_to_host(h.data(), d, n * 8));
        cpx_free(d);
        h_primeList = (uint32_t *)std::malloc((n ? n : 1) * 4);
        for (uint64_t i = 0; i < n; i++) h_primeList[i] = (uint32_t)h[i];
        void *p = nullptr;
        cudapix_compat::ok(cpx_device_alloc((n ? n : 1) * 4, &p));
        d_primeList = (uint32_t *)p;
        if (n) cudapix_compat::ok(cpx_copy_to_device(d_primeList, h_primeList, n * 4));
        primeListLength = (uint32_t)n;
    }

  public:
    explicit Phi(uint32_t max) : max_(max), p_max_(isqrt32(max)) {}
    Phi(uint32_t max, uint32_t p_max) : max_(max), p_max_(p_max) {}
    ~Phi()
    {
        if (d_lpf) cpx_free(d_lpf);
        if (d_primeList) cpx_free(d_primeList);
        std::free(h_primeList);
    }
    Phi(const Phi &) = delete;
    Phi &operator=(const Phi &) = delete;

    // lpf of the odd n in [0, max) (src/phi.cu:16), built on first use; owned by the Phi
    uint32_t *get_d_lpf()
    {
        if (!d_lpf) d_lpf = gen_d_lpf<uint32_t>(0u, max_);
        return d_lpf;
    }
    uint32_t *get_d_primeList()
    {
        primes();
        return d_primeList;
    }
    uint32_t *get_h_primeList()
    {
        primes();
        return h_primeList;
    }
    uint32_t get_primeListLength()
    {
        primes();
        return primeListLength;
    }
    // The reference fills a private cache that phi() never reads (src/phi.cu:58-73);
    // phi() here is exact without it, so there is nothing to build.
    void makeModCache(uint32_t) {}

    uint64_t phi(uint32_t x, uint32_t a)
    {
        uint64_t r;
        cudapix_compat::ok(cpx_phi(cudapix_compat::ctx(), x, a + 1, &r));
        return r;
    }
    uint32_t *generateRange(uint32_t num, uint32_t a)
    {
        uint32_t *p;
        cudapix_compat::ok(cpx_phi_range(cudapix_compat::ctx(), num, a + 1, &p));
        return p;
    }
};

class Phisieve {
    cpx_phisieve *ps = nullptr;
    uint32_t bits;

  public:
    explicit Phisieve(uint32_t maxPrime, uint32_t blockSize = 1u << 28) : bits(blockSize)
    {
        cudapix_compat::ok(cpx_phisieve_create(cudapix_compat::ctx(), maxPrime, blockSize, &ps));
    }
    ~Phisieve() { cpx_phisieve_destroy(ps); }
    void firstSieve(uint16_t c) { cudapix_compat::ok(cpx_phisieve_first(ps, c)); }
    void markNext() { cudapix_compat::ok(cpx_phisieve_mark_next(ps)); }
    void updateCount() { cudapix_compat::ok(cpx_phisieve_update(ps)); }
    uint32_t *getCountDevice()
    {
        uint32_t *d;
        uint32_t a;
        cudapix_compat::ok(cpx_phisieve_counts(ps, &d, &a));
        return d;
    }
    uint32_t *getCountHost()
    {
        uint32_t *h = (uint32_t *)std::malloc((size_t)bits * 4);
        cudapix_compat::ok(cpx_copy_to_host(h, getCountDevice(), (size_t)bits * 4));
        return h;
    }
    uint32_t get_a_current()
    {
        uint32_t a;
        cudapix_compat::ok(cpx_phisieve_counts(ps, nullptr, &a));
        return a;
    }
    void set_a_current(uint32_t a) { cudapix_compat::ok(cpx_phisieve_set_a(ps, a)); }
};

// The hard leaves of this library's exact split (x/(p_b m) >= p_b^2, so
// p_b <= x^(1/4)); with S2_easy and the trivial leaves they give the
// reference's S2 + S3 exactly (its own split between the two is off by ~1 ppm).
struct S2hardHost {
    static uint64_t S2hard(uint64_t x, uint64_t y, uint16_t c)
    {
        int64_t r;
        cudapix_compat::ok(cpx_S2_hard_u64(cudapix_compat::ctx(), x, y, c, &r));
        return (uint64_t)r;
    }
    // maxPrime caps the sieving primes (include/sieve/S2_hard_host.cuh:36).  Hard
    // leaves stop at x^(1/4), so any maxPrime >= x^(1/4) (the reference's one call
    // with it, src/Gourdon/gourdonvariant.cpp:61, passes x^(1/4)) gives all of them;
    // a smaller cap is refused.
    static uint64_t S2hard(uint64_t x, uint64_t y, uint16_t c, uint64_t maxPrime)
    {
        uint64_t sx, cx, qx;
        cudapix_compat::ok(cpx_iroots(cpx_u128{x, 0}, &sx, &cx, &qx));
        if (maxPrime < qx) {
            std::fprintf(stderr, "cudapix_b200: S2hard with maxPrime below x^(1/4) is not supported\n");
            std::abort();
        }
        return S2hard(x, y, c);
    }
};

struct deleglise_rivat64 {
    static uint64_t pi_deleglise_rivat(uint64_t x, uint64_t y, uint16_t c)
    {
        uint64_t r;
        cudapix_compat::ok(cpx_pi_u64(cudapix_compat::ctx(), x, y, c, &r, nullptr));
        return r;
    }
};

struct deleglise_rivat128 {
    static uint128_t pi_deleglise_rivat(uint128_t x, uint64_t y, uint16_t c)
    {
        cpx_u128 r;
        cudapix_compat::ok(cpx_pi_u128(cudapix_compat::ctx(), cudapix_compat::to(x), y, c, &r, nullptr));
        return cudapix_compat::from(r);
    }
};

// Gourdon's decomposition (include/Gourdon/gourdonvariant.hpp:7-56): the
// terms are computed once, on construction; pi() = A - B + C + D + phi_0 + sigma
// with D = S2hardHost::S2hard(x, y, c, x^(1/4)) (gourdonvariant.cpp:61).
class GourdonVariant64 {
    cpx_gourdon_terms t_;
    static int64_t s64(cpx_u128 v) { return (int64_t)v.lo; }

  public:
    GourdonVariant64(uint64_t x, uint64_t y, uint16_t c)
    {
        cudapix_compat::ok(cpx_gourdon_u64(cudapix_compat::ctx(), x, y, c, &t_));
    }
    static uint64_t piGourdon(uint64_t x, uint64_t y, uint16_t c) { return GourdonVariant64(x, y, c).pi(); }
    uint64_t pi() { return t_.pi.lo; }
    uint64_t A() { return t_.A.lo; }
    uint64_t B() { return t_.B.lo; }
    uint64_t C() { return t_.C.lo; }
    uint64_t D() { return (uint64_t)s64(t_.D); }
    int64_t sigma() { return s64(t_.sigma); }
    uint64_t phi_0() { return (uint64_t)s64(t_.phi0); }
};
