// terms.cu -- the Deleglise-Rivat term kernels over a batch of queries.
//
// Each kernel walks a flattened index space of "units" over all queries of a
// batch (prefix arrays built on the host), so one launch serves one query or
// thousands.  Sums are exact: 64-bit per thread, 128-bit per query.
//
// Reference functions restated (file:line in curtisseizert/CUDApix):
//   P2 (64/128-bit)        src/P2.cu:18-70, 99-156
//   S2_trivial             src/trivial.cu:31-95
//   Ordinary, ordinaryKernel(Iter)   src/ordinary.cu:23-135
//   easy leaves (S2, sigma)          src/Deleglise-Rivat/S2.cu:30-118, sigma.cu:25-214
//   hard leaves (S2hardHost, S2ctl)  src/sieve/S2_hard_host.cu:49-191,
//                                    src/sieve/S2_hard_device.cu:12-382
// The easy/hard split here is this library's own exact one; the reference's
// split is off by ~1 ppm (README.md:3,8).
#include "terms.cuh"

namespace cpx {

constexpr unsigned FULL = 0xffffffffu;
__constant__ uint32_t c_pc[9] = {1, 2, 3, 5, 7, 11, 13, 17, 19};  // p_c for c = 0..8

__device__ __forceinline__ uint32_t find_q(const uint64_t *__restrict__ pre, uint32_t Q, uint64_t u)
{
    uint32_t lo = 0, hi = Q;  // pre[lo] <= u < pre[hi]
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (__ldg(pre + mid) <= u) lo = mid;
        else hi = mid;
    }
    return lo;
}

// bits j of table entry w with a < 128w + 2j + 1 <= b
__device__ __forceinline__ uint64_t range_mask(uint64_t w, uint64_t a, uint64_t b)
{
    const uint64_t base = 128 * w;
    if (b < base + 1) return 0;
    uint64_t hiJ = (b - base - 1) >> 1;
    if (hiJ > 63) hiJ = 63;
    const uint64_t loJ = (a >= base) ? ((a - base + 1) >> 1) : 0;
    if (loJ > hiJ) return 0;
    const uint64_t upto = (hiJ == 63) ? ~0ull : ((2ull << hiJ) - 1);
    return upto & ~((1ull << loJ) - 1);
}

struct LaneAcc {
    uint32_t q = 0xFFFFFFFFu;
    i128 v = 0;
};

__device__ __forceinline__ void acc_add(unsigned long long *acc, uint32_t q, int term, i128 v)
{
    if (q != 0xFFFFFFFFu && v != 0) cpx_atomic_add_i128(acc + (uint64_t)q * kAccStride + 2 * term, v);
}

__device__ __forceinline__ void lane_switch(LaneAcc &a, uint32_t q, unsigned long long *acc, int term)
{
    if (q != a.q) {
        acc_add(acc, a.q, term, a.v);
        a.q = q;
        a.v = 0;
    }
}

// all 32 lanes must call
__device__ __forceinline__ void warp_flush(LaneAcc &a, unsigned long long *acc, int term)
{
    const uint32_t q0 = __shfl_sync(FULL, a.q, 0);
    if (__all_sync(FULL, a.q == q0)) {
        const i128 s = cpx_warp_sum_i128(a.v);
        if ((threadIdx.x & 31) == 0) acc_add(acc, q0, term, s);
    } else {
        acc_add(acc, a.q, term, a.v);
    }
    a.v = 0;
}

// Warp-contiguous partition of [0, total): each warp owns a slice and walks it
// 32 units at a time (coalesced, and queries change rarely inside a slice).
struct WarpSlice {
    uint64_t u0, u1;
};
__device__ __forceinline__ WarpSlice warp_slice(uint64_t total)
{
    const uint64_t gw = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    const uint64_t per = (total + nw - 1) / nw;
    uint64_t u0 = gw * per, u1 = u0 + per;
    if (u0 > total) u0 = total;
    if (u1 > total) u1 = total;
    return {u0, u1};
}

// cached query lookup per lane
struct QCache {
    uint32_t q = 0xFFFFFFFFu;
    uint64_t lo = 1, hi = 0;  // [lo, hi) unit range of q
};
__device__ __forceinline__ uint32_t qlookup(QCache &c, const uint64_t *pre, uint32_t Q, uint64_t u)
{
    if (u >= c.lo && u < c.hi) return c.q;
    c.q = find_q(pre, Q, u);
    c.lo = __ldg(pre + c.q);
    c.hi = __ldg(pre + c.q + 1);
    return c.q;
}

template <class XT> __device__ __forceinline__ XT xload(const QD &d) { return (XT)d.x; }

// ------------------------------------------------------------------ ordinary
// S0 = sum_{odd n <= y, lpf(n) > p_c} mu(n) phi(x/n, c);
// phi(m, c) = floor(m / W) phi(W) + WH[((m mod W) + 1) / 2], W = p_c#.
template <int C> struct Wheel;
template <> struct Wheel<1> { static constexpr uint64_t W = 2, TOT = 1; static constexpr int32_t PC = 2; };
template <> struct Wheel<2> { static constexpr uint64_t W = 6, TOT = 2; static constexpr int32_t PC = 3; };
template <> struct Wheel<3> { static constexpr uint64_t W = 30, TOT = 8; static constexpr int32_t PC = 5; };
template <> struct Wheel<4> { static constexpr uint64_t W = 210, TOT = 48; static constexpr int32_t PC = 7; };
template <> struct Wheel<5> { static constexpr uint64_t W = 2310, TOT = 480; static constexpr int32_t PC = 11; };
template <> struct Wheel<6> { static constexpr uint64_t W = 30030, TOT = 5760; static constexpr int32_t PC = 13; };
template <> struct Wheel<7> { static constexpr uint64_t W = 510510, TOT = 92160; static constexpr int32_t PC = 17; };
template <> struct Wheel<8> { static constexpr uint64_t W = 9699690, TOT = 1658880; static constexpr int32_t PC = 19; };

template <int C, class XT>
__global__ void __launch_bounds__(kThreads) k_ordinary(const QD *__restrict__ qd, uint32_t Q,
                                                       const uint64_t *__restrict__ pre, uint64_t total,
                                                       const int32_t *__restrict__ MU,
                                                       const uint32_t *__restrict__ WH,
                                                       unsigned long long *__restrict__ acc)
{
    using Wh = Wheel<C>;
    const WarpSlice sl = warp_slice(total);
    const int lane = threadIdx.x & 31;
    LaneAcc a;
    QCache qc;
    XT x = 0;
    uint64_t y = 0;
    for (uint64_t base = sl.u0; base < sl.u1; base += 32) {
        const uint64_t u = base + lane;
        if (u < sl.u1) {
            const uint32_t q = qlookup(qc, pre, Q, u);
            if (q != a.q) {
                lane_switch(a, q, acc, ACC_ORD);
                x = xload<XT>(qd[q]);
                y = qd[q].y;
            }
            const uint64_t local = u - qc.lo;
            const int4 v4 = __ldg(reinterpret_cast<const int4 *>(MU) + local);
            const int32_t vals[4] = {v4.x, v4.y, v4.z, v4.w};
#pragma unroll
            for (int k = 0; k < 4; k++) {
                const uint64_t n = 2 * (4 * local + k) + 1;
                const int32_t v = vals[k];
                if (n > y || v == 0) continue;
                if ((v > 0 ? v : -v) <= Wh::PC) continue;
                const XT m = x / (XT)n;
                const XT qw = m / (XT)Wh::W;
                const uint32_t r = (uint32_t)(m - qw * (XT)Wh::W);
                const i128 ph = (i128)qw * (i128)Wh::TOT + (i128)__ldg(WH + ((r + 1) >> 1));
                a.v += (v > 0) ? ph : -ph;
            }
        }
    }
    warp_flush(a, acc, ACC_ORD);
}

// ------------------------------------------------------------------------ P2
// P2 = sum_{y < p <= sqrt x} [pi(x/p) - pi(p) + 1]; one table entry per unit.
template <class XT>
__global__ void __launch_bounds__(kThreads) k_p2(const QD *__restrict__ qd, uint32_t Q,
                                                 const uint64_t *__restrict__ pre, uint64_t total,
                                                 const cpx_pient *__restrict__ T,
                                                 unsigned long long *__restrict__ acc)
{
    const WarpSlice sl = warp_slice(total);
    const int lane = threadIdx.x & 31;
    LaneAcc a;
    QCache qc;
    XT x = 0;
    uint64_t y = 0, sx = 0;
    for (uint64_t base = sl.u0; base < sl.u1; base += 32) {
        const uint64_t u = base + lane;
        if (u < sl.u1) {
            const uint32_t q = qlookup(qc, pre, Q, u);
            if (q != a.q) {
                lane_switch(a, q, acc, ACC_P2);
                x = xload<XT>(qd[q]);
                y = qd[q].y;
                sx = qd[q].sx;
            }
            const uint64_t w = (y >> 7) + (u - qc.lo);
            const ulonglong2 e = __ldg(reinterpret_cast<const ulonglong2 *>(T) + w);
            uint64_t bits = e.x & range_mask(w, y, sx);
            int64_t s = 0;
            while (bits) {
                const int j = __ffsll((long long)bits) - 1;
                bits &= bits - 1;
                const uint64_t p = 128 * w + 2 * j + 1;
                const uint64_t i = 1 + e.y + __popcll(e.x & ((2ull << j) - 1));  // pi(p)
                const uint64_t xp = (uint64_t)(x / (XT)p);
                s += (int64_t)cpx_pi_dev(T, xp) - (int64_t)i + 1;
            }
            a.v += s;
        }
    }
    warp_flush(a, acc, ACC_P2);
}

// ------------------------------------------------------------------- trivial
// S1 = C(pi(y) - pi(cbrt x), 2);  U = sum_{isqrt(x/y) < p <= cbrt x} [pi(y) - pi(x/p^2)]
template <class XT>
__global__ void __launch_bounds__(kThreads) k_trivial(const QD *__restrict__ qd, uint32_t Q,
                                                      const uint64_t *__restrict__ pre, uint64_t total,
                                                      const cpx_pient *__restrict__ T,
                                                      unsigned long long *__restrict__ acc)
{
    const WarpSlice sl = warp_slice(total);
    const int lane = threadIdx.x & 31;
    LaneAcc a;
    QCache qc;
    XT x = 0;
    uint64_t y = 0, tx = 0, cx = 0, piy = 0;
    for (uint64_t base = sl.u0; base < sl.u1; base += 32) {
        const uint64_t u = base + lane;
        if (u < sl.u1) {
            const uint32_t q = qlookup(qc, pre, Q, u);
            if (q != a.q) {
                lane_switch(a, q, acc, ACC_TRIV);
                x = xload<XT>(qd[q]);
                y = qd[q].y;
                tx = qd[q].tx;
                cx = qd[q].cx;
                piy = cpx_pi_dev(T, y);
            }
            const uint64_t local = u - qc.lo;
            i128 s = 0;
            if (local == 0) {
                const uint64_t pic = cpx_pi_dev(T, cx);
                if (piy > pic) s += (i128)(piy - pic) * (i128)(piy - pic - 1) / 2;
            }
            if (cx > tx) {
                const uint64_t w = (tx >> 7) + local;
                const ulonglong2 e = __ldg(reinterpret_cast<const ulonglong2 *>(T) + w);
                uint64_t bits = e.x & range_mask(w, tx, cx);
                while (bits) {
                    const int j = __ffsll((long long)bits) - 1;
                    bits &= bits - 1;
                    const uint64_t p = 128 * w + 2 * j + 1;
                    const uint64_t v = (uint64_t)(x / ((XT)p * (XT)p));
                    s += (i128)piy - (i128)cpx_pi_dev(T, v);
                }
            }
            a.v += s;
        }
    }
    warp_flush(a, acc, ACC_TRIV);
}

// ---------------------------------------------------------------------- easy
// Easy leaves are the non-trivial leaves with u = x/(p_b m) < p_b^2, where
// phi(u, b - 1) = pi(u) - b + 2 is one pi-table lookup.  k_easy takes the
// prime m = q: p_c < p <= icbrt(x), max(p, y/p, x/p^3) < q <= min(y, x/p^2)
// (for p > iroot4(x) the bound x/p^3 is below p).  A warp takes one table
// entry of p candidates at a time (ticket counter); its lanes stride over the
// table entries of the q range.  k_easy_comp takes the composite m.
template <class XT>
__global__ void __launch_bounds__(kThreads) k_easy(const QD *__restrict__ qd, uint32_t Q,
                                                   const uint64_t *__restrict__ pre, uint64_t total,
                                                   const cpx_pient *__restrict__ T,
                                                   unsigned int *__restrict__ ticket,
                                                   unsigned long long *__restrict__ acc)
{
    const int lane = threadIdx.x & 31;
    for (;;) {
        uint64_t unit = 0;
        if (lane == 0) unit = atomicAdd(ticket, 1u);
        unit = __shfl_sync(FULL, unit, 0);
        if (unit >= total) break;
        const uint32_t q = find_q(pre, Q, unit);
        const QD &d = qd[q];
        const XT x = xload<XT>(d);
        const uint64_t y = d.y, pc = c_pc[d.c], cx = d.cx;
        const uint64_t w = (pc >> 7) + (unit - __ldg(pre + q));
        const ulonglong2 e = __ldg(reinterpret_cast<const ulonglong2 *>(T) + w);
        uint64_t pb = e.x & range_mask(w, pc, cx);
        i128 s = 0;
        while (pb) {
            const int j = __ffsll((long long)pb) - 1;
            pb &= pb - 1;
            const uint64_t p = 128 * w + 2 * j + 1;
            const uint64_t b = 1 + e.y + __popcll(e.x & ((2ull << j) - 1));
            const XT xp = x / (XT)p;
            uint64_t qlo = y / p;
            if (qlo < p) qlo = p;
            const XT xpp = xp / (XT)p;
            {
                // p <= iroot4(x): only q > x/p^3 (x/(pq) < p^2) are easy
                const XT x3 = xpp / (XT)p;
                if (x3 > (XT)qlo) qlo = (x3 >= (XT)y) ? y : (uint64_t)x3;
            }
            const uint64_t qhi = (xpp < (XT)y) ? (uint64_t)xpp : y;
            if (qhi <= qlo) continue;
            const uint64_t wq0 = qlo >> 7, wq1 = (qhi - 1) >> 7;
            uint64_t ps = 0, cnt = 0;
            for (uint64_t wq = wq0 + lane; wq <= wq1; wq += 32) {
                const ulonglong2 e2 = __ldg(reinterpret_cast<const ulonglong2 *>(T) + wq);
                uint64_t qb = e2.x & range_mask(wq, qlo, qhi);
                while (qb) {
                    const int j2 = __ffsll((long long)qb) - 1;
                    qb &= qb - 1;
                    const uint64_t qq = 128 * wq + 2 * j2 + 1;
                    const uint64_t uu = (uint64_t)(xp / (XT)qq);
                    ps += cpx_pi_dev(T, uu);
                    cnt++;
                }
            }
            s += (i128)ps + (i128)cnt * (2 - (i128)b);
        }
        const i128 ws = cpx_warp_sum_i128(s);
        if (lane == 0) acc_add(acc, q, ACC_EASY, ws);
    }
}

// Composite easy leaves: p_b <= min(iroot4(x), sqrt y), m composite with
// lpf(m) > p_b, mu(m) != 0, max(y/p_b, x/p_b^3) < m <= y; value
// -mu(m) (pi(x/(p_b m)) - b + 2).  Work = (level record, chunk of 1024 odd m);
// a warp walks its chunk 128 m at a time, one 16-byte load of packed mu*lpf per lane.
template <class XT>
__global__ void __launch_bounds__(kThreads) k_easy_comp(const QD *__restrict__ qd, const EasyLvl *__restrict__ lv,
                                                        uint32_t nlv, uint64_t total,
                                                        const int32_t *__restrict__ MU,
                                                        const cpx_pient *__restrict__ T,
                                                        unsigned long long *__restrict__ acc)
{
    const int lane = threadIdx.x & 31;
    const uint64_t gw = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t unit = gw; unit < total; unit += nw) {
        uint32_t lo = 0, hi = nlv;  // lv[lo].unit0 <= unit < lv[hi].unit0
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (lv[mid].unit0 <= unit) lo = mid;
            else hi = mid;
        }
        const EasyLvl r = lv[lo];
        const QD &d = qd[r.q];
        const XT xp = xload<XT>(d) / (XT)r.p;
        const uint64_t base = r.i_base + (unit - r.unit0) * 1024;  // multiple of 4
        int64_t s = 0;
        for (int it = 0; it < 8; it++) {
            const uint64_t i0 = base + 128 * it + 4 * lane;
            if (i0 >= r.i_hi) break;
            const int4 v4 = __ldg(reinterpret_cast<const int4 *>(MU) + (i0 >> 2));
            const int32_t vals[4] = {v4.x, v4.y, v4.z, v4.w};
#pragma unroll
            for (int k = 0; k < 4; k++) {
                const uint64_t i = i0 + k;
                if (i < r.i_lo || i >= r.i_hi) continue;
                const int32_t v = vals[k];
                const uint64_t m = 2 * i + 1;
                const uint32_t av = (uint32_t)(v > 0 ? v : -v);
                if (v == 0 || av <= r.p || (uint64_t)av >= m) continue;  // mu = 0, lpf <= p, or m prime
                const uint64_t uu = (uint64_t)(xp / (XT)m);
                const int64_t val = (int64_t)cpx_pi_dev(T, uu) - (int64_t)r.b + 2;
                s += (v > 0) ? -val : val;
            }
        }
        LaneAcc a;
        a.q = r.q;
        a.v = s;
        warp_flush(a, acc, ACC_EASY);
    }
}

// ---------------------------------------------------------------------- hard
// Segmented phi sieve.  One CTA owns one segment of 2^lbits odd numbers
// n = lo + 2i + 1 of one query, held as a bitmap in shared memory.  For each
// b = c+1 .. B(seg) it (1) writes the segment's count at level b-1, (2) if
// the segment holds leaves of p_b, builds per-thread/per-chunk popcount
// prefixes and answers every leaf phi(x/(p_b m), b-1) - carry as
// prefix + popcount(word & mask), (3) crosses off p_b, counting the bits it
// clears.  Carries between segments are added by k_hard_combine.
//
// Bitmap layout: 16-byte chunks of 4 words; thread t owns chunks
// [CPT*t, CPT*(t+1)).  Chunk c is stored at c ^ ((c >> log2 CPT) & 7) so that
// the owners' 128-bit loads and stores are free of bank conflicts.

__device__ __forceinline__ uint32_t swz(uint32_t c, int s) { return s ? (c ^ ((c >> s) & 7u)) : c; }

// bits k < 32 of a word whose first number is = r (mod p) that are multiples of p
__device__ __forceinline__ uint32_t mult_mask(uint32_t r, uint32_t p, uint32_t Mp)
{
    const uint32_t k0 = (r == 0) ? 0u : ((r & 1u) ? (p - r) >> 1 : p - (r >> 1));
    return k0 < 32 ? (Mp << k0) : 0u;
}
__device__ __forceinline__ uint32_t every_pth_bit(uint32_t p)
{
    uint32_t m = 0;
    for (uint32_t k = 0; k < 32; k += p) m |= 1u << k;
    return m;
}

template <class XT> struct HardSmem {
    // offsets into the dynamic shared memory block
    static __host__ __device__ size_t bytes(uint32_t lbits, uint32_t threads)
    {
        const size_t L = size_t(1) << lbits;
        size_t o = L / 8;               // bitmap
        o += (L / 128) * 2;             // chunk prefixes (u16)
        o = (o + 15) & ~size_t(15);
        o += threads * 4;               // toff
        o += 32 * 4;                    // wsum
        o += threads * (4 * 5);         // s_p, s_mlo, s_mhi, s_i0, s_r0
        o = (o + 15) & ~size_t(15);
        o += threads * sizeof(XT);      // s_xp
        o += 64;                        // s_clr[2], s_ms
        o = (o + 15) & ~size_t(15);
        o += 32 * sizeof(i128);         // reductions
        return o;
    }
};

template <class XT>
__global__ void __launch_bounds__(512) k_hard(const QD *__restrict__ qd, uint32_t Q,
                                              const uint64_t *__restrict__ pre_seg, uint64_t total,
                                              const uint32_t *__restrict__ seg_B,
                                              const uint64_t *__restrict__ seg_off,
                                              const uint32_t *__restrict__ P, const int32_t *__restrict__ MU,
                                              const cpx_pient *__restrict__ Tpi,
                                              uint32_t *__restrict__ out_cnt, int32_t *__restrict__ out_ms,
                                              uint64_t cap, unsigned long long *__restrict__ acc,
                                              uint32_t lbits_max)
{
    extern __shared__ uint4 smem4[];
    const uint64_t unit = blockIdx.x;
    if (unit >= total) return;
    const uint32_t B = seg_B[unit];
    const uint32_t q = find_q(pre_seg, Q, unit);
    const QD &d = qd[q];
    const uint32_t c = d.c;
    if (B <= c) return;  // uniform over the CTA
    const uint32_t T = blockDim.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t lbits = d.lbits;
    const uint32_t L = 1u << lbits;
    const uint32_t NC = L >> 7;       // chunks
    const uint32_t CPT = NC / T;      // chunks per thread (>= 1)
    const int s = __ffs(CPT) - 1;     // log2 CPT
    const uint64_t seg = unit - pre_seg[q];
    const uint64_t lo = seg * 2 * (uint64_t)L, hi = lo + 2 * (uint64_t)L;
    const uint64_t off = seg_off[unit];
    if (off + (B - c) > cap) return;  // the host sized the ragged outputs exactly; never write past them
    const XT x = xload<XT>(d);
    const uint64_t y = d.y;

    // carve the shared block (sized for lbits_max)
    unsigned char *sp = reinterpret_cast<unsigned char *>(smem4);
    const size_t Lmax = size_t(1) << lbits_max;
    uint32_t *bm = reinterpret_cast<uint32_t *>(sp);
    size_t o = Lmax / 8;
    uint16_t *cp16 = reinterpret_cast<uint16_t *>(sp + o);
    o += (Lmax / 128) * 2;
    o = (o + 15) & ~size_t(15);
    uint32_t *toff = reinterpret_cast<uint32_t *>(sp + o);
    o += T * 4;
    uint32_t *wsum = reinterpret_cast<uint32_t *>(sp + o);
    o += 32 * 4;
    uint32_t *s_p = reinterpret_cast<uint32_t *>(sp + o);
    uint32_t *s_mlo = s_p + T, *s_mhi = s_mlo + T, *s_i0 = s_mhi + T, *s_r0 = s_i0 + T;
    o += T * 20;
    o = (o + 15) & ~size_t(15);
    XT *s_xp = reinterpret_cast<XT *>(sp + o);
    o += T * sizeof(XT);
    int *s_clr = reinterpret_cast<int *>(sp + o);
    int *s_ms = s_clr + 2;
    o += 64;
    o = (o + 15) & ~size_t(15);
    i128 *s_red = reinterpret_cast<i128 *>(sp + o);

    const uint32_t c0 = CPT * tid;   // first owned chunk
    const uint32_t w0 = 4 * c0;      // first owned word
    // ---- pre-sieve with p_2 .. p_c
    uint32_t cnt0 = 0;
    {
        uint32_t pr[8], rr[8], st[8], Mp[8];
        const uint32_t np = c - 1;
        for (uint32_t i = 0; i < np; i++) {
            pr[i] = P[i + 1];
            rr[i] = (uint32_t)(((lo + 1) % pr[i] + (64ull * w0) % pr[i]) % pr[i]);
            st[i] = 64u % pr[i];
            Mp[i] = every_pth_bit(pr[i]);
        }
        for (uint32_t j = 0; j < CPT; j++) {
            uint32_t wv[4];
#pragma unroll
            for (int k = 0; k < 4; k++) {
                uint32_t m = 0;
                for (uint32_t i = 0; i < np; i++) {
                    m |= mult_mask(rr[i], pr[i], Mp[i]);
                    rr[i] += st[i];
                    if (rr[i] >= pr[i]) rr[i] -= pr[i];
                }
                wv[k] = ~m;
                cnt0 += __popc(wv[k]);
            }
            reinterpret_cast<uint4 *>(bm)[swz(c0 + j, s)] = make_uint4(wv[0], wv[1], wv[2], wv[3]);
        }
    }
    if (tid == 0) {
        s_clr[0] = s_clr[1] = 0;
        *s_ms = 0;
    }
    // block sum of cnt0 -> thread 0
    uint32_t tot = 0;
    {
        uint32_t v = cnt0;
#pragma unroll
        for (int dd = 16; dd > 0; dd >>= 1) v += __shfl_down_sync(FULL, v, dd);
        if (lane == 0) wsum[warp] = v;
        __syncthreads();
        if (tid == 0) {
            for (uint32_t k = 0; k < T / 32; k++) tot += wsum[k];
        }
        __syncthreads();
    }

    int64_t S = 0;
    for (uint32_t bb = c + 1; bb <= B; bb += T) {
        const uint32_t nbat = min(T, B - bb + 1);
        if (tid < nbat) {
            const uint32_t b = bb + tid;
            const uint64_t p = P[b - 1];
            const XT xp = x / (XT)p;
            uint64_t mlo = y / p;
            const XT t1 = xp / (XT)hi;
            if (t1 > (XT)mlo) mlo = (uint64_t)t1;
            uint64_t mhi = y;
            if (lo) {
                const XT t2 = xp / (XT)lo;
                if (t2 < (XT)mhi) mhi = (uint64_t)t2;
            }
            {
                // hard leaves only: x/(p m) >= p^2, i.e. m <= x/p^3
                const XT t3 = xp / (XT)(p * p);
                if (t3 < (XT)mhi) mhi = (uint64_t)t3;
            }
            if (mhi < mlo) mhi = mlo;
            s_p[tid] = (uint32_t)p;
            s_xp[tid] = xp;
            s_mlo[tid] = (uint32_t)mlo;
            s_mhi[tid] = (uint32_t)mhi;
            const uint64_t r0 = (lo + 1) % p;
            s_r0[tid] = (uint32_t)r0;
            uint64_t m = lo + 1 + (r0 ? p - r0 : 0);
            if ((m & 1) == 0) m += p;
            s_i0[tid] = (m < hi) ? (uint32_t)((m - lo - 1) >> 1) : 0xFFFFFFFFu;
        }
        __syncthreads();
        for (uint32_t k = 0; k < nbat; k++) {
            const uint32_t b = bb + k;
            const uint32_t p = s_p[k];
            const uint32_t mlo = s_mlo[k], mhi = s_mhi[k];
            const uint64_t slot = off + (b - c - 1);
            if (tid == 0) {
                tot -= (uint32_t)s_clr[(b - 1) & 1];
                s_clr[(b - 1) & 1] = 0;
                out_cnt[slot] = tot;
            }
            if (mhi > mlo) {
                // per-chunk and per-thread popcount prefixes
                uint32_t run = 0;
                for (uint32_t j = 0; j < CPT; j++) {
                    const uint4 v = reinterpret_cast<const uint4 *>(bm)[swz(c0 + j, s)];
                    cp16[c0 + j] = (uint16_t)run;
                    run += __popc(v.x) + __popc(v.y) + __popc(v.z) + __popc(v.w);
                }
                uint32_t inc = run;
#pragma unroll
                for (int oo = 1; oo < 32; oo <<= 1) {
                    const uint32_t t = __shfl_up_sync(FULL, inc, oo);
                    if (lane >= (uint32_t)oo) inc += t;
                }
                toff[tid] = inc - run;
                if (lane == 31) wsum[warp] = inc;
                __syncthreads();
                const XT xp = s_xp[k];
                int32_t msl = 0;
                // survivors of the segment with n <= uu: per-thread, per-chunk
                // prefixes plus a popcount inside the 16-byte chunk
                auto seg_count = [&](uint64_t uu) -> uint32_t {
                    const uint32_t kk = (uint32_t)((uu - lo + 1) >> 1);  // bits [0, kk)
                    if (!kk) return 0u;
                    const uint32_t jb = kk - 1, w = jb >> 5, ch = w >> 2, ow = ch >> s;
                    uint32_t cv = toff[ow] + cp16[ch];
                    for (uint32_t i = 0; i < (ow >> 5); i++) cv += wsum[i];
                    const uint4 v4 = reinterpret_cast<const uint4 *>(bm)[swz(ch, s)];
                    const uint32_t wi = w & 3, msk = (2u << (jb & 31)) - 1u;
                    if (wi == 0) cv += __popc(v4.x & msk);
                    else if (wi == 1) cv += __popc(v4.x) + __popc(v4.y & msk);
                    else if (wi == 2) cv += __popc(v4.x) + __popc(v4.y) + __popc(v4.z & msk);
                    else cv += __popc(v4.x) + __popc(v4.y) + __popc(v4.z) + __popc(v4.w & msk);
                    return cv;
                };
                if ((uint64_t)p * p > y) {
                    // m must be a prime q > p: walk the pi-table bitmap of (max(mlo, p), mhi]
                    const uint64_t qa = mlo > p ? mlo : p;
                    if (mhi > qa) {
                        const uint64_t w0q = qa >> 7, w1q = (mhi - 1) >> 7;
                        for (uint64_t wq = w0q + tid; wq <= w1q; wq += T) {
                            const ulonglong2 e = __ldg(reinterpret_cast<const ulonglong2 *>(Tpi) + wq);
                            uint64_t qb = e.x & range_mask(wq, qa, mhi);
                            while (qb) {
                                const int j = __ffsll((long long)qb) - 1;
                                qb &= qb - 1;
                                const uint64_t m = 128 * wq + 2 * j + 1;
                                S += seg_count((uint64_t)(xp / (XT)m));  // mu(q) = -1
                                msl += 1;
                            }
                        }
                    }
                } else {
                    // any squarefree m with lpf(m) > p: 16-byte loads of packed mu*lpf
                    const uint64_t i_lo = ((uint64_t)mlo + 1) >> 1, i_hi = ((uint64_t)mhi - 1) >> 1;  // m = 2i + 1
                    for (uint64_t g = (i_lo >> 2) + tid; g <= (i_hi >> 2); g += T) {
                        const int4 v4 = __ldg(reinterpret_cast<const int4 *>(MU) + g);
                        const int32_t vals[4] = {v4.x, v4.y, v4.z, v4.w};
#pragma unroll
                        for (int kq = 0; kq < 4; kq++) {
                            const uint64_t i = 4 * g + kq;
                            const int32_t v = vals[kq];
                            if (i < i_lo || i > i_hi || v == 0) continue;
                            if ((uint32_t)(v > 0 ? v : -v) <= p) continue;
                            const uint32_t cv = seg_count((uint64_t)(xp / (XT)(2 * i + 1)));
                            if (v > 0) {
                                S -= cv;
                                msl -= 1;
                            } else {
                                S += cv;
                                msl += 1;
                            }
                        }
                    }
                }
#pragma unroll
                for (int dd = 16; dd > 0; dd >>= 1) msl += __shfl_down_sync(FULL, msl, dd);
                if (lane == 0 && msl) atomicAdd(s_ms, msl);
                __syncthreads();
                if (tid == 0) {
                    out_ms[slot] = *s_ms;
                    *s_ms = 0;
                }
            } else if (tid == 0) {
                out_ms[slot] = 0;
            }
            // cross off p_b, counting bits that were still set
            uint32_t cleared = 0;
            if (p < 64) {
                const uint32_t Mp = every_pth_bit(p);  // p < 32 has several multiples per word
                const uint32_t st = 64u % p;
                uint32_t r = (s_r0[k] + (64u * w0) % p) % p;
                for (uint32_t j = 0; j < CPT; j++) {
                    uint4 v = reinterpret_cast<const uint4 *>(bm)[swz(c0 + j, s)];
                    uint32_t a4[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
                    for (int kk = 0; kk < 4; kk++) {
                        const uint32_t mk = mult_mask(r, p, Mp);
                        cleared += __popc(a4[kk] & mk);
                        a4[kk] &= ~mk;
                        r += st;
                        if (r >= p) r -= p;
                    }
                    reinterpret_cast<uint4 *>(bm)[swz(c0 + j, s)] = make_uint4(a4[0], a4[1], a4[2], a4[3]);
                }
            } else {
                const uint32_t i0 = s_i0[k];
                if (i0 != 0xFFFFFFFFu) {
                    for (uint64_t i = (uint64_t)i0 + (uint64_t)tid * p; i < L; i += (uint64_t)T * p) {
                        const uint32_t w = (uint32_t)(i >> 5), bit = 1u << (i & 31);
                        const uint32_t pw = (swz(w >> 2, s) << 2) | (w & 3);
                        const uint32_t old = atomicAnd(&bm[pw], ~bit);
                        cleared += (old & bit) ? 1u : 0u;
                    }
                }
            }
#pragma unroll
            for (int dd = 16; dd > 0; dd >>= 1) cleared += __shfl_down_sync(FULL, cleared, dd);
            if (lane == 0 && cleared) atomicAdd(&s_clr[b & 1], (int)cleared);
            __syncthreads();
        }
    }
    const i128 Sb = cpx_block_sum_i128((i128)S, s_red);
    if (tid == 0) acc_add(acc, q, ACC_HARD, Sb);
}

// B(seg) = pi(min(r4, isqrt((x - 1) / lo), isqrt(hi - 1))): the levels b a
// segment sieves.  p_b^2 * lo < x bounds the levels whose leaves can reach
// the segment or a later one; p_b^2 < hi skips the levels whose leaves all lie
// above the segment, because below p_b^2 the carry phi(v, b - 1) is
// 1 + pi(v) - (b - 1) and k_hard_combine reads it from the pi table.
// Levels per segment = max(0, B - c).
template <class XT>
__global__ void k_hard_plan(const QD *__restrict__ qd, uint32_t Q, const uint64_t *__restrict__ pre_seg,
                            uint64_t total, const uint32_t *__restrict__ P, uint32_t np,
                            uint32_t *__restrict__ seg_B, uint64_t *__restrict__ seg_lv)
{
    const uint64_t u = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= total) return;
    const uint32_t q = find_q(pre_seg, Q, u);
    const QD &d = qd[q];
    const uint64_t seg = u - pre_seg[q];
    const uint64_t lo = seg * 2 * (1ull << d.lbits), hi = lo + 2 * (1ull << d.lbits);
    uint32_t B;
    {
        const XT x = xload<XT>(d);
        uint64_t v = d.r4;
        if (lo) {
            const uint64_t v1 = cpx_isqrt((u128)((x - 1) / (XT)lo));
            if (v1 < v) v = v1;
        }
        const uint64_t v2 = cpx_isqrt((u128)(hi - 1));
        if (v2 < v) v = v2;
        uint32_t a = 0, bnd = np;  // count of P[i] <= v
        while (a < bnd) {
            const uint32_t mid = (a + bnd) >> 1;
            if (P[mid] <= v) a = mid + 1;
            else bnd = mid;
        }
        B = a;
    }
    seg_B[u] = B;
    seg_lv[u] = B > d.c ? B - d.c : 0;
}

// H += sum over segments of carry(seg, b) * msum(seg, b); carry = count of
// survivors of level b-1 below the segment.  Level b is sieved from the first
// segment reaching p_b^2; below p_b^2 the survivors of level b-1 are 1 and the
// primes from p_b on, so the carry starts at 1 + max(0, pi(lo - 1) - (b - 1))
// from the pi table and then adds the sieved segments' counts.  One thread per
// (query, b).
__global__ void k_hard_combine(const QD *__restrict__ qd, uint32_t Q, const uint64_t *__restrict__ pre_comb,
                               uint64_t total, const uint64_t *__restrict__ pre_seg,
                               const uint32_t *__restrict__ seg_B, const uint64_t *__restrict__ seg_off,
                               const uint32_t *__restrict__ cnt, const int32_t *__restrict__ ms, uint64_t cap,
                               const uint32_t *__restrict__ P, const cpx_pient *__restrict__ T,
                               unsigned long long *__restrict__ acc)
{
    const uint64_t u = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    LaneAcc a;
    if (u < total) {
        const uint32_t q = find_q(pre_comb, Q, u);
        const uint64_t lvl = u - pre_comb[q];
        const QD &d = qd[q];
        const uint32_t b = d.c + 1 + (uint32_t)lvl;
        const uint64_t span = 2ull << d.lbits;
        const uint64_t p = P[b - 1];
        const uint64_t first = (p * p) / span;  // first segment with hi > p^2
        const uint64_t s0 = pre_seg[q] + first, s1 = pre_seg[q + 1];
        uint64_t carry = 0;
        if (first > 0 && s0 < s1) {
            const uint64_t lo = first * span;
            const uint64_t pl = cpx_pi_dev(T, lo - 1);
            carry = 1 + (pl > b - 1 ? pl - (b - 1) : 0);
        }
        i128 H = 0;
        for (uint64_t sg = s0; sg < s1; sg++) {
            if (seg_B[sg] < b) break;
            const uint64_t idx = seg_off[sg] + lvl;
            if (idx >= cap) break;
            H += (i128)carry * (i128)ms[idx];
            carry += cnt[idx];
        }
        a.q = q;
        a.v = H;
    }
    warp_flush(a, acc, ACC_HARD);
}

__global__ void k_finalize(const QD *__restrict__ qd, uint32_t Q, const cpx_pient *__restrict__ T,
                           unsigned long long *__restrict__ acc, u128 *__restrict__ out, int full)
{
    const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= Q) return;
    unsigned long long *A = acc + (uint64_t)q * kAccStride;
    auto rd = [&](int t) { return (i128)(((u128)A[2 * t + 1] << 64) | A[2 * t]); };
    auto wr = [&](int t, i128 v) {
        A[2 * t] = (unsigned long long)(u128)v;
        A[2 * t + 1] = (unsigned long long)((u128)v >> 64);
    };
    const QD &d = qd[q];
    i128 pi;
    if (!full) {
        wr(ACC_PIY, 0);
        wr(ACC_PI, 0);
        return;
    }
    if (d.direct) {
        pi = (i128)cpx_pi_dev(T, (uint64_t)d.x);
        wr(ACC_PIY, 0);
    } else {
        const i128 piy = (i128)cpx_pi_dev(T, d.y);
        wr(ACC_PIY, piy);
        pi = rd(ACC_ORD) + rd(ACC_TRIV) + rd(ACC_EASY) + rd(ACC_HARD) + piy - 1 - rd(ACC_P2);
    }
    wr(ACC_PI, pi);
    if (out) out[q] = (u128)pi;
}

// ------------------------------------------------------------------ launchers

static unsigned grid_for(cpx_ctx *ctx, uint64_t total_units, uint64_t units_per_thread_min = 1)
{
    const uint64_t want = (total_units + kThreads * units_per_thread_min - 1) / (kThreads * units_per_thread_min);
    const uint64_t cap = (uint64_t)ctx->sm_count * 8;
    return (unsigned)std::max<uint64_t>(1, std::min(want, cap));
}

template <int C, class XT> static void ord_launch(cpx_ctx *ctx, const Plan &pl)
{
    k_ordinary<C, XT><<<grid_for(ctx, pl.n_ord), kThreads, 0, ctx->stream>>>(pl.qd, pl.Q, pl.pre_ord, pl.n_ord,
                                                                               ctx->tab.MU, ctx->tab.WH, pl.acc);
}

template <class XT> static void ord_dispatch(cpx_ctx *ctx, const Plan &pl)
{
    switch (pl.c) {
    case 1: ord_launch<1, XT>(ctx, pl); break;
    case 2: ord_launch<2, XT>(ctx, pl); break;
    case 3: ord_launch<3, XT>(ctx, pl); break;
    case 4: ord_launch<4, XT>(ctx, pl); break;
    case 5: ord_launch<5, XT>(ctx, pl); break;
    case 6: ord_launch<6, XT>(ctx, pl); break;
    case 7: ord_launch<7, XT>(ctx, pl); break;
    case 8: ord_launch<8, XT>(ctx, pl); break;
    default: fail(CPX_EINVAL, "c must be in 1..8");
    }
}

void launch_ordinary(cpx_ctx *ctx, const Plan &pl)
{
    if (!pl.n_ord) return;
    if (pl.wide) ord_dispatch<u128>(ctx, pl);
    else ord_dispatch<uint64_t>(ctx, pl);
    CPX_LAUNCH("k_ordinary");
    note_launch(ctx);
}

void launch_p2(cpx_ctx *ctx, const Plan &pl)
{
    if (!pl.n_p2) return;
    if (pl.wide)
        k_p2<u128><<<grid_for(ctx, pl.n_p2), kThreads, 0, ctx->stream>>>(pl.qd, pl.Q, pl.pre_p2, pl.n_p2,
                                                                         ctx->tab.T, pl.acc);
    else
        k_p2<uint64_t><<<grid_for(ctx, pl.n_p2), kThreads, 0, ctx->stream>>>(pl.qd, pl.Q, pl.pre_p2, pl.n_p2,
                                                                             ctx->tab.T, pl.acc);
    CPX_LAUNCH("k_p2");
    note_launch(ctx);
}

void launch_trivial(cpx_ctx *ctx, const Plan &pl)
{
    if (!pl.n_triv) return;
    if (pl.wide)
        k_trivial<u128><<<grid_for(ctx, pl.n_triv), kThreads, 0, ctx->stream>>>(pl.qd, pl.Q, pl.pre_triv,
                                                                                pl.n_triv, ctx->tab.T, pl.acc);
    else
        k_trivial<uint64_t><<<grid_for(ctx, pl.n_triv), kThreads, 0, ctx->stream>>>(pl.qd, pl.Q, pl.pre_triv,
                                                                                    pl.n_triv, ctx->tab.T, pl.acc);
    CPX_LAUNCH("k_trivial");
    note_launch(ctx);
}

void launch_easy(cpx_ctx *ctx, const Plan &pl)
{
    if (!pl.n_easy) return;
    CPX_CUDA(cudaMemsetAsync(pl.ticket, 0, sizeof(unsigned int), ctx->stream));
    const unsigned grid = (unsigned)std::max<uint64_t>(
        1, std::min<uint64_t>((pl.n_easy + (kThreads / 32) - 1) / (kThreads / 32), (uint64_t)ctx->sm_count * 8));
    if (pl.wide)
        k_easy<u128><<<grid, kThreads, 0, ctx->stream>>>(pl.qd, pl.Q, pl.pre_easy, pl.n_easy, ctx->tab.T,
                                                         pl.ticket, pl.acc);
    else
        k_easy<uint64_t><<<grid, kThreads, 0, ctx->stream>>>(pl.qd, pl.Q, pl.pre_easy, pl.n_easy, ctx->tab.T,
                                                             pl.ticket, pl.acc);
    CPX_LAUNCH("k_easy");
    note_launch(ctx);
}

void launch_easy_comp(cpx_ctx *ctx, const Plan &pl)
{
    if (!pl.n_ecomp) return;
    const unsigned grid = (unsigned)std::max<uint64_t>(
        1, std::min<uint64_t>((pl.n_ecomp + (kThreads / 32) - 1) / (kThreads / 32), (uint64_t)ctx->sm_count * 16));
    if (pl.wide)
        k_easy_comp<u128><<<grid, kThreads, 0, ctx->stream>>>(pl.qd, pl.elv, pl.n_elv, pl.n_ecomp, ctx->tab.MU,
                                                              ctx->tab.T, pl.acc);
    else
        k_easy_comp<uint64_t><<<grid, kThreads, 0, ctx->stream>>>(pl.qd, pl.elv, pl.n_elv, pl.n_ecomp, ctx->tab.MU,
                                                                  ctx->tab.T, pl.acc);
    CPX_LAUNCH("k_easy_comp");
    note_launch(ctx);
}

size_t hard_smem_bytes(uint32_t lbits, uint32_t threads, bool wide)
{
    return wide ? HardSmem<u128>::bytes(lbits, threads) : HardSmem<uint64_t>::bytes(lbits, threads);
}

template <class XT> static void hard_go(cpx_ctx *ctx, const Plan &pl)
{
    const Tables &tb = ctx->tab;
    k_hard_plan<XT><<<(unsigned)((pl.n_seg + 255) / 256), 256, 0, ctx->stream>>>(
        pl.qd, pl.Q, pl.pre_seg, pl.n_seg, tb.P, (uint32_t)tb.prm_n, pl.seg_B, pl.seg_off);
    CPX_LAUNCH("k_hard_plan");
    note_launch(ctx);
    scan_u64(ctx, pl.seg_off, pl.n_seg);
    const size_t smem = HardSmem<XT>::bytes(pl.lbits_max, pl.hard_threads);
    CPX_CUDA(cudaFuncSetAttribute(k_hard<XT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    if (ctx->timing) CPX_CUDA(cudaEventRecord(ctx->ev_hard0, ctx->stream));
    k_hard<XT><<<(unsigned)pl.n_seg, pl.hard_threads, smem, ctx->stream>>>(
        pl.qd, pl.Q, pl.pre_seg, pl.n_seg, pl.seg_B, pl.seg_off, tb.P, tb.MU, tb.T, pl.hard_cnt, pl.hard_ms,
        pl.hard_entries, pl.acc, pl.lbits_max);
    CPX_LAUNCH("k_hard");
    if (ctx->timing) CPX_CUDA(cudaEventRecord(ctx->ev_hard1, ctx->stream));
    note_launch(ctx);
    if (pl.n_comb) {
        k_hard_combine<<<(unsigned)((pl.n_comb + 255) / 256), 256, 0, ctx->stream>>>(
            pl.qd, pl.Q, pl.pre_comb, pl.n_comb, pl.pre_seg, pl.seg_B, pl.seg_off, pl.hard_cnt, pl.hard_ms,
            pl.hard_entries, tb.P, tb.T, pl.acc);
        CPX_LAUNCH("k_hard_combine");
        note_launch(ctx);
    }
}

void launch_hard(cpx_ctx *ctx, const Plan &pl)
{
    if (!pl.n_seg) return;
    if (pl.n_seg > 0x7FFFFFFFull) fail(CPX_ERANGE, "too many hard-leaf segments in one launch");
    if (pl.wide) hard_go<u128>(ctx, pl);
    else hard_go<uint64_t>(ctx, pl);
}

void launch_finalize(cpx_ctx *ctx, const Plan &pl, u128 *d_out_pi, bool full)
{
    k_finalize<<<(pl.Q + 127) / 128, 128, 0, ctx->stream>>>(pl.qd, pl.Q, ctx->tab.T, pl.acc, d_out_pi, full ? 1 : 0);
    CPX_LAUNCH("k_finalize");
    note_launch(ctx);
}

}  // namespace cpx
