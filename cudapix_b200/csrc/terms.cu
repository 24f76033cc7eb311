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
#include "kern_common.cuh"

namespace cpx {


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
                const XT m = cpx_qdiv(x, n);
                XT qw;
                uint32_t r;
                if ((u128)m >> 64) {
                    qw = m / (XT)Wh::W;
                    r = (uint32_t)(m - qw * (XT)Wh::W);
                } else {  // below 2^64 (every n > x / 2^64): 64-bit division by the constant
                    const uint64_t m64 = (uint64_t)m, q64 = m64 / Wh::W;
                    qw = (XT)q64;
                    r = (uint32_t)(m64 - q64 * Wh::W);
                }
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
                const uint64_t xp = (uint64_t)cpx_qdiv(x, p);
                s += (int64_t)cpx_pi_dev(T, xp) - (int64_t)i + 1;
            }
            a.v += s;
        }
    }
    warp_flush(a, acc, ACC_P2);
}

// P2 by the prime list, when it reaches every query's sqrt x: one prime
// p = p_k per lane, k in (pi(y), pi(sqrt x)], adding pi(x/p) - k + 1.  The
// quotient x/p < z is cpx_quot40_core's when x < 2^53 and z < 2^41.
template <class XT>
__global__ void __launch_bounds__(kThreads) k_p2_primes(const QD *__restrict__ qd, uint32_t Q,
                                                        const uint64_t *__restrict__ pre, uint64_t total,
                                                        const uint32_t *__restrict__ P,
                                                        const cpx_pient *__restrict__ T,
                                                        unsigned long long *__restrict__ acc)
{
    const WarpSlice sl = warp_slice(total);
    const int lane = threadIdx.x & 31;
    LaneAcc a;
    QCache qc;
    XT x = 0;
    double xd = 0.0;
    uint64_t k0 = 0;
    bool fast = false;
    int64_t s = 0;  // this lane's sum for query a.q since the last fold
    for (uint64_t base = sl.u0; base < sl.u1; base += 32) {
        const uint64_t u = base + lane;
        if (u < sl.u1) {
            const uint32_t q = qlookup(qc, pre, Q, u);
            if (q != a.q) {
                a.v += s;
                s = 0;
                lane_switch(a, q, acc, ACC_P2);
                const QD &d = qd[q];
                x = xload<XT>(d);
                k0 = d.piy;
                fast = ((u128)x >> 53) == 0 && (d.z >> 41) == 0;
                xd = (double)(uint64_t)x;
            }
            const uint64_t k = k0 + 1 + (u - qc.lo);
            const uint32_t p = __ldg(P + k - 1);
            const uint64_t v = fast ? cpx_quot40_core<uint64_t>((uint64_t)x, xd, p, cpx_rcp_approx(p))
                                    : (uint64_t)cpx_qdiv(x, (uint64_t)p);
            s += (int64_t)cpx_pi_ge2(T, v) - (int64_t)k + 1;  // v >= p >= 2
        }
    }
    a.v += s;
    warp_flush(a, acc, ACC_P2);
}

// P2 for a query whose z lies beyond the resident pi table: the values
// v = x/p in [A, B) of one table window.  One lane per table entry of p
// candidates in (plo, phi] (p with x/p in the window); pi(v) = base + odd
// primes of the window up to v, pi(p) from the resident table.
template <class XT>
__global__ void __launch_bounds__(kThreads) k_p2_window(XT x, uint64_t plo, uint64_t phi, uint64_t A,
                                                        const cpx_pient *__restrict__ Tw, uint64_t base,
                                                        const cpx_pient *__restrict__ T,
                                                        unsigned long long *__restrict__ acc_q)
{
    const uint64_t w0 = plo >> 7, w1 = (phi - 1) >> 7;
    const uint64_t w = w0 + (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    int64_t s = 0;
    if (w <= w1) {
        const ulonglong2 e = __ldg(reinterpret_cast<const ulonglong2 *>(T) + w);
        uint64_t bits = e.x & range_mask(w, plo, phi);
        while (bits) {
            const int j = __ffsll((long long)bits) - 1;
            bits &= bits - 1;
            const uint64_t p = 128 * w + 2 * j + 1;
            const uint64_t i = 1 + e.y + __popcll(e.x & ((2ull << j) - 1));  // pi(p)
            const uint64_t v = (uint64_t)cpx_qdiv(x, p);
            uint64_t piv = base;  // v = A (even): pi(A) = pi(A - 1)
            if (v > A) {
                // the entry holding v - 1, as in cpx_pi_from_entry (A is a multiple of 128)
                const ulonglong2 ew = __ldg(reinterpret_cast<const ulonglong2 *>(Tw) + ((v - 1 - A) >> 7));
                const uint32_t jv = (uint32_t)(((v - 1) & 127) >> 1);
                piv += ew.y + __popcll(ew.x & ((2ull << jv) - 1));
            }
            s += (int64_t)piv - (int64_t)i + 1;
        }
    }
    __shared__ i128 red[32];
    const i128 b = cpx_block_sum_i128((i128)s, red);
    if (threadIdx.x == 0 && b != 0) cpx_atomic_add_i128(acc_q, b);
}

__global__ void k_pi_at(const cpx_pient *__restrict__ T, uint64_t n, uint64_t *out) { *out = cpx_pi_dev(T, n); }

constexpr uint64_t kP2WindowWords = 1ull << 27;  // at most 2^34 integers (2 GiB of window table) per window

void p2_windowed(cpx_ctx *ctx, const QD &d, unsigned long long *acc_q, bool wide)
{
    const u128 x = d.x;
    const uint64_t y = d.y, sx = d.sx;
    if (sx <= y) return;
    const uint64_t vmin = (uint64_t)(x / sx), vmax = (uint64_t)(x / (y + 1));
    uint64_t A = (vmin >> 7) << 7;
    // base = pi(A - 1) from the resident table (it reaches sqrt(x) + 1 >= A - 1)
    uint64_t *d_b = ctx->b_small.as<uint64_t>(8) + 6;
    k_pi_at<<<1, 1, 0, ctx->stream>>>(ctx->tab.T, A ? A - 1 : 0, d_b);
    CPX_LAUNCH("k_pi_at");
    note_launch(ctx);
    uint64_t base = 0;
    CPX_CUDA(cudaMemcpyAsync(&base, d_b, 8, cudaMemcpyDeviceToHost, ctx->stream));
    CPX_CUDA(cudaStreamSynchronize(ctx->stream));
    // windows of `p2_table_limit` integers (the resident-table bound), at most 2^34
    const uint64_t ww = std::min<uint64_t>(kP2WindowWords,
                                           std::max<uint64_t>(kTabSegWords, (ctx->p2_table_limit >> 7) / kTabSegWords *
                                                                                kTabSegWords));
    cpx_pient *Tw = ctx->b_win.as<cpx_pient>(ww + kTabSegWords);
    while (A <= vmax) {
        const uint64_t nwords = std::min<uint64_t>(ww, ((vmax - A) >> 7) + 1);
        const uint64_t odd = build_pitable_window(ctx, A >> 7, nwords, Tw);
        const uint64_t B = A + 128 * ((nwords + kTabSegWords - 1) / kTabSegWords * kTabSegWords);
        // p in (max(y, x/B), min(sx, x/A)]
        uint64_t plo = (uint64_t)(x / B), phi = A ? (uint64_t)std::min<u128>(x / A, (u128)sx) : sx;
        if (plo < y) plo = y;
        if (phi > plo) {
            const uint64_t nent = ((phi - 1) >> 7) - (plo >> 7) + 1;
            const unsigned grid = (unsigned)((nent + kThreads - 1) / kThreads);
            if (wide)
                k_p2_window<u128><<<grid, kThreads, 0, ctx->stream>>>(x, plo, phi, A, Tw, base, ctx->tab.T, acc_q);
            else
                k_p2_window<uint64_t><<<grid, kThreads, 0, ctx->stream>>>((uint64_t)x, plo, phi, A, Tw, base,
                                                                           ctx->tab.T, acc_q);
            CPX_LAUNCH("k_p2_window");
            note_launch(ctx);
        }
        base += odd;
        A = B;
    }
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
// (for p > iroot4(x) the bound x/p^3 is below p); k_easy_comp takes the
// composite m.
//
// Per p the q range (qlo, qhi] is split at q1 ~ sqrt(x/p).  Below q1 every q
// gives its own u and the leaves are taken one by one (sparse part): the q
// are the primes p_k, k in (pi(qlo), pi(q1)], read from the resident prime
// list (which reaches y), 32 consecutive k a warp step.  Above
// q1 runs of consecutive primes q share pi(x/(pq)) (clustered part): with
// G(k) = pi(clamp(x/(p p_k), q1, qhi)) the primes q of the run with
// pi(x/(pq)) = k number G(k) - G(k+1), and summation by parts turns
//   Sum_{q in (q1, qhi]} (pi(x/(pq)) - b + 2)
// into (klo - b + 2) pi(qhi) - (khi - b + 2) pi(q1) + Sum_{klo < k <= khi} G(k)
// with klo = pi(x/(p qhi)), khi = pi(x/(p (q1 + 1))): one quotient and one
// table lookup per prime u instead of per leaf.  The u primes come from the
// resident prime list, so q1 is raised until x/(p (q1 + 1)) <= prm_max.

constexpr uint64_t kEasySparse = 1024;  // primes q per sparse work chunk (2048: 12.8 ms, 4096: 14.9 ms on the batch)
constexpr uint64_t kEasyClu = 512;      // u primes per clustered work chunk

struct EasyP {
    uint64_t qlo, qhi, q1;  // sparse q in (qlo, q1], clustered q in (q1, qhi]
    uint64_t kq0, kq1;      // pi(qlo), pi(q1): the sparse q are p_k, kq0 < k <= kq1
    uint64_t klo, khi;      // pi(x / (p qhi)), pi(x / (p (q1 + 1)))
    uint64_t nsp, ncl;      // work chunks of the two parts
};

template <class XT>
__device__ __noinline__ bool easy_plan(XT x, uint64_t y, uint64_t p, uint64_t prm_max,
                                          const cpx_pient *__restrict__ T, XT &xp, EasyP &e)
{
    xp = cpx_qdiv(x, p);
    uint64_t qlo = y / p;
    if (qlo < p) qlo = p;
    const XT xpp = cpx_qdiv(xp, p);
    const XT x3 = cpx_qdiv(xpp, p);  // p <= iroot4(x): only q > x/p^3 (x/(pq) < p^2) are easy
    if (x3 > (XT)qlo) qlo = (x3 >= (XT)y) ? y : (uint64_t)x3;
    const uint64_t qhi = (xpp < (XT)y) ? (uint64_t)xpp : y;
    if (qhi <= qlo) return false;
    uint64_t q1 = cpx_isqrt((u128)xp);
    const XT lim = xp / (XT)prm_max;
    if (lim > (XT)q1) q1 = (lim >= (XT)qhi) ? qhi : (uint64_t)lim;
    q1 = q1 < qlo ? qlo : (q1 > qhi ? qhi : q1);
    e.qlo = qlo;
    e.qhi = qhi;
    e.q1 = q1;
    if (q1 > qlo) {
        e.kq0 = cpx_pi_dev(T, qlo);
        e.kq1 = cpx_pi_dev(T, q1);
    } else {
        e.kq0 = e.kq1 = 0;
    }
    e.nsp = (e.kq1 - e.kq0 + kEasySparse - 1) / kEasySparse;
    if (qhi > q1) {
        e.klo = cpx_pi_dev(T, (uint64_t)cpx_qdiv(xp, qhi));
        e.khi = cpx_pi_dev(T, (uint64_t)cpx_qdiv(xp, q1 + 1));
        e.ncl = e.khi > e.klo ? (e.khi - e.klo + kEasyClu - 1) / kEasyClu : 1;
    } else {
        e.klo = e.khi = 0;
        e.ncl = 0;
    }
    return true;
}

// The plan of one easy unit (query, p = p_b), written by pass 1 for pass 2.
struct __align__(16) EasyRec {
    u128 xp;
    uint64_t klo, khi;
    uint32_t qlo, q1, qhi, kq0;
    uint32_t kq1, b, q, pad;
};
static_assert(sizeof(EasyRec) == 64, "EasyRec is four 16-byte words");

__device__ __forceinline__ void easy_unpack(const EasyRec &r, EasyP &e)
{
    e.qlo = r.qlo;
    e.q1 = r.q1;
    e.qhi = r.qhi;
    e.kq0 = r.kq0;
    e.kq1 = r.kq1;
    e.klo = r.klo;
    e.khi = r.khi;
    e.nsp = (e.kq1 - e.kq0 + kEasySparse - 1) / kEasySparse;
    e.ncl = e.qhi > e.q1 ? (e.khi > e.klo ? (e.khi - e.klo + kEasyClu - 1) / kEasyClu : 1) : 0;
}

// Pass 1: work chunks of each p (one thread per p = P[c + i]); cnt[total] is
// left 0 so that the exclusive scan of cnt ends with the grand total.  With
// rec, the units that have leaves also leave their plan there.
template <class XT>
__global__ void k_easy_count(const QD *__restrict__ qd, uint32_t Q, const uint64_t *__restrict__ pre, uint64_t total,
                             const uint32_t *__restrict__ P, uint64_t prm_max, const cpx_pient *__restrict__ T,
                             uint64_t *__restrict__ cnt, EasyRec *__restrict__ rec)
{
    const uint64_t unit = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (unit > total) return;
    if (unit == total) {
        cnt[unit] = 0;
        return;
    }
    const uint32_t q = find_q(pre, Q, unit);
    const QD &d = qd[q];
    const uint64_t p = __ldg(P + d.c + (unit - pre[q]));
    XT xp;
    EasyP e;
    const bool any = easy_plan<XT>(xload<XT>(d), d.y, p, prm_max, T, xp, e);
    cnt[unit] = any ? e.nsp + e.ncl : 0;
    if (rec && any && e.nsp + e.ncl) {
        EasyRec r;
        r.xp = (u128)xp;
        r.klo = e.klo;
        r.khi = e.khi;
        r.qlo = (uint32_t)e.qlo;
        r.q1 = (uint32_t)e.q1;
        r.qhi = (uint32_t)e.qhi;
        r.kq0 = (uint32_t)e.kq0;
        r.kq1 = (uint32_t)e.kq1;
        r.b = d.c + 1 + (uint32_t)(unit - pre[q]);
        r.q = q;
        r.pad = 0;
        rec[unit] = r;
    }
}

// Pass 2: each warp owns a contiguous slice of chunks.  A sparse chunk is
// kEasySparse consecutive primes q of one p (lane l takes k = k0 + l, k0 + l +
// 32, ...); a clustered chunk is kEasyClu consecutive u primes of one p.
template <class XT>
__global__ void __launch_bounds__(kThreads) k_easy(const QD *__restrict__ qd, uint32_t Q,
                                                   const uint64_t *__restrict__ pre, uint64_t total_units,
                                                   const uint64_t *__restrict__ off,
                                                   const uint32_t *__restrict__ P, uint64_t prm_max,
                                                   const cpx_pient *__restrict__ T,
                                                   unsigned long long *__restrict__ acc,
                                                   const EasyRec *__restrict__ rec)
{
    const int lane = threadIdx.x & 31;
    const WarpSlice sl = warp_slice(off[total_units]);
    LaneAcc a;
    // decoded state of the current p, kept across its consecutive chunks
    uint64_t c_unit = ~0ull, c_first = 0, c_last = 0, b = 0;
    uint32_t q = 0;
    XT xp = 0;
    EasyP e = {};
    for (uint64_t ch = sl.u0; ch < sl.u1; ch++) {
        if (ch > c_last || c_unit == ~0ull) {
            // the unit of chunk ch: a binary search for the slice's first
            // chunk, then a walk forward (units without leaves have no chunks)
            if (c_unit == ~0ull) {
                uint64_t lo = 0, hi = total_units;  // off[lo] <= ch < off[hi]
                while (hi - lo > 1) {
                    const uint64_t mid = (lo + hi) >> 1;
                    if (__ldg(off + mid) <= ch) lo = mid;
                    else hi = mid;
                }
                c_unit = lo;
            } else {
                do c_unit++;
                while (__ldg(off + c_unit + 1) <= ch);
            }
            if (rec) {
                const EasyRec r = rec[c_unit];
                xp = (XT)r.xp;
                easy_unpack(r, e);
                b = r.b;
                q = r.q;
            } else {
                q = find_q(pre, Q, c_unit);
                const QD &d = qd[q];
                const uint64_t i = c_unit - __ldg(pre + q);
                b = d.c + 1 + i;  // p = p_b
                easy_plan<XT>(xload<XT>(d), d.y, __ldg(P + d.c + i), prm_max, T, xp, e);
            }
            c_first = __ldg(off + c_unit);
            c_last = c_first + e.nsp + e.ncl - 1;
        }
        if (q != a.q) {  // q is the same on every lane of the warp
            warp_flush(a, acc, ACC_EASY);
            a.q = q;
        }
        const uint64_t r = ch - c_first;
        if (r < e.nsp) {
            const uint64_t k0 = e.kq0 + 1 + r * kEasySparse, k1 = min(e.kq1, e.kq0 + (r + 1) * kEasySparse);
            // x < 2^64 and x/p < 2^40: every quotient below 2^30 (u < sqrt(x) and
            // x < 2^60 here), taken by cpx_pi_quot40; else x/p < 2^53 with
            // quotients below 2^41 (x/p < 2^41 qlo): cpx_quot40; below 2^44:
            // cpx_quot53; else the general quotient.  One loop per case.
            const uint32_t *Pq = P + (k0 - 1);
            const uint32_t nq = (uint32_t)(k1 - k0 + 1);
            const double xpd = (double)(uint64_t)xp;
            uint64_t ps = 0;
            uint32_t t = lane;
            if (sizeof(XT) == 8 && (uint64_t)xp < (1ull << 40)) {
                const uint64_t n = (uint64_t)xp;
                // four leaves a lane a step: their table gathers overlap
                for (; t + 96 < nq; t += 128) {
                    const uint32_t d0 = __ldg(Pq + t), d1 = __ldg(Pq + t + 32), d2 = __ldg(Pq + t + 64),
                                   d3 = __ldg(Pq + t + 96);
                    ps += (cpx_pi_quot40(T, n, xpd, d0) + cpx_pi_quot40(T, n, xpd, d1)) +
                          (cpx_pi_quot40(T, n, xpd, d2) + cpx_pi_quot40(T, n, xpd, d3));
                }
                for (; t < nq; t += 32) ps += cpx_pi_quot40(T, n, xpd, __ldg(Pq + t));
            } else if (xp < ((XT)1 << 53) && ((uint64_t)xp >> 41) < e.qlo) {
                // quotients below 2^41 (q > qlo): cpx_quot40, four leaves a step
                const uint64_t n = (uint64_t)xp;
                for (; t + 96 < nq; t += 128) {
                    const uint32_t d0 = __ldg(Pq + t), d1 = __ldg(Pq + t + 32), d2 = __ldg(Pq + t + 64),
                                   d3 = __ldg(Pq + t + 96);
                    ps += (cpx_pi_ge2(T, cpx_quot40(n, xpd, d0)) + cpx_pi_ge2(T, cpx_quot40(n, xpd, d1))) +
                          (cpx_pi_ge2(T, cpx_quot40(n, xpd, d2)) + cpx_pi_ge2(T, cpx_quot40(n, xpd, d3)));
                }
                for (; t < nq; t += 32) ps += cpx_pi_ge2(T, cpx_quot40(n, xpd, __ldg(Pq + t)));
            } else if (xp < ((XT)1 << 53) && ((uint64_t)xp >> 44) < e.qlo) {
                const uint64_t n = (uint64_t)xp;
                for (; t + 32 < nq; t += 64)
                    ps += cpx_pi_ge2(T, cpx_quot53(n, xpd, __ldg(Pq + t))) +
                          cpx_pi_ge2(T, cpx_quot53(n, xpd, __ldg(Pq + t + 32)));
                if (t < nq) ps += cpx_pi_ge2(T, cpx_quot53(n, xpd, __ldg(Pq + t)));
            } else {
                for (; t < nq; t += 32) ps += cpx_pi_dev(T, (uint64_t)cpx_qdiv(xp, (uint64_t)__ldg(Pq + t)));
            }
            i128 add = (i128)ps;
            if (lane == 0) add += (i128)(k1 - k0 + 1) * (2 - (i128)b);
            a.v += add;
        } else {
            const uint64_t j = r - e.nsp;
            const uint64_t k0 = e.klo + 1 + j * kEasyClu, k1 = min(e.khi, e.klo + (j + 1) * kEasyClu);
            uint64_t ps = 0;
            // x/(p p_k) <= qhi < 2^31 for k > klo: cpx_quot40 when x/p < 2^53,
            // else cpx_qdiv
            const bool f40 = xp < ((XT)1 << 53);
            const double xpd = (double)(uint64_t)xp;
            auto g = [&](uint64_t k) -> uint64_t {
                const uint32_t pk = __ldg(P + k - 1);
                uint64_t v = f40 ? cpx_quot40((uint64_t)xp, xpd, pk) : (uint64_t)cpx_qdiv(xp, (uint64_t)pk);
                v = v < e.q1 ? e.q1 : (v > e.qhi ? e.qhi : v);
                return cpx_pi_ge2(T, v);
            };
            uint64_t k = k0 + lane;
            for (; k + 96 <= k1; k += 128) ps += (g(k) + g(k + 32)) + (g(k + 64) + g(k + 96));
            for (; k <= k1; k += 32) ps += g(k);
            i128 add = (i128)ps;
            if (j == 0 && lane == 0)
                add += ((i128)e.klo - (i128)b + 2) * (i128)cpx_pi_dev(T, e.qhi) -
                       ((i128)e.khi - (i128)b + 2) * (i128)cpx_pi_dev(T, e.q1);
            a.v += add;
        }
    }
    warp_flush(a, acc, ACC_EASY);
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
        const XT xp = cpx_qdiv(xload<XT>(d), r.p);
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
                const uint64_t uu = (uint64_t)cpx_qdiv(xp, m);
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
    KSpan ks(ctx, "k_ordinary");
    if (pl.wide) ord_dispatch<u128>(ctx, pl);
    else ord_dispatch<uint64_t>(ctx, pl);
    CPX_LAUNCH("k_ordinary");
    note_launch(ctx);
}

void launch_p2(cpx_ctx *ctx, const Plan &pl)
{
    if (!pl.n_p2) return;
    KSpan ks(ctx, "k_p2");
    if (pl.p2_primes) {
        if (pl.wide)
            k_p2_primes<u128><<<grid_for(ctx, pl.n_p2), kThreads, 0, ctx->stream>>>(pl.qd, pl.Q, pl.pre_p2, pl.n_p2,
                                                                                    ctx->tab.P, ctx->tab.T, pl.acc);
        else
            k_p2_primes<uint64_t><<<grid_for(ctx, pl.n_p2), kThreads, 0, ctx->stream>>>(
                pl.qd, pl.Q, pl.pre_p2, pl.n_p2, ctx->tab.P, ctx->tab.T, pl.acc);
    } else if (pl.wide)
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
    uint64_t *off = pl.easy_off;
    EasyRec *rec = static_cast<EasyRec *>(pl.easy_rec);
    const unsigned gc = (unsigned)((pl.n_easy + 1 + 255) / 256);
    const Tables &tb = ctx->tab;
    if (pl.wide)
        k_easy_count<u128><<<gc, 256, 0, ctx->stream>>>(pl.qd, pl.Q, pl.pre_easy, pl.n_easy, tb.P, tb.prm_max,
                                                         tb.T, off, rec);
    else
        k_easy_count<uint64_t><<<gc, 256, 0, ctx->stream>>>(pl.qd, pl.Q, pl.pre_easy, pl.n_easy, tb.P, tb.prm_max,
                                                             tb.T, off, rec);
    CPX_LAUNCH("k_easy_count");
    note_launch(ctx);
    scan_u64(ctx, off, pl.n_easy + 1);
    const unsigned grid = (unsigned)ctx->sm_count * 8;
    KSpan ks(ctx, "k_easy");
    if (pl.wide)
        k_easy<u128><<<grid, kThreads, 0, ctx->stream>>>(pl.qd, pl.Q, pl.pre_easy, pl.n_easy, off, tb.P, tb.prm_max,
                                                         tb.T, pl.acc, rec);
    else
        k_easy<uint64_t><<<grid, kThreads, 0, ctx->stream>>>(pl.qd, pl.Q, pl.pre_easy, pl.n_easy, off, tb.P,
                                                             tb.prm_max, tb.T, pl.acc, rec);
    CPX_LAUNCH("k_easy");
    note_launch(ctx);
}

void launch_easy_comp(cpx_ctx *ctx, const Plan &pl)
{
    if (!pl.n_ecomp) return;
    const unsigned grid = (unsigned)std::max<uint64_t>(
        1, std::min<uint64_t>((pl.n_ecomp + (kThreads / 32) - 1) / (kThreads / 32), (uint64_t)ctx->sm_count * 16));
    KSpan ks(ctx, "k_easy_comp");
    if (pl.wide)
        k_easy_comp<u128><<<grid, kThreads, 0, ctx->stream>>>(pl.qd, pl.elv, pl.n_elv, pl.n_ecomp, ctx->tab.MU,
                                                              ctx->tab.T, pl.acc);
    else
        k_easy_comp<uint64_t><<<grid, kThreads, 0, ctx->stream>>>(pl.qd, pl.elv, pl.n_elv, pl.n_ecomp, ctx->tab.MU,
                                                                  ctx->tab.T, pl.acc);
    CPX_LAUNCH("k_easy_comp");
    note_launch(ctx);
}

void launch_finalize(cpx_ctx *ctx, const Plan &pl, u128 *d_out_pi, bool full)
{
    k_finalize<<<(pl.Q + 127) / 128, 128, 0, ctx->stream>>>(pl.qd, pl.Q, ctx->tab.T, pl.acc, d_out_pi, full ? 1 : 0);
    CPX_LAUNCH("k_finalize");
    note_launch(ctx);
}

}  // namespace cpx
