// driver.cu -- host planning and execution of a batch of pi(x) queries (or of
// single terms) over the resident tables.
//
// Restates the reference driver (src/Deleglise-Rivat/deleglise-rivat.cpp:13-80:
// bounds, pi values at the bounds, the term identity) with exact integer
// roots, and replaces its one-term-at-a-time, synchronise-after-every-launch
// flow with one pass of a handful of kernels over every query of a batch.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <exception>
#include <mutex>
#include <thread>

#include "driver.h"
#include "misc.h"
#include "terms.cuh"

namespace cpx {

static const uint32_t kSmallPrimes[9] = {1, 2, 3, 5, 7, 11, 13, 17, 19};

uint32_t alpha_milli(u128 x)
{
    // alpha(x) of src/main.cpp:128-194: a cubic in log x.  Only chooses y.
    const double lx = std::log((double)x);
    double a, b, c, d;
    if ((double)x <= 1e21) {
        a = 0.000711339, b = -0.0160586, c = 0.123034, d = 0.802942;
    } else {
        a = 0.00149066, b = -0.0375705, c = 0.282139, d = 0.591972;
    }
    double al = a * lx * lx * lx + b * lx * lx + c * lx + d;
    if (al < 1.0) al = 1.0;
    return (uint32_t)std::lround(al * 1000.0);
}

uint64_t default_y(u128 x, uint32_t num, uint32_t den)
{
    if (num == 0 || den == 0) {
        num = alpha_milli(x);
        den = 1000;
    }
    // the reference's rule (src/main.cpp:59-64): y = alpha * floor(x^(1/3)),
    // truncated to an integer; here alpha = num/den and every step is exact
    const uint64_t cb = cpx_icbrt(x);
    uint64_t y = (uint64_t)((u128)cb * num / den);
    const uint64_t lo = cb, hi = cpx_isqrt(x);
    if (y < lo) y = lo;
    if (hi > 0 && y >= hi) y = hi - 1;
    return y;
}

const std::vector<uint32_t> &host_primes(cpx_ctx *ctx)
{
    Tables &tb = ctx->tab;
    if (ctx->hP_version != tb.prm_max) {
        ctx->hP.resize(tb.prm_n);
        CPX_CUDA(cudaMemcpy(ctx->hP.data(), tb.P, tb.prm_n * 4, cudaMemcpyDeviceToHost));
        ctx->hP_version = tb.prm_max;
    }
    return ctx->hP;
}

uint64_t host_pi(const std::vector<uint32_t> &P, uint64_t v)
{
    return (uint64_t)(std::upper_bound(P.begin(), P.end(), (uint64_t)v,
                                       [](uint64_t a, uint32_t b) { return a < b; }) -
                      P.begin());
}

bool dr_domain_ok(u128 x, uint64_t y, uint32_t c)
{
    if (c < 1 || c > 8) return false;
    if (x < 1000000) return false;
    const uint64_t sx = cpx_isqrt(x), cx = cpx_icbrt(x), r4 = cpx_iroot4(x);
    const uint32_t pc = kSmallPrimes[c];
    if (y < cx || y >= sx) return false;
    if (r4 < pc) return false;
    if (cpx_isqrt(x / y) < pc) return false;
    if (y >= 0x7FFFFFF0ull) return false;
    return true;
}

// P2 takes its primes from the prime list for sqrt x up to this bound (the
// list then holds up to 28 M primes, 112 MB); beyond it from pi-table bitmaps
constexpr uint64_t kP2PrimeMax = 1ull << 29;
static uint64_t tb_prm_max(const cpx_ctx *ctx) { return ctx->tab.P ? ctx->tab.prm_max : 0; }

// An upper bound of x^(2/5), at most 2^31: the u primes an easy leaf's
// clustered part needs (the kernels fall back to single leaves above the
// resident prime list, so the bound only has to be close).
static uint64_t easy_u_bound(u128 x)
{
    const double v = std::pow((double)x, 0.4) * 1.001 + 16.0;
    return v >= 2147483648.0 ? 2147483648ull : (uint64_t)v;
}

// Segments (of `span` integers) that sieve level b, p = p_b: those with
// hi > p^2 and (lo = 0 or p^2 lo < x); the same rule as k_hard_plan.
static uint64_t segments_at_level(u128 x, uint64_t span, uint64_t p, uint64_t seg0, uint64_t nseg)
{
    const uint64_t p2 = p * p;  // p <= iroot4(x) < 2^32
    const uint64_t first = std::max<uint64_t>(p2 / span, seg0);
    // largest s >= 0 with s * span * p^2 < x (p^2 span < 2^64 for the segment sizes used)
    const u128 d = (u128)p2 * span;
    const uint64_t end = seg0 + nseg;
    const uint64_t last = (x >> 64) || (d >> 64) ? (uint64_t)std::min<u128>((x - 1) / d, (u128)end)
                                                 : ((uint64_t)x - 1) / (uint64_t)d;
    const uint64_t hi = std::min<uint64_t>(last, end - 1);
    return hi >= first ? hi - first + 1 : 0;
}

// Number of (sub-segment, level) leaf sets of one query that k_hard hands to
// k_hard_leaves at threshold thr: the same candidate bounds as k_hard's warps
// (m in (max(y/p, xp/hi_w), min(y, xp/lo_w, x/p^3)], prime m only when
// p^2 > y).  Along a level the candidate count rises while the sub-segments
// reach into the leaves' smallest u and falls once xp/lo_w is the upper
// bound, so each level is scanned from its first sub-segment with leaves to
// the first light one past that point.  Stops counting at `limit`.
template <class XT>
static uint64_t heavy_leaf_sets(const QD &d, const std::vector<uint32_t> &hP, uint32_t threads, uint64_t thr,
                                uint64_t limit)
{
    const uint64_t NW = threads / 32, Lw = (1ull << d.lbits) / NW, span_w = 2 * Lw;
    const uint64_t w_beg = d.seg0 * NW, nsub = (d.seg0 + d.nseg) * NW, L2 = 2ull << d.lbits;
    const XT x = (XT)d.x;
    const uint64_t y = d.y;
    uint64_t jobs = 0;
    for (uint32_t b = d.c + 1; b <= d.nb && jobs < limit; b++) {
        const uint64_t p = hP[b - 1];
        const XT xp = x / (XT)p;
        const XT x3 = xp / (XT)(p * p);
        const uint64_t mtop = x3 < (XT)y ? (uint64_t)x3 : y;
        if (mtop <= y / p) continue;
        // No sub-segment holds more than mtop^2 span_w / (xp + span_w mtop) + 2
        // candidate m (the densest one starts at u = xp / mtop), and a set's
        // count is at most half its m range + 16: skip levels below thr.
        const double dm = (double)mtop, dsw = (double)span_w;
        const double most = 1.001 * dm * dm * dsw / ((double)xp + dsw * dm) + 2.0;
        if (0.5 * most + 17.0 < (double)thr) continue;
        const bool prime_lvl = p * p > y;
        for (uint64_t w = std::max<uint64_t>((uint64_t)(xp / (XT)mtop) / span_w, w_beg); w < nsub; w++) {
            const uint64_t lo_w = w * span_w, hi_w = lo_w + span_w;
            const uint64_t lo = (w / NW) * L2;
            if (lo && (u128)p * p > (u128)((x - 1) / (XT)lo)) break;  // p^2 lo >= x here and above
            if ((u128)p * p > (u128)(lo + L2 - 1)) continue;
            uint64_t mlo = y / p;
            const XT t1 = xp / (XT)hi_w;
            if (t1 > (XT)mlo) mlo = (uint64_t)t1;
            uint64_t mhi = mtop;
            bool interior = false;
            if (lo_w) {
                const XT t2 = xp / (XT)lo_w;
                if (t2 < (XT)mhi) {
                    mhi = (uint64_t)t2;
                    interior = true;
                }
            }
            if (mhi <= mlo) {
                if (interior) break;
                continue;
            }
            uint64_t work;
            const uint64_t qa = mlo > p ? mlo : p;
            if (prime_lvl) work = (mhi > qa) ? 8 * (((mhi - 1) >> 7) - (qa >> 7) + 1) : 0;
            else work = ((mhi - 1) >> 1) - ((mlo + 1) >> 1) + 1;
            if (work >= thr) {
                if (++jobs >= limit) break;
            } else if (interior) {
                break;
            }
        }
    }
    return jobs;
}

// Hard-leaf segment sizes for a batch.  A query never gets a segment longer
// than needed to cover [0, z]; below the context default the sizes of the
// largest queries shrink (one cap for all) until the whole batch has about
// four segments per SM, so one large query still fills the GPU while a big
// batch keeps long segments (fewer segment-levels to sieve).
static u128 xmax_all(const std::vector<QD> &qd)
{
    u128 m = 0;
    for (const QD &d : qd)
        if (!d.direct && d.x > m) m = d.x;
    return m;
}

static void choose_lbits(cpx_ctx *ctx, std::vector<QD> &qd, uint32_t c, uint32_t threads, uint32_t forced,
                         uint32_t cap_all, const TuneEntry *tune)
{
    const uint32_t minb = (threads >= 512) ? 16 : (threads >= 256 ? 15 : 14);
    std::vector<uint32_t> nat(qd.size(), 0);
    for (size_t i = 0; i < qd.size(); i++) {
        const QD &d = qd[i];
        if (d.direct || d.nb <= c) continue;
        if (forced) {
            nat[i] = std::max(minb, std::min<uint32_t>(forced, 20));
            continue;
        }
        uint32_t qcap = cap_all ? cap_all : ctx->hard_log2_bits;
        if (!cap_all && tune && tune[decade_of(d.x)].lbits) qcap = tune[decade_of(d.x)].lbits;
        uint32_t lb = minb;
        while (lb < qcap && (2ull << lb) < d.z + 1) lb++;
        nat[i] = lb;
    }
    uint32_t cap = 20;  // the per-query caps are in nat[]; this batch-wide cap only shrinks them
    const uint64_t target = (uint64_t)ctx->sm_count * 4;
    for (;;) {
        uint64_t segs = 0;
        for (size_t i = 0; i < qd.size(); i++)
            if (nat[i]) {
                const uint32_t lb = std::min(nat[i], cap);
                segs += (qd[i].z + 1 + (2ull << lb) - 1) / (2ull << lb);
            }
        if (forced || segs >= target || cap <= minb) break;
        cap--;
    }
    for (size_t i = 0; i < qd.size(); i++)
        if (nat[i]) qd[i].lbits = std::min(nat[i], cap);
}

// Segment size and group size of the batch-shared sieve (order: the queries
// with hard leaves, z descending).  The segment is the smallest that covers
// the largest z, at most the cap; the segment and then the groups (32
// queries at most) shrink while the batch has fewer than four work units per
// SM.
static uint32_t choose_shared(cpx_ctx *ctx, const std::vector<QD> &qd, const std::vector<uint32_t> &order,
                              uint32_t threads, uint32_t forced, uint32_t cap_all, uint32_t &gsize)
{
    const uint32_t minb = (threads >= 1024) ? 17 : (threads >= 512) ? 16 : (threads >= 256 ? 15 : 14);
    const uint32_t cap = std::max(minb, std::min<uint32_t>(forced ? forced : (cap_all ? cap_all : ctx->hard_log2_bits), 20));
    uint32_t lb = minb;
    while (lb < cap && (2ull << lb) < qd[order[0]].z + 1) lb++;
    auto units = [&](uint32_t l, uint32_t G) {
        uint64_t u = 0;
        for (size_t k = 0; k < order.size(); k += G) u += (qd[order[k]].z + 1 + (2ull << l) - 1) / (2ull << l);
        return u;
    };
    const uint64_t target = (uint64_t)ctx->sm_count * 4;
    gsize = kGroupMax;
    if (!forced)
        while (lb > minb && units(lb, gsize) < target) lb--;
    while (gsize > 1 && units(lb, gsize) < target) gsize /= 2;
    return lb;
}

// Alpha scales of a batch under the batch tuning.  Its alpha (tuned on a
// sample batch) pays off for queries that share their sieve with others; a
// query with fewer than 16 companions within half a decade of x sieves
// mostly alone and takes its decade's tuned scale (the reference alpha when
// untuned).  Larger x share less (their easy leaves, which no query shares,
// grow as pi(y)^2), so a decade may carry a batch scale of its own (bdec):
// on the B200, batches of 64 queries in [1e16, 1e17) and [1e17, 1e18) ran
// fastest at 1/4 and 1/2 of the reference alpha, against 1/8 below 1e16.
static std::vector<uint32_t> batch_alpha_scales(const u128 *xs, uint32_t Q, uint32_t batch_sc, const TuneEntry *tune,
                                                const uint32_t *bdec)
{
    std::vector<std::pair<double, uint32_t>> lx(Q);
    for (uint32_t i = 0; i < Q; i++) lx[i] = {std::log10((double)xs[i]), i};
    std::sort(lx.begin(), lx.end());
    std::vector<uint32_t> sc(Q);
    size_t a = 0, b = 0;
    for (size_t k = 0; k < Q; k++) {
        while (lx[k].first - lx[a].first > 0.5) a++;
        while (b < Q && lx[b].first - lx[k].first <= 0.5) b++;
        uint32_t v = batch_sc;
        {
            const uint32_t e = decade_of(xs[lx[k].second]);
            if (bdec && e < kTuneDecades && bdec[e]) v = bdec[e];  // the batch scale of the decade
        }
        if (b - a < 17) {
            const uint32_t e = decade_of(xs[lx[k].second]);
            v = (tune && e < kTuneDecades && tune[e].alpha_milli) ? tune[e].alpha_milli : 1000;
        }
        sc[lx[k].second] = v;
    }
    return sc;
}

// Groups that share one sieve of segment sg in the batch-shared sieve.  The
// early segments hold most of the leaves, so a unit of many groups there
// would outlast the rest of the launch; the later ones are mostly crossing
// off, which the groups of a block share.
static uint32_t shared_block(uint64_t sg)
{
    return sg < 4 ? 1u : sg < 16 ? 2u : sg < 64 ? 4u : kBlockMax;
}

// Bytes of the counting sweep's carry rows for the queries `order` of a
// shared sieve with segments of 2^lbits odd numbers and `threads` per block.
static uint64_t carry_row_bytes(const std::vector<QD> &qd, const std::vector<uint32_t> &order,
                                const std::vector<uint32_t> &hP, uint32_t lbits, uint32_t threads, uint32_t c)
{
    const uint64_t span = 2ull << lbits;
    u128 xmax = 0;
    uint64_t r4max = 0, nseg = 0;
    for (uint32_t i : order) {
        xmax = std::max(xmax, qd[i].x);
        r4max = std::max(r4max, qd[i].r4);
        nseg = std::max(nseg, (qd[i].z + 1 + span - 1) / span);
    }
    const uint64_t nbm = host_pi(hP, r4max);
    uint64_t rows = 0;
    for (uint64_t b = c + 1; b <= nbm; b++) rows += segments_at_level(xmax, span, hP[b - 1], 0, nseg);
    return rows * (threads / 32) * 8;
}

// One query whose per-(segment, level) hard-leaf outputs would take more than
// kWindowBytes: its other terms run as usual, its hard leaves run in windows
// of consecutive segments of at most kWindowEntries (segment, level) pairs
// (the part path of a query split over GPUs, here one window after another
// on one GPU), and the windows' per-level records are merged in segment order:
// a level's survivors below a window are the carries its leaves lacked.
void merge_hard_part(std::vector<u128> &carry, i128 &H, const HardLevel *rec, uint32_t nlv)
{
    for (uint32_t b = 0; b < nlv; b++) {
        const HardLevel &lv = rec[b];
        if (lv.anchored) {
            carry[b] = (u128)lv.carry0 + lv.count;
        } else {
            H += (i128)carry[b] * lv.msum;
            carry[b] += lv.count;
        }
    }
}

constexpr uint64_t kWindowBytes = 32ull << 30;
constexpr uint64_t kWindowEntries = 1ull << 31;

static void run_hard_windows(cpx_ctx *ctx, const BatchReq &rq, const QD &d, uint32_t threads)
{
    const uint32_t c = rq.c;
    uint64_t y = d.y;
    i128 t[7] = {};
    if (rq.terms & ~(unsigned)TERM_HARD) {
        BatchReq r1 = rq;
        r1.terms = rq.terms & ~(unsigned)TERM_HARD;
        r1.ys = &y;
        r1.out_pi = nullptr;
        r1.out_y = nullptr;
        r1.out_terms = t;
        run_batch(ctx, r1);
        t[5] = t[6] = 0;
    }
    const uint32_t nlv = d.nb - c;
    const uint64_t W = std::max<uint64_t>(1, kWindowEntries / nlv);
    std::vector<HardLevel> rec(nlv);
    std::vector<u128> carry(nlv, 0);
    i128 H = 0;
    for (uint64_t s0 = 0; s0 < d.nseg; s0 += W) {
        i128 th[7] = {};
        BatchReq rh;
        rh.xs = rq.xs;
        rh.ys = &y;
        rh.n = 1;
        rh.c = c;
        rh.terms = TERM_HARD;
        rh.lbits = d.lbits;
        rh.threads = threads;
        rh.seg_lo = s0;
        rh.seg_hi = std::min(d.nseg, s0 + W);
        rh.hard_levels = rec.data();
        rh.out_terms = th;
        rh.wide = rq.wide;
        rh.max_table_n = rq.max_table_n;
        run_batch(ctx, rh);
        H += th[4];
        merge_hard_part(carry, H, rec.data(), nlv);
    }
    t[4] = H;
    if (rq.terms == TERM_PI) {
        t[5] = (i128)count_primes(ctx, 0, y + 1);
        t[6] = t[1] + t[2] + t[3] + t[4] + t[5] - 1 - t[0];
    }
    if (rq.out_pi) rq.out_pi[0] = (u128)t[6];
    if (rq.out_terms)
        for (int k = 0; k < 7; k++) rq.out_terms[k] = t[k];
    if (rq.out_y) rq.out_y[0] = y;
}

// Captures the launches of one batch into a CUDA graph and runs it.  The
// executable graph is kept in the context: a later batch with the same kernel
// sequence only updates its nodes' parameters (grids, pointers) in place, a
// different sequence rebuilds it.
template <class F> static void launch_as_graph(cpx_ctx *ctx, F &&launches)
{
    CPX_CUDA(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
    try {
        launches();
    } catch (...) {
        cudaGraph_t g = nullptr;
        cudaStreamEndCapture(ctx->stream, &g);
        if (g) cudaGraphDestroy(g);
        cudaGetLastError();
        throw;
    }
    cudaGraph_t g = nullptr;
    CPX_CUDA(cudaStreamEndCapture(ctx->stream, &g));
    bool updated = false;
    if (ctx->graph_exec) {
        cudaGraphExecUpdateResultInfo info;
        if (cudaGraphExecUpdate(ctx->graph_exec, g, &info) == cudaSuccess) {
            updated = true;
        } else {
            cudaGetLastError();
            cudaGraphExecDestroy(ctx->graph_exec);
            ctx->graph_exec = nullptr;
        }
    }
    if (!updated) {
        const cudaError_t e = cudaGraphInstantiate(&ctx->graph_exec, g, 0);
        if (e != cudaSuccess) {
            cudaGraphDestroy(g);
            ctx->graph_exec = nullptr;
            check_cuda(e, "cudaGraphInstantiate");
        }
        ctx->graph_builds++;
    } else {
        ctx->graph_updates++;
    }
    cudaGraphDestroy(g);
    CPX_CUDA(cudaGraphLaunch(ctx->graph_exec, ctx->stream));
}

// Runs f(0) .. f(n - 1) on up to 16 host threads (the calling thread
// included); the first exception thrown by any f is rethrown here.
constexpr size_t kPlanBlock = 64;  // queries per planning block
template <class F> static void parallel_blocks(size_t n, F &&f)
{
    const size_t hw = std::max<size_t>(1, std::thread::hardware_concurrency());
    const size_t nt = std::min<size_t>(std::min<size_t>(hw, 16), n);
    if (nt <= 1) {
        for (size_t k = 0; k < n; k++) f(k);
        return;
    }
    std::atomic<size_t> next(0);
    std::exception_ptr err;
    std::mutex em;
    auto worker = [&] {
        try {
            for (;;) {
                const size_t k = next.fetch_add(1);
                if (k >= n) break;
                f(k);
            }
        } catch (...) {
            std::lock_guard<std::mutex> g(em);
            if (!err) err = std::current_exception();
        }
    };
    std::vector<std::thread> th;
    th.reserve(nt - 1);
    for (size_t t = 1; t < nt; t++) th.emplace_back(worker);
    worker();
    for (auto &t : th) t.join();
    if (err) std::rethrow_exception(err);
}

// Roots, y and validity of every query of a request, and the table bounds
// the batch needs (pi table to N, mu/lpf to Y, primes to P, wheel for c).
void compute_needs(const BatchReq &rq, std::vector<QD> &qd, TableNeed &need, bool &wide)
{
    const uint32_t Q = (uint32_t)rq.n;
    const uint32_t c = rq.c;
    const unsigned mask = rq.terms;
    if (c < 1 || c > 8) fail(CPX_EINVAL, "c must be in 1..8");
    qd.assign(Q, QD{});
    // per query in parallel blocks of 256; each block keeps its own maxima
    struct Part {
        uint64_t N = 1 << 16, Y = 0, Pneed = 64;
        bool wide = false, any_direct = false;
    };
    const size_t nblk = (Q + 255) / 256;
    std::vector<Part> parts(nblk);
    auto one = [&](uint32_t i, Part &pt) {
        uint64_t &N = pt.N, &Y = pt.Y, &Pneed = pt.Pneed;
        bool &wide = pt.wide, &any_direct = pt.any_direct;
        QD &d = qd[i];
        memset(&d, 0, sizeof(d));
        const u128 x = rq.xs[i];
        d.x = x;
        d.c = c;
        if (x >> 64) wide = true;
        const uint64_t sx = cpx_isqrt(x), cx = cpx_icbrt(x), r4 = cpx_iroot4(x);
        uint64_t y = rq.ys ? rq.ys[i] : 0;
        if (mask == TERM_PI) {
            if (!y) {
                uint32_t sc = (rq.alpha_scales && rq.alpha_scales[i]) ? rq.alpha_scales[i] : rq.alpha_scale;
                if (!sc && rq.tune) sc = rq.tune[decade_of(x)].alpha_milli;
                if (!rq.alpha_num && sc) {
                    const uint64_t am = std::max<uint64_t>(1000, (uint64_t)alpha_milli(x) * sc / 1000);
                    y = default_y(x, (uint32_t)std::min<uint64_t>(am, 0xFFFFFFFFull), 1000);
                } else {
                    y = default_y(x, rq.alpha_num, rq.alpha_den);
                }
            }
            if (!dr_domain_ok(x, y, c)) {
                if (x >= ((u128)1 << 32)) fail(CPX_EINVAL, "y outside the Deleglise-Rivat domain for this x");
                d.direct = 1;
                d.y = 0;
                any_direct = true;
                N = std::max<uint64_t>(N, (uint64_t)x + 1);
                return;
            }
        } else if (y == 0) {
            fail(CPX_EINVAL, "y must be >= 1");
        }
        if (y >= 0x7FFFFFF0ull && (mask & (TERM_ORD | TERM_HARD)))
            fail(CPX_ERANGE, "y must be below 2^31 for the mu/lpf table");
        const u128 z128 = x / y;
        if (z128 >> 63) fail(CPX_ERANGE, "x / y must be below 2^63");
        d.y = y;
        d.z = (uint64_t)z128;
        d.sx = sx;
        d.cx = cx;
        d.r4 = r4;
        d.tx = cpx_isqrt(z128);
        if (mask & TERM_P2) {
            if (d.z + 1 > rq.p2_table_limit) {
                // P2 by table windows over [sqrt x, z]: the resident table reaches sqrt x
                d.p2win = 1;
                N = std::max<uint64_t>(N, sx + 2);
                Pneed = std::max<uint64_t>(Pneed, cpx_isqrt((u128)d.z) + 2);
            } else {
                N = std::max<uint64_t>(N, std::max(d.z, sx) + 1);
                // the primes p of P2 from the prime list (k_p2_primes)
                if (sx <= kP2PrimeMax) Pneed = std::max<uint64_t>(Pneed, sx + 1);
            }
        }
        if (mask & TERM_TRIV) N = std::max<uint64_t>(N, std::max(y, cx) + 1);
        if (mask & TERM_EASY) N = std::max<uint64_t>(N, std::max(sx, y) + 1);
        if (mask & (TERM_ORD | TERM_HARD)) Y = std::max(Y, y);
        if (mask & TERM_HARD) {
            Pneed = std::max<uint64_t>(Pneed, r4 + 1);
            // carries below p_b^2 come from the pi table; prime m of the sparse levels from its bitmap
            N = std::max<uint64_t>(N, std::max<uint64_t>(r4 * r4 + 2, y + 1));
        }
        if (mask & TERM_EASY) {
            // the p of the easy leaves (p <= icbrt(x)), their sparse q (q <= y) and
            // the u primes of their clustered parts (u <= min(p^2, sqrt(x/p)) <= x^(2/5))
            Pneed = std::max<uint64_t>(Pneed, std::max<uint64_t>(std::max(cx, y) + 1, easy_u_bound(x)));
            Y = std::max(Y, y);
        }
        if (mask == TERM_PI) N = std::max<uint64_t>(N, y + 1);
    };
    parallel_blocks(nblk, [&](size_t k) {
        const uint32_t i1 = (uint32_t)std::min<size_t>(Q, (k + 1) * 256);
        for (uint32_t i = (uint32_t)(k * 256); i < i1; i++) one(i, parts[k]);
    });
    uint64_t N = 1 << 16, Y = 0, Pneed = 64;
    wide = rq.wide;
    bool any_direct = false;
    for (const Part &pt : parts) {
        N = std::max(N, pt.N);
        Y = std::max(Y, pt.Y);
        Pneed = std::max(Pneed, pt.Pneed);
        wide |= pt.wide;
        any_direct |= pt.any_direct;
    }
    if (N > rq.max_table_n) fail(CPX_ERANGE, "pi table bound exceeds the configured limit");
    need.P = std::max<uint64_t>(Pneed, cpx_isqrt(Y + 1) + 2);
    need.N = ((mask & (TERM_P2 | TERM_TRIV | TERM_EASY | TERM_HARD)) || mask == TERM_PI || any_direct) ? N : 0;
    need.Y = Y ? Y + 8 : 0;
    need.c = (mask & TERM_ORD) ? c : 0;
}

bool tables_cover(const cpx_ctx *ctx, const TableNeed &need)
{
    const Tables &tb = ctx->tab;
    if (!tb.P || tb.prm_max < need.P) return false;
    if (need.N && (!tb.T || tb.tab_n < need.N)) return false;
    if (need.Y && (!tb.MU || tb.mu_n < need.Y)) return false;
    if (need.c && (!tb.WH || tb.wh_c != need.c)) return false;
    return true;
}

void grow_tables(cpx_ctx *ctx, const TableNeed &need)
{
    ensure_primes(ctx, need.P);
    if (need.N) ensure_pitable(ctx, need.N);
    if (need.Y) ensure_mulpf(ctx, need.Y);
    if (need.c) ensure_wheel(ctx, need.c);
}


static double ms_since(std::chrono::steady_clock::time_point &t)
{
    const auto now = std::chrono::steady_clock::now();
    const double ms = std::chrono::duration<double, std::milli>(now - t).count();
    t = now;
    return ms;
}

void run_batch(cpx_ctx *ctx, const BatchReq &rq)
{
    const uint32_t Q = (uint32_t)rq.n;
    if (Q == 0) return;
    cpx_batch_stats st = {};
    st.queries = Q;
    auto clk = std::chrono::steady_clock::now();
    const uint32_t c = rq.c;
    if (c < 1 || c > 8) fail(CPX_EINVAL, "c must be in 1..8");
    const unsigned mask = rq.terms;
    if (rq.seg_hi && (Q != 1 || mask != TERM_HARD || !rq.lbits || rq.seg_lo >= rq.seg_hi))
        fail(CPX_EINVAL, "a segment range needs one query, the hard term alone and fixed segment bits");
    // tuned settings: per decade for the plain path (up to 4 queries), the
    // batch entry above that; a request's own settings win
    const bool small = Q <= 4;
    const TuneEntry *tune = (small && ctx->tuned) ? ctx->tune : nullptr;
    const TuneEntry *btune = (!small && ctx->batch_tuned) ? &ctx->batch_tune : nullptr;

    // ---- host planning: roots, y, validity, table bounds
    std::vector<QD> qd;
    TableNeed need;
    bool wide = false;
    std::vector<uint32_t> ascale;
    bool batch_alpha = btune && !rq.alpha_scale && !rq.alpha_num && !rq.alpha_scales && btune->alpha_milli;
replan:  // again without the batch alpha when its shared sieve would not fit (below)
    {
        BatchReq r2 = rq;
        r2.p2_table_limit = ctx->p2_table_limit;
        r2.tune = tune;
        if (batch_alpha) {
            ascale = batch_alpha_scales(rq.xs, Q, btune->alpha_milli, ctx->tuned ? ctx->tune : nullptr,
                                        ctx->batch_alpha_dec);
            r2.alpha_scales = ascale.data();
        }
        compute_needs(r2, qd, need, wide);
    }
    // threads per segment, offload threshold and segment-bit cap: the tuned
    // values (of the largest query's decade for the plain path) unless the
    // request fixes them
    uint32_t threads = rq.threads ? rq.threads : ctx->hard_threads;
    uint64_t offload0 = ctx->hard_offload_min;
    uint32_t lbits_cap = rq.lbits_cap;
    if (tune) {
        u128 xmax = 0;
        for (const QD &d : qd)
            if (!d.direct && d.x > xmax) xmax = d.x;
        const TuneEntry &t = tune[decade_of(xmax)];
        if (!rq.threads && t.threads) threads = t.threads;
        if (t.offload) offload0 = t.offload;
    } else if (btune) {
        if (!rq.threads && btune->threads) threads = btune->threads;
        if (btune->offload) offload0 = btune->offload;
        if (!lbits_cap) lbits_cap = btune->lbits;
    }
    // untuned very large queries (z >= 2^40, about x >= 1e19): 128 threads a
    // segment (four warps over 2^18 odd numbers) visit fewer (warp, level)
    // pairs; on a B200 the hard leaves of pi(1e20) took 6.1 s against 7.9 s
    // with 256
    if (!rq.threads && !ctx->hard_params_set && !btune && !(tune && tune[decade_of(xmax_all(qd))].threads)) {
        uint64_t zmax = 0;
        for (const QD &d : qd)
            if (!d.direct) zmax = std::max(zmax, d.z);
        if (zmax >> 40) threads = 128;
    }
    if (threads != 128 && threads != 256 && threads != 512 && threads != 1024)
        fail(CPX_EINVAL, "hard threads must be 128/256/512/1024");
    // serving lanes run their batches side by side: a 1024-thread sieve block
    // fills an SM and would keep the other lanes' blocks off it
    if (ctx->tables_borrowed) threads = std::min<uint32_t>(threads, 512);
    bool any_p2win = false;
    for (const QD &d : qd) any_p2win |= d.p2win != 0;
    st.roots_ms = ms_since(clk);
    // ---- tables
    if (ctx->tables_borrowed) {
        if (!tables_cover(ctx, need)) fail(CPX_ESTATE, "the shared tables do not cover this batch");
    } else {
        grow_tables(ctx, need);
    }
    const std::vector<uint32_t> &hP = host_primes(ctx);
    st.tables_ms = ms_since(clk);

    // hard leaves: one sieve per query, or (batches) one shared by groups of queries
    std::vector<uint32_t> horder;  // queries with hard leaves, z descending
    bool shared = false;
    uint32_t gsize = 0, sh_lbits = 0;
    if (mask & TERM_HARD) {
        for (uint32_t i = 0; i < Q; i++) {
            QD &d = qd[i];
            if (d.direct) continue;
            d.nb = (uint32_t)host_pi(hP, d.r4);
            if (d.nb > c) horder.push_back(i);
        }
        // x >= 2^64 keeps one sieve per query: the shared sieve's 128-bit
        // kernels are checked against the oracle on x < 2^64 only
        bool any_big = false;
        for (uint32_t i : horder) any_big |= (qd[i].x >> 64) != 0;
        const uint32_t mode = ctx->hard_shared;
        shared = !rq.seg_hi && !rq.hard_levels && !horder.empty() && !any_big &&
                 (mode == 2 || (mode == 1 && !small && horder.size() >= 8));
        if (shared) {
            std::sort(horder.begin(), horder.end(), [&](uint32_t a, uint32_t b) {
                return qd[a].z != qd[b].z ? qd[a].z > qd[b].z : a < b;
            });
            sh_lbits = choose_shared(ctx, qd, horder, threads, rq.lbits, lbits_cap, gsize);
            // the counting sweep keeps 8 bytes per (sub-segment, level) of [0, z_max): above four
            // times the leaf-set budget (16 GiB by default), plan again without the batch alpha
            // (shorter z), else one sieve per query
            if (carry_row_bytes(qd, horder, hP, sh_lbits, threads, c) > 4 * ctx->hard_offload_bytes) {
                if (batch_alpha) {
                    batch_alpha = false;
                    goto replan;
                }
                shared = false;
            }
        }
        if (shared) {
            for (uint32_t i : horder) qd[i].lbits = sh_lbits;
        } else {
            threads = std::min<uint32_t>(threads, 512);  // 1024-thread blocks: the shared sieve only
            choose_lbits(ctx, qd, c, threads, rq.lbits, lbits_cap, tune);
        }
    }

    // P2 walks the prime list when it reaches every query's sqrt x (and the
    // batch has no windowed P2); else pi-table entries of candidates
    bool p2_primes = (mask & TERM_P2) != 0;
    for (uint32_t i = 0; i < Q && p2_primes; i++) {
        const QD &d = qd[i];
        if (!d.direct && d.sx > d.y && (d.p2win || d.sx > kP2PrimeMax || d.sx > tb_prm_max(ctx))) p2_primes = false;
    }

    // ---- units per kernel family (queries planned in parallel blocks)
    std::vector<uint64_t> pre(6 * (size_t)(Q + 1), 0);
    uint64_t *p_ord = pre.data(), *p_p2 = p_ord + (Q + 1), *p_triv = p_p2 + (Q + 1), *p_easy = p_triv + (Q + 1),
             *p_seg = p_easy + (Q + 1), *p_comb = p_seg + (Q + 1);
    std::vector<uint64_t> q_ent(Q, 0);
    const size_t nblk = (Q + kPlanBlock - 1) / kPlanBlock;
    std::vector<std::vector<EasyLvl>> blk_elv(nblk);
    std::vector<uint64_t> blk_ecomp(nblk, 0);
    parallel_blocks(nblk, [&](size_t k) {
        const uint32_t i0 = (uint32_t)(k * kPlanBlock), i1 = (uint32_t)std::min<size_t>(Q, (k + 1) * kPlanBlock);
        std::vector<EasyLvl> &elv = blk_elv[k];
        uint64_t n_ecomp = 0;  // relative to the block
        for (uint32_t i = i0; i < i1; i++) {
            QD &d = qd[i];
            uint64_t n_ord = 0, n_p2 = 0, n_triv = 0, n_easy = 0, n_seg = 0, n_comb = 0;
            if (!d.direct) {
                const u128 x = d.x;
                const uint64_t pc = kSmallPrimes[c];
                if (mask & TERM_ORD) n_ord = ((d.y + 1) / 2 + 3) / 4;
                if ((mask & TERM_P2) && d.sx > d.y && !d.p2win) {
                    if (p2_primes) {
                        d.piy = (uint32_t)host_pi(hP, d.y);
                        n_p2 = host_pi(hP, d.sx) - d.piy;
                    } else {
                        n_p2 = ((d.sx - 1) >> 7) - (d.y >> 7) + 1;
                    }
                }
                if (mask & TERM_TRIV) n_triv = (d.cx > d.tx) ? ((d.cx - 1) >> 7) - (d.tx >> 7) + 1 : 1;
                // primes p_c < p <= icbrt(x) (or <= easy_pmax)
                const uint64_t pe = rq.easy_pmax ? std::min<uint64_t>(d.cx, rq.easy_pmax) : d.cx;
                if ((mask & TERM_EASY) && pe > pc) n_easy = host_pi(hP, pe) - c;
                if (mask & TERM_EASY) {
                    // composite easy leaves: levels b with p_b <= iroot4(x), p_b^2 < y and
                    // max(y/p_b, x/p_b^3) < y
                    const uint64_t nb4 = host_pi(hP, d.r4);
                    for (uint64_t b = c + 1; b <= nb4; b++) {
                        const uint64_t p = hP[b - 1];
                        if (p * p >= d.y) break;
                        const u128 x3 = (x >> 64) ? x / ((u128)p * p * p) : (u128)((uint64_t)x / (p * p * p));
                        uint64_t mlo = d.y / p;
                        if (x3 > (u128)mlo) mlo = x3 >= (u128)d.y ? d.y : (uint64_t)x3;
                        if (mlo >= d.y) continue;
                        const uint64_t mfirst = (mlo + 1) | 1;
                        EasyLvl r;
                        r.q = i;
                        r.b = (uint32_t)b;
                        r.p = (uint32_t)p;
                        r.pad = 0;
                        r.i_lo = (mfirst - 1) / 2;
                        r.i_hi = (d.y - 1) / 2 + 1;
                        if (r.i_lo >= r.i_hi) continue;
                        r.i_base = r.i_lo & ~uint64_t(3);
                        r.unit0 = n_ecomp;
                        n_ecomp += (r.i_hi - r.i_base + 1023) / 1024;
                        elv.push_back(r);
                    }
                }
                if ((mask & TERM_HARD) && d.nb > c && shared) {
                    const uint64_t span = 2ull << d.lbits;
                    d.nseg = (d.z + 1 + span - 1) / span;
                } else if ((mask & TERM_HARD) && d.nb > c) {
                    const uint64_t span = 2ull << d.lbits;
                    d.nseg = (d.z + 1 + span - 1) / span;
                    if (rq.seg_hi) {  // one part of a query split over GPUs
                        d.seg0 = std::min(rq.seg_lo, d.nseg);
                        d.nseg = std::min(rq.seg_hi, d.nseg) - d.seg0;
                    }
                    n_seg = d.nseg;
                    n_comb = d.nb - c;
                    uint64_t ent = 0;
                    for (uint32_t b = c + 1; b <= d.nb; b++)
                        ent += segments_at_level(x, span, hP[b - 1], d.seg0, d.nseg);
                    q_ent[i] = ent;
                }
            }
            p_ord[i + 1] = n_ord;
            p_p2[i + 1] = n_p2;
            p_triv[i + 1] = n_triv;
            p_easy[i + 1] = n_easy;
            p_seg[i + 1] = n_seg;
            p_comb[i + 1] = n_comb;
        }
        blk_ecomp[k] = n_ecomp;
    });
    for (int f = 0; f < 6; f++) {
        uint64_t *a = pre.data() + (size_t)f * (Q + 1);
        for (uint32_t i = 0; i < Q; i++) a[i + 1] += a[i];
    }
    uint64_t hard_entries = 0;
    double hard_bytes = 0.0;  // one pass over the segment bitmap per (segment, level)
    uint32_t lbits_max = 0;
    for (uint32_t i = 0; i < Q; i++) {
        if (!q_ent[i]) continue;
        hard_entries += q_ent[i];
        hard_bytes += (double)q_ent[i] * (double)(1u << qd[i].lbits) / 8.0;
        lbits_max = std::max(lbits_max, qd[i].lbits);
    }
    std::vector<EasyLvl> elv;
    uint64_t n_ecomp = 0;
    for (size_t k = 0; k < nblk; k++) {
        for (EasyLvl r : blk_elv[k]) {
            r.unit0 += n_ecomp;
            elv.push_back(r);
        }
        n_ecomp += blk_ecomp[k];
    }
    if (!lbits_max) lbits_max = 15;
    if (Q == 1 && !shared && (mask & TERM_HARD) && !rq.seg_hi && !rq.hard_levels && !qd[0].direct &&
        hard_entries * 8 > kWindowBytes) {
        run_hard_windows(ctx, rq, qd[0], threads);
        return;
    }

    // ---- the batch-shared sieve: groups, and the carry rows of its counting
    // sweep (row b: the sub-segments of the segments that sieve level b)
    std::vector<HardGroup> groups;
    std::vector<uint64_t> units, lvl_off;
    uint64_t sh_nseg = 0, sh_r4max = 0;
    u128 sh_xmax = 0;
    uint32_t sh_nlv = 0;
    if (shared) {
        const uint64_t span = 2ull << sh_lbits;
        const uint64_t NW = threads / 32;
        for (size_t k = 0; k < horder.size(); k += gsize) {
            HardGroup hg;
            memset(&hg, 0, sizeof hg);
            hg.n = (uint32_t)std::min<size_t>(gsize, horder.size() - k);
            for (uint32_t t = 0; t < hg.n; t++) {
                const QD &d = qd[horder[k + t]];
                hg.q[t] = horder[k + t];
                hg.xmax = std::max(hg.xmax, d.x);
                hg.r4max = std::max(hg.r4max, d.r4);
                hg.nseg = std::max(hg.nseg, d.nseg);
            }
            groups.push_back(hg);
            sh_nseg = std::max(sh_nseg, hg.nseg);
            sh_xmax = std::max(sh_xmax, hg.xmax);
            sh_r4max = std::max(sh_r4max, hg.r4max);
        }
        // units, segment-major: at segment sg the groups with nseg > sg (a
        // prefix: z descending) in blocks of shared_block(sg) consecutive
        // groups, each block sieving the segment once for all of them
        for (uint64_t sg = 0; sg < sh_nseg; sg++) {
            size_t ng = 0;
            while (ng < groups.size() && groups[ng].nseg > sg) ng++;
            const uint32_t G = shared_block(sg);
            for (size_t g = 0; g < ng; g += G) {
                const uint64_t n = std::min<size_t>(G, ng - g);
                units.push_back(sg << 32 | (uint64_t)g << 4 | (n - 1));
            }
        }
        const uint64_t nbm = host_pi(hP, sh_r4max);
        sh_nlv = nbm > c ? (uint32_t)(nbm - c) : 0;
        lvl_off.assign(sh_nlv + 1, 0);
        double ent = 0.0;  // segment-levels sieved: the sweep, then every unit
        for (uint32_t lv = 0; lv < sh_nlv; lv++) {
            const uint64_t n = segments_at_level(sh_xmax, span, hP[c + lv], 0, sh_nseg);
            lvl_off[lv + 1] = lvl_off[lv] + NW * n;
            ent += (double)n;
        }
        // every bound below is at most r4max: count among the first nbm primes
        const auto pend = hP.begin() + std::min<size_t>(hP.size(), nbm + 1);
        for (const uint64_t u : units) {
            // levels the unit sieves: those of its first group (the largest x)
            const HardGroup &hg = groups[(u >> 4) & 0x0FFFFFFF];
            const uint64_t lo = (u >> 32) * span, hi = lo + span;
            uint64_t v = hg.r4max;
            if (lo) {
                const u128 t = (hg.xmax >> 64) ? (hg.xmax - 1) / lo : (u128)((uint64_t)(hg.xmax - 1) / lo);
                v = std::min<uint64_t>(v, cpx_isqrt(t));
            }
            v = std::min<uint64_t>(v, cpx_isqrt((u128)(hi - 1)));
            const uint64_t nb = (uint64_t)(std::upper_bound(hP.begin(), pend, v,
                                                            [](uint64_t a, uint32_t b) { return a < b; }) -
                                           hP.begin());
            if (nb > c) ent += (double)(nb - c);
        }
        hard_bytes = ent * (double)(1ull << sh_lbits) / 8.0;
        lbits_max = sh_lbits;
    }

    // ---- device buffers
    Plan pl;
    pl.Q = Q;
    pl.c = c;
    pl.wide = wide;
    pl.hard_threads = threads;
    pl.lbits_max = lbits_max;
    pl.n_ord = p_ord[Q];
    pl.n_p2 = p_p2[Q];
    pl.p2_primes = p2_primes;
    pl.n_triv = p_triv[Q];
    pl.n_easy = p_easy[Q];
    pl.n_seg = p_seg[Q];
    pl.n_comb = p_comb[Q];
    pl.hard_entries = hard_entries;
    const size_t qd_bytes = sizeof(QD) * Q, pre_bytes = (pre.size() * 8 + 15) & ~size_t(15);
    const size_t elv_bytes = elv.size() * sizeof(EasyLvl);
    const size_t grp_bytes = groups.size() * sizeof(HardGroup);
    const size_t pg_bytes = (units.size() * 8 + 15) & ~size_t(15), lo_bytes = (lvl_off.size() * 8 + 15) & ~size_t(15);
    const bool persist = shared && ctx->hard_persist;
    const size_t stage_bytes = qd_bytes + pre_bytes + elv_bytes + grp_bytes + pg_bytes + lo_bytes;
    const size_t acc_words = (size_t)Q * kAccStride;
    unsigned char *dbuf = (unsigned char *)ctx->b_work[0].get(stage_bytes + acc_words * 8 + 64);
    QD *d_qd = reinterpret_cast<QD *>(dbuf);
    uint64_t *d_pre = reinterpret_cast<uint64_t *>(dbuf + qd_bytes);
    EasyLvl *d_elv = reinterpret_cast<EasyLvl *>(dbuf + qd_bytes + pre_bytes);
    unsigned char *d_sh = dbuf + qd_bytes + pre_bytes + elv_bytes;  // groups, unit offsets, row offsets
    unsigned long long *d_acc = reinterpret_cast<unsigned long long *>(dbuf + stage_bytes);
    pl.elv = d_elv;
    pl.n_elv = (uint32_t)elv.size();
    pl.n_ecomp = n_ecomp;
    pl.qd = d_qd;
    pl.pre_ord = d_pre;
    pl.pre_p2 = d_pre + (Q + 1);
    pl.pre_triv = d_pre + 2 * (Q + 1);
    pl.pre_easy = d_pre + 3 * (Q + 1);
    pl.pre_seg = d_pre + 4 * (Q + 1);
    pl.pre_comb = d_pre + 5 * (Q + 1);
    pl.acc = d_acc;
    pl.ticket = ctx->b_work[1].as<unsigned int>(4);
    if (shared) {
        pl.shared = true;
        pl.sh_lbits = sh_lbits;
        pl.sh_nlv = sh_nlv;
        pl.n_grp = (uint32_t)groups.size();
        pl.sh_nseg = sh_nseg;
        pl.sh_r4max = sh_r4max;
        pl.sh_xmax = sh_xmax;
        pl.n_gunits = units.size();
        pl.n_carry = lvl_off.back();
        pl.grp = reinterpret_cast<const HardGroup *>(d_sh);
        pl.units = reinterpret_cast<const uint64_t *>(d_sh + grp_bytes);
        pl.lvl_off = reinterpret_cast<const uint64_t *>(d_sh + grp_bytes + pg_bytes);
        if (persist) pl.unit_next = d_acc + acc_words;  // zeroed with the accumulators
        pl.carry = ctx->b_work[4].as<uint64_t>(pl.n_carry + 1);
        const size_t ntab = groups.size() * (size_t)sh_nlv * 32, xb = wide ? 16 : 8;
        unsigned char *tab = static_cast<unsigned char *>(ctx->b_work[5].get(ntab * (xb + 8) + 64));
        pl.gxp = tab;
        pl.gae = reinterpret_cast<uint2 *>(tab + ntab * xb);
    }
    if (pl.n_seg || pl.n_gunits) {
        if (!shared) {
            pl.seg_B = ctx->b_work[2].as<uint32_t>(pl.n_seg + 1);
            pl.seg_off = ctx->b_work[3].as<uint64_t>(pl.n_seg + 1);
            pl.hard_cnt = ctx->b_work[4].as<uint32_t>(hard_entries + 1);
            pl.hard_ms = ctx->b_work[5].as<int32_t>(hard_entries + 1);
        }
        // snapshot pool for the heavy (sub-segment, level) leaf sets, counted on
        // the host; the threshold doubles until the pool fits the budget
        const size_t stride = hard_snapshot_stride(lbits_max - (uint32_t)(__builtin_ctz(threads) - 5));
        const uint64_t budget = std::max<uint64_t>(1, ctx->hard_offload_bytes / (stride + sizeof(HardJob)));
        uint64_t thr = offload0, njobs = 0;
        while (thr) {
            std::atomic<uint64_t> total(0);
            parallel_blocks(nblk, [&](size_t k) {
                const size_t i1 = std::min<size_t>(Q, (k + 1) * kPlanBlock);
                for (size_t i = k * kPlanBlock; i < i1 && total.load() <= budget; i++) {
                    const QD &d = qd[i];
                    if (d.direct || d.nb <= c) continue;
                    total += wide ? heavy_leaf_sets<u128>(d, hP, threads, thr, budget + 1)
                                  : heavy_leaf_sets<uint64_t>(d, hP, threads, thr, budget + 1);
                }
            });
            njobs = total.load();
            if (njobs <= budget) break;
            thr = (thr >= (1ull << 40)) ? 0 : 2 * thr;
        }
        pl.offload_min = thr;
        pl.max_jobs = thr ? (uint32_t)std::min<uint64_t>(njobs + 64, 0xFFFFFFF0ull) : 0;
        pl.jobs = ctx->b_jobs.as<HardJob>(pl.max_jobs + 1);
        uint64_t *ctl = ctx->b_jobctl.as<uint64_t>(pl.max_jobs + 4);
        pl.njobs = reinterpret_cast<unsigned int *>(ctl);
        pl.nsnap = reinterpret_cast<unsigned int *>(ctl + 1);
        pl.job_units = ctl + 2;
        pl.snap = static_cast<unsigned char *>(ctx->b_snap.get((pl.max_jobs + 1) * stride));
    }
    if (pl.n_easy) {
        // the chunk offsets, then (up to 1 GiB) the units' plans
        const size_t ob = ((pl.n_easy + 1) * 8 + 63) & ~size_t(63), rb = pl.n_easy * 64;
        const bool with_rec = rb <= (size_t(1) << 30);
        unsigned char *eb = static_cast<unsigned char *>(ctx->b_work[7].get(ob + (with_rec ? rb : 0) + 64));
        pl.easy_off = reinterpret_cast<uint64_t *>(eb);
        pl.easy_rec = with_rec ? eb + ob : nullptr;
    }
    uint32_t n_levels = 0;
    if (rq.hard_levels && !qd[0].direct && qd[0].nb > c) {
        n_levels = qd[0].nb - c;
        pl.hard_levels = ctx->b_levels.as<HardLevel>(n_levels + 1);
        CPX_CUDA(cudaMemsetAsync(pl.hard_levels, 0, n_levels * sizeof(HardLevel), ctx->stream));
    }
    // every buffer the launches touch exists before the first launch (no
    // allocation between kernels, so the sequence can be captured in a graph)
    scan_reserve(ctx, std::max<uint64_t>(std::max<uint64_t>(pl.n_seg, pl.n_easy + 1), (uint64_t)pl.max_jobs + 1));
    pl.time_hard = ctx->timing && !rq.graph;
    if (mask & TERM_HARD) {
        if (shared) prepare_hard_shared(ctx, pl);
        else prepare_hard(ctx, pl);
    }
    u128 *d_out = ctx->b_work[6].as<u128>(Q);

    st.plan_ms = ms_since(clk);
    st.segments = shared ? pl.n_gunits : pl.n_seg;
    st.shared_groups = groups.size();
    st.hard_jobs = pl.max_jobs;
    st.offload_min = pl.offload_min;
    // one staging copy host -> device
    std::vector<unsigned char> stage(stage_bytes);
    memcpy(stage.data(), qd.data(), qd_bytes);
    memcpy(stage.data() + qd_bytes, pre.data(), pre.size() * 8);
    if (elv_bytes) memcpy(stage.data() + qd_bytes + pre_bytes, elv.data(), elv_bytes);
    if (shared) {
        unsigned char *h_sh = stage.data() + qd_bytes + pre_bytes + elv_bytes;
        memcpy(h_sh, groups.data(), grp_bytes);
        memcpy(h_sh + grp_bytes, units.data(), units.size() * 8);
        memcpy(h_sh + grp_bytes + pg_bytes, lvl_off.data(), lvl_off.size() * 8);
    }
    CPX_CUDA(cudaMemcpyAsync(dbuf, stage.data(), stage.size(), cudaMemcpyHostToDevice, ctx->stream));
    CPX_CUDA(cudaMemsetAsync(d_acc, 0, acc_words * 8 + 8, ctx->stream));  // and the unit counter

    // ---- kernels
    auto launch_all = [&] {
        if (mask & TERM_ORD) launch_ordinary(ctx, pl);
        if (mask & TERM_P2) launch_p2(ctx, pl);
        if (mask & TERM_TRIV) launch_trivial(ctx, pl);
        if (mask & TERM_EASY) {
            launch_easy(ctx, pl);
            launch_easy_comp(ctx, pl);
        }
        if (mask & TERM_HARD) {
            if (pl.shared) launch_hard_shared(ctx, pl);
            else launch_hard(ctx, pl);
        }
        if (!any_p2win) launch_finalize(ctx, pl, d_out, mask == TERM_PI);
    };
    ctx->n_span = 0;
    ctx->span_on = ctx->timing && !rq.graph;
    if (ctx->timing) CPX_CUDA(cudaEventRecord(ctx->ev_b0, ctx->stream));
    if (rq.graph && !any_p2win) launch_as_graph(ctx, launch_all);
    else launch_all();
    if (any_p2win) {
        // P2 of the queries beyond the resident table, window by window
        for (uint32_t i = 0; i < Q; i++)
            if (qd[i].p2win) p2_windowed(ctx, qd[i], d_acc + (size_t)i * kAccStride + 2 * ACC_P2, wide);
        launch_finalize(ctx, pl, d_out, mask == TERM_PI);
    }
    if (ctx->timing) CPX_CUDA(cudaEventRecord(ctx->ev_b1, ctx->stream));

    st.launch_ms = ms_since(clk);
    // ---- results
    std::vector<unsigned long long> acc(acc_words);
    CPX_CUDA(cudaMemcpyAsync(acc.data(), d_acc, acc_words * 8, cudaMemcpyDeviceToHost, ctx->stream));
    CPX_CUDA(cudaStreamSynchronize(ctx->stream));
    ctx->last_h2d = stage.size();
    ctx->last_d2h = acc_words * 8;
    st.wait_ms = ms_since(clk);
    ctx->last_stats = st;
    for (uint32_t i = 0; i < Q; i++) {
        const unsigned long long *A = acc.data() + (size_t)i * kAccStride;
        auto rd = [&](int t) { return (i128)(((u128)A[2 * t + 1] << 64) | A[2 * t]); };
        if (rq.out_pi) rq.out_pi[i] = (u128)rd(ACC_PI);
        if (rq.out_terms) {
            i128 *o = rq.out_terms + (size_t)i * 7;
            o[0] = rd(ACC_P2);
            o[1] = rd(ACC_ORD);
            o[2] = rd(ACC_TRIV);
            o[3] = rd(ACC_EASY);
            o[4] = rd(ACC_HARD);
            o[5] = rd(ACC_PIY);
            o[6] = rd(ACC_PI);
        }
        if (rq.out_y) rq.out_y[i] = qd[i].y;
    }
    if (n_levels) {
        CPX_CUDA(cudaMemcpy(rq.hard_levels, pl.hard_levels, n_levels * sizeof(HardLevel), cudaMemcpyDeviceToHost));
    }
    if (ctx->timing) CPX_CUDA(cudaEventElapsedTime(&ctx->last_batch_ms, ctx->ev_b0, ctx->ev_b1));
    finish_spans(ctx);
    if (pl.time_hard && (pl.n_seg || pl.n_gunits)) {
        float ms = 0.f;
        CPX_CUDA(cudaEventElapsedTime(&ms, ctx->ev_hard0, ctx->ev_hard1));
        ctx->last_hard_ms = ms;
        ctx->last_hard_bytes = hard_bytes;
    }
}

}  // namespace cpx
