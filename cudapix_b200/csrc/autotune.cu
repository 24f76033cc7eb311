// autotune.cu -- tuning of the batch engine, measured on the device.
//
// No reference counterpart (the reference fixes its segment length and block
// shape at compile time, src/sieve/S2_hard_device.cuh:7-22, and chooses alpha
// by a formula, src/main.cpp:128-194).  Candidate settings are timed with
// CUDA events by coordinate descent: the alpha scale (per mille of the
// reference alpha), the cap of the hard-leaf segment bits with the threads per
// segment, the alpha scale again, then the candidate threshold of offloaded
// leaf sets.
// Results are exact under every setting; only the time changes.  Two kinds of
// entries: one per decade of x, tuned on lone queries at the bottom and the
// geometric middle of the decade (the plain path; used by batches of up to
// four queries), and one batch entry tuned on a sample batch (used by larger
// batches: a setting good for a lone query, which must cut its segments small
// to occupy every SM, is not good inside a full batch).  The table persists
// as JSON.
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>

#include "driver.h"

namespace cpx {

uint32_t decade_of(u128 x)
{
    uint32_t e = 0;
    while (x >= 10) {
        x /= 10;
        e++;
    }
    return e;
}

// Times one candidate setting on a batch (one warm run, best of two).
static float time_batch(cpx_ctx *ctx, const std::vector<u128> &xs, uint32_t lb, uint32_t th, uint32_t off,
                        uint32_t ascale)
{
    std::vector<u128> out(xs.size());
    BatchReq rq;
    rq.xs = xs.data();
    rq.n = xs.size();
    rq.c = 6;
    rq.alpha_scale = ascale;
    rq.lbits_cap = lb;
    rq.threads = th;
    rq.out_pi = out.data();
    ctx->hard_offload_min = off;
    run_batch(ctx, rq);  // warm: tables and buffers
    float best = 1e30f;
    for (int k = 0; k < 2; k++) {
        run_batch(ctx, rq);
        best = std::min(best, ctx->last_batch_ms);
    }
    return best;
}

// (segment-bit cap, threads per segment) candidates; 1024 threads only in
// batches that share the sieve (others run them as 512)
static const uint32_t kCand[][2] = {{15, 128}, {16, 256}, {17, 256}, {18, 256}, {18, 512},
                                    {19, 512},  {20, 512}, {19, 1024}, {20, 1024}};

// alpha scales (per mille of the reference alpha; 0 = the reference alpha).
// A batch whose queries share one sieve pays little for a longer sieve
// interval, so its best alpha lies well below the reference's.
static const uint32_t kScales[] = {0, 125, 250, 500, 2000, 4000};

// Coordinate descent; the cost of a setting is the summed time of the sample
// batches (each timed on its own).  Alpha first, then the segment bits with
// the threads, alpha again, then the offload threshold.
static TuneEntry descend(cpx_ctx *ctx, const std::vector<std::vector<u128>> &samples, uint32_t off0)
{
    auto cost = [&](uint32_t lb, uint32_t th, uint32_t off, uint32_t sc) {
        float t = 0.f;
        for (const auto &xs : samples) t += time_batch(ctx, xs, lb, th, off, sc);
        return t;
    };
    TuneEntry b;
    b.lbits = 0;
    b.threads = ctx->hard_threads;
    b.alpha_milli = 0;
    b.offload = off0;
    b.ms = cost(0, b.threads, off0, 0);
    auto alpha_pass = [&] {
        const uint32_t cur = b.alpha_milli;
        for (const uint32_t sc : kScales) {
            if (sc == cur) continue;
            const float ms = cost(b.lbits, b.threads, off0, sc);
            if (ms < b.ms) {
                b.ms = ms;
                b.alpha_milli = sc;
            }
        }
    };
    alpha_pass();
    for (const auto &cd : kCand) {
        const float ms = cost(cd[0], cd[1], off0, b.alpha_milli);
        if (ms < b.ms) {
            b.ms = ms;
            b.lbits = cd[0];
            b.threads = cd[1];
        }
    }
    alpha_pass();
    for (const uint32_t off : {256u, 4096u, 16384u}) {
        const float ms = cost(b.lbits, b.threads, off, b.alpha_milli);
        if (ms < b.ms) {
            b.ms = ms;
            b.offload = off;
        }
    }
    return b;
}

// measures raw settings (no tuning applied) and restores the context after
struct TuneGuard {
    cpx_ctx *ctx;
    bool timing0, tuned0, btuned0;
    uint32_t off0;
    explicit TuneGuard(cpx_ctx *c)
        : ctx(c), timing0(c->timing), tuned0(c->tuned), btuned0(c->batch_tuned), off0(c->hard_offload_min)
    {
        ctx->timing = true;
        ctx->tuned = ctx->batch_tuned = false;
    }
    ~TuneGuard()
    {
        ctx->timing = timing0;
        ctx->hard_offload_min = off0;
        ctx->tuned = tuned0;
        ctx->batch_tuned = btuned0;
    }
};

void autotune(cpx_ctx *ctx, uint32_t e_lo, uint32_t e_hi, double seconds)
{
    if (e_lo < 6 || e_hi > 30 || e_lo > e_hi) fail(CPX_EINVAL, "decades must satisfy 6 <= lo <= hi <= 30");
    TuneEntry found[kTuneDecades] = {};
    {
        TuneGuard g(ctx);
        const auto t0 = std::chrono::steady_clock::now();
        for (uint32_t e = e_lo; e <= e_hi; e++) {
            // two lone queries, at the bottom and the geometric middle of the decade
            const std::vector<std::vector<u128>> samples{{(u128)powl(10.0L, (long double)e)},
                                                         {(u128)powl(10.0L, (long double)e + 0.5L)}};
            found[e] = descend(ctx, samples, g.off0);
            if (std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() > seconds) break;
        }
    }
    for (uint32_t e = e_lo; e <= e_hi; e++)
        if (found[e].threads) ctx->tune[e] = found[e];
    ctx->tuned = true;
}

void autotune_batch(cpx_ctx *ctx, const u128 *xs, size_t n)
{
    if (n < 5) fail(CPX_EINVAL, "a batch sample needs at least 5 queries");
    TuneEntry b;
    {
        TuneGuard g(ctx);
        b = descend(ctx, {std::vector<u128>(xs, xs + n)}, g.off0);
    }
    ctx->batch_tune = b;
    ctx->batch_tuned = true;
}

static void put_entry(FILE *f, bool &first, uint32_t e, const TuneEntry &t)
{
    fprintf(f,
            "%s {\"decade\": %u, \"alpha_scale_milli\": %u, \"log2_bits\": %u, \"threads\": %u, "
            "\"offload_min\": %u, \"ms\": %.9g}",
            first ? "" : ",\n", e, t.alpha_milli, t.lbits, t.threads, t.offload, (double)t.ms);
    first = false;
}

void tune_save(const cpx_ctx *ctx, const char *path)
{
    FILE *f = fopen(path, "w");
    if (!f) fail(CPX_EINVAL, std::string("cannot write ") + path);
    fprintf(f, "{\"format\": \"cudapix_b200 tuning 1\", \"entries\": [\n");
    bool first = true;
    if (ctx->tuned)
        for (uint32_t e = 0; e < kTuneDecades; e++)
            if (ctx->tune[e].threads) put_entry(f, first, e, ctx->tune[e]);
    if (ctx->batch_tuned) {
        put_entry(f, first, kBatchEntry, ctx->batch_tune);
        for (uint32_t e = 0; e < kTuneDecades; e++)
            if (ctx->batch_alpha_dec[e]) {
                TuneEntry t = ctx->batch_tune;
                t.alpha_milli = ctx->batch_alpha_dec[e];
                put_entry(f, first, kBatchDecade0 + e, t);
            }
    }
    fprintf(f, "\n]}\n");
    fclose(f);
}

// Reads the file tune_save writes (one entry object per line, though any
// layout of the same objects reads the same: every "decade" key is parsed).
void tune_load(cpx_ctx *ctx, const char *path)
{
    FILE *f = fopen(path, "r");
    if (!f) fail(CPX_EINVAL, std::string("cannot read ") + path);
    std::string text;
    {
        char buf[4096];
        size_t n;
        while ((n = fread(buf, 1, sizeof buf, f)) > 0) text.append(buf, n);
    }
    fclose(f);
    TuneEntry tab[kTuneDecades] = {}, batch = {};
    uint32_t bdec[kTuneDecades] = {};
    bool any = false, have_batch = false;
    const bool fmt = text.find("cudapix_b200 tuning 1") != std::string::npos;
    for (const char *p = strstr(text.c_str(), "\"decade\""); p; p = strstr(p + 1, "\"decade\"")) {
        unsigned e, am, lb, th, off;
        double ms;
        if (sscanf(p,
                   "\"decade\": %u, \"alpha_scale_milli\": %u, \"log2_bits\": %u, \"threads\": %u, "
                   "\"offload_min\": %u, \"ms\": %lf",
                   &e, &am, &lb, &th, &off, &ms) != 6 ||
            (e >= kTuneDecades && e != kBatchEntry && (e < kBatchDecade0 || e >= kBatchDecade0 + kTuneDecades)) ||
            (th != 128 && th != 256 && th != 512 && th != 1024) ||
            (lb && (lb < 15 || lb > 20)))
            fail(CPX_EINVAL, std::string("malformed tuning entry in ") + path);
        const TuneEntry t{am, lb, th, off, (float)ms};
        if (e == kBatchEntry) {
            batch = t;
            have_batch = true;
        } else if (e >= kBatchDecade0) {
            bdec[e - kBatchDecade0] = am;
        } else {
            tab[e] = t;
            any = true;
        }
    }
    if (!fmt || (!any && !have_batch)) fail(CPX_EINVAL, std::string("no tuning entries in ") + path);
    for (uint32_t e = 0; e < kTuneDecades; e++) ctx->tune[e] = tab[e];
    ctx->tuned = any;
    ctx->batch_tune = batch;
    ctx->batch_tuned = have_batch;
    for (uint32_t e = 0; e < kTuneDecades; e++) ctx->batch_alpha_dec[e] = have_batch ? bdec[e] : 0;
}

}  // namespace cpx
