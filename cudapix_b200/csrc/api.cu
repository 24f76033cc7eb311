// api.cu -- the extern "C" boundary (include/cpx.h).  Every entry point
// catches the library's exceptions and turns them into status codes.
#include <new>

#include "driver.h"
#include "misc.h"

using namespace cpx;

namespace {

u128 U(cpx_u128 v) { return ((u128)v.hi << 64) | v.lo; }
cpx_u128 C128(u128 v) { return cpx_u128{(uint64_t)v, (uint64_t)(v >> 64)}; }
cpx_u128 C128s(i128 v) { return C128((u128)v); }

template <class F> int guarded(cpx_ctx *ctx, F &&f)
{
    if (!ctx) return CPX_EINVAL;
    std::lock_guard<std::recursive_mutex> lk(ctx->mu);
    if (ctx->server_attached) {
        ctx->last_error = "the context serves a cpx_server; destroy the server first";
        return CPX_ESTATE;
    }
    try {
        DeviceGuard dg(ctx->device);
        if (dg.err != cudaSuccess) fail(CPX_ECUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(dg.err));
        f();
        ctx->last_error.clear();
        return CPX_OK;
    } catch (const Error &e) {
        ctx->last_error = e.msg;
        return e.code;
    } catch (const std::bad_alloc &) {
        ctx->last_error = "host allocation failed";
        return CPX_EOOM;
    } catch (const std::exception &e) {
        ctx->last_error = e.what();
        return CPX_EINVAL;
    }
}

// one query through the batch machinery with the chosen term set
void one(cpx_ctx *ctx, u128 x, uint64_t y, uint32_t c, unsigned terms, i128 *t7, uint64_t *y_used = nullptr)
{
    BatchReq rq;
    rq.xs = &x;
    rq.ys = &y;
    rq.n = 1;
    rq.c = c;
    rq.terms = terms;
    rq.out_terms = t7;
    rq.out_y = y_used;
    run_batch(ctx, rq);
}

}  // namespace

namespace cpx {

// every work buffer of a context
template <class F> static void each_buf(cpx_ctx *ctx, F &&f)
{
    for (auto &b : ctx->b_scan) f(b);
    for (auto &b : ctx->b_work) f(b);
    for (DevBuf *b : {&ctx->b_segtot, &ctx->b_small, &ctx->b_tmp, &ctx->b_win, &ctx->b_win2, &ctx->b_flush,
                      &ctx->b_jobs, &ctx->b_jobctl, &ctx->b_snap, &ctx->b_levels})
        f(*b);
}

int init_context(cpx_ctx *ctx, int device)
{
    ctx->device = device;
    DeviceGuard dg(device);
    cudaError_t e = dg.err;
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&ctx->sm_count, cudaDevAttrMultiProcessorCount, device);
    int optin = 0;
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
    int per_sm = 0;
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, device);
    for (cudaEvent_t *ev : {&ctx->ev_hard0, &ctx->ev_hard1, &ctx->ev_b0, &ctx->ev_b1, &ctx->ev_t0, &ctx->ev_t1})
        if (e == cudaSuccess) e = cudaEventCreate(ev);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return CPX_ECUDA;
    }
    ctx->smem_optin = (size_t)optin;
    ctx->smem_per_sm = (size_t)per_sm;
    each_buf(ctx, [&](DevBuf &b) { b.stream = ctx->stream; });
    return CPX_OK;
}

void release_context(cpx_ctx *ctx)
{
    std::lock_guard<std::recursive_mutex> lk(ctx->mu);
    DeviceGuard dg(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    Tables &tb = ctx->tab;
    if (!ctx->tables_borrowed) {
        if (tb.T) cudaFree(tb.T);
        if (tb.P) cudaFree(tb.P);
        if (tb.MU) cudaFree(tb.MU);
        if (tb.WH) cudaFree(tb.WH);
    }
    tb = Tables{};
    each_buf(ctx, [](DevBuf &b) { b.release(); });
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);  // the buffers' stream-ordered frees
    each_buf(ctx, [](DevBuf &b) { b.stream = nullptr; });
    if (ctx->graph_exec) cudaGraphExecDestroy(ctx->graph_exec);
    ctx->graph_exec = nullptr;
    for (cudaEvent_t *ev : {&ctx->ev_hard0, &ctx->ev_hard1, &ctx->ev_b0, &ctx->ev_b1, &ctx->ev_t0, &ctx->ev_t1}) {
        if (*ev) cudaEventDestroy(*ev);
        *ev = nullptr;
    }
    for (cudaEvent_t &ev : ctx->span_ev) {
        if (ev) cudaEventDestroy(ev);
        ev = nullptr;
    }
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    ctx->stream = nullptr;
}

}  // namespace cpx

extern "C" {

const char *cpx_version(void) { return "cudapix_b200 0.1 (sm_100a)"; }

int cpx_create(int device, cpx_ctx **out)
{
    if (!out) return CPX_EINVAL;
    *out = nullptr;
    cpx_ctx *ctx = new (std::nothrow) cpx_ctx();
    if (!ctx) return CPX_EOOM;
    const int rc = init_context(ctx, device);
    if (rc != CPX_OK) {
        release_context(ctx);
        delete ctx;
        return rc;
    }
    *out = ctx;
    return CPX_OK;
}

int cpx_destroy(cpx_ctx *ctx)
{
    if (!ctx) return CPX_EINVAL;
    if (ctx->server_attached) return CPX_ESTATE;
    release_context(ctx);
    delete ctx;
    return CPX_OK;
}

const char *cpx_last_error(cpx_ctx *ctx) { return ctx ? ctx->last_error.c_str() : "null context"; }
void *cpx_stream(cpx_ctx *ctx) { return ctx ? (void *)ctx->stream : nullptr; }
uint64_t cpx_launch_count(cpx_ctx *ctx) { return ctx ? ctx->launches : 0; }
int cpx_sm_count(cpx_ctx *ctx) { return ctx ? ctx->sm_count : 0; }
int cpx_free(void *p) { return cudaFree(p) == cudaSuccess ? CPX_OK : CPX_ECUDA; }

int cpx_device_alloc(size_t bytes, void **p)
{
    if (!p) return CPX_EINVAL;
    cudaError_t e = cudaMalloc(p, bytes);
    if (e == cudaErrorMemoryAllocation) {
        cudaGetLastError();
        return CPX_EOOM;
    }
    return e == cudaSuccess ? CPX_OK : CPX_ECUDA;
}

int cpx_copy_to_host(void *dst, const void *src, size_t bytes)
{
    return cudaMemcpy(dst, src, bytes, cudaMemcpyDeviceToHost) == cudaSuccess ? CPX_OK : CPX_ECUDA;
}

int cpx_copy_to_device(void *dst, const void *src, size_t bytes)
{
    return cudaMemcpy(dst, src, bytes, cudaMemcpyHostToDevice) == cudaSuccess ? CPX_OK : CPX_ECUDA;
}

int cpx_device_count(void)
{
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}

int cpx_set_hard_params(cpx_ctx *ctx, uint32_t log2_bits, uint32_t threads)
{
    return guarded(ctx, [&] {
        if (log2_bits < 15 || log2_bits > 20) fail(CPX_EINVAL, "log2_bits must be in 15..20");
        if (threads != 128 && threads != 256 && threads != 512) fail(CPX_EINVAL, "threads must be 128/256/512");
        if ((1u << log2_bits) < 128u * threads) fail(CPX_EINVAL, "segment smaller than 128 bits per thread");
        ctx->hard_log2_bits = log2_bits;
        ctx->hard_threads = threads;
        ctx->hard_params_set = true;
    });
}

int cpx_set_hard_offload(cpx_ctx *ctx, uint32_t min_candidates)
{
    return guarded(ctx, [&] { ctx->hard_offload_min = min_candidates; });
}

int cpx_set_hard_shared(cpx_ctx *ctx, uint32_t mode)
{
    return guarded(ctx, [&] {
        if (mode > 2) fail(CPX_EINVAL, "shared-sieve mode must be 0, 1 or 2");
        ctx->hard_shared = mode;
    });
}

int cpx_leaf_count(cpx_ctx *ctx, cpx_u128 x, uint64_t y, uint16_t c, cpx_leaf_counts *out)
{
    return guarded(ctx, [&] {
        if (!out) fail(CPX_EINVAL, "null output");
        const u128 xv = U(x);
        uint64_t yy = y ? y : default_y(xv, 0, 0);
        uint64_t v[4];
        leaf_counts(ctx, xv, yy, c ? c : 6, v);
        out->hard = v[0];
        out->easy_composite = v[1];
        out->easy_prime = v[2];
        out->trivial = v[3];
    });
}

// segment bits a forced request gets for the context's threads (choose_lbits)
static uint32_t part_bits(const cpx_ctx *ctx, uint32_t log2_bits)
{
    const uint32_t th = ctx->hard_threads;
    const uint32_t minb = (th >= 512) ? 16 : (th >= 256 ? 15 : 14);
    return std::max(minb, std::min<uint32_t>(log2_bits, 20));
}

int cpx_S2_hard_layout(cpx_ctx *ctx, cpx_u128 x, uint64_t y, uint16_t c, uint32_t log2_bits, uint64_t *nseg,
                       uint32_t *nlevels)
{
    return guarded(ctx, [&] {
        if (!nseg || !nlevels || !y) fail(CPX_EINVAL, "null output or y = 0");
        const u128 xv = U(x);
        const uint64_t z = (uint64_t)(xv / y), r4 = cpx_iroot4(xv);
        const uint32_t cc = c ? c : 6;
        ensure_primes(ctx, r4 + 2);
        const uint64_t nb = host_pi(host_primes(ctx), r4);
        const uint64_t span = 2ull << part_bits(ctx, log2_bits);
        *nseg = (z + 1 + span - 1) / span;
        *nlevels = nb > cc ? (uint32_t)(nb - cc) : 0;
    });
}

int cpx_S2_hard_part(cpx_ctx *ctx, cpx_u128 x, uint64_t y, uint16_t c, uint32_t log2_bits, uint64_t seg_lo,
                     uint64_t seg_hi, cpx_u128 *h_part, cpx_hard_level *levels)
{
    static_assert(sizeof(cpx_hard_level) == sizeof(HardLevel), "level record layout");
    return guarded(ctx, [&] {
        if (!h_part || !levels) fail(CPX_EINVAL, "null output");
        if (!log2_bits) fail(CPX_EINVAL, "log2_bits must be given (the same for every part)");
        u128 xv = U(x);
        uint64_t yv = y;
        i128 t[7] = {};
        BatchReq rq;
        rq.xs = &xv;
        rq.ys = &yv;
        rq.n = 1;
        rq.c = c ? c : 6;
        rq.terms = TERM_HARD;
        rq.lbits = log2_bits;
        rq.threads = ctx->hard_threads;
        rq.seg_lo = seg_lo;
        rq.seg_hi = seg_hi;
        rq.hard_levels = reinterpret_cast<HardLevel *>(levels);
        rq.out_terms = t;
        run_batch(ctx, rq);
        *h_part = C128s(t[4]);
    });
}

int cpx_S2_hard_merge(const cpx_u128 *h, const cpx_hard_level *levels, uint32_t nparts, uint32_t nlevels,
                      cpx_u128 *out)
{
    if (!h || !out || (nlevels && !levels)) return CPX_EINVAL;
    std::vector<u128> carry(nlevels, 0);
    i128 H = 0;
    for (uint32_t k = 0; k < nparts; k++) {
        H += (i128)U(h[k]);
        merge_hard_part(carry, H, reinterpret_cast<const HardLevel *>(levels) + (size_t)k * nlevels, nlevels);
    }
    *out = C128s(H);
    return CPX_OK;
}

int cpx_autotune(cpx_ctx *ctx, uint32_t decade_lo, uint32_t decade_hi, double seconds)
{
    return guarded(ctx, [&] { autotune(ctx, decade_lo, decade_hi, seconds > 0 ? seconds : 1e30); });
}

int cpx_autotune_batch(cpx_ctx *ctx, const cpx_u128 *xs, size_t n)
{
    return guarded(ctx, [&] {
        if (!xs) fail(CPX_EINVAL, "null buffer");
        std::vector<u128> xv(n);
        for (size_t i = 0; i < n; i++) xv[i] = U(xs[i]);
        autotune_batch(ctx, xv.data(), n);
    });
}

int cpx_tune_save(cpx_ctx *ctx, const char *path)
{
    return guarded(ctx, [&] {
        if (!path) fail(CPX_EINVAL, "null path");
        tune_save(ctx, path);
    });
}

int cpx_tune_load(cpx_ctx *ctx, const char *path)
{
    return guarded(ctx, [&] {
        if (!path) fail(CPX_EINVAL, "null path");
        tune_load(ctx, path);
    });
}

int cpx_tune_get(cpx_ctx *ctx, uint32_t decade, cpx_tune_entry *out)
{
    return guarded(ctx, [&] {
        const bool bd = decade >= kBatchDecade0 && decade < kBatchDecade0 + kTuneDecades;
        if (!out || (decade >= kTuneDecades && decade != kBatchEntry && !bd)) fail(CPX_EINVAL, "bad decade or null output");
        const bool b = decade == kBatchEntry || bd;
        TuneEntry t = b ? ctx->batch_tune : ctx->tune[decade];
        bool on = b ? ctx->batch_tuned : ctx->tuned;
        if (bd) {
            t.alpha_milli = ctx->batch_alpha_dec[decade - kBatchDecade0];
            on = on && t.alpha_milli;
        }
        *out = cpx_tune_entry{decade, t.alpha_milli, t.lbits, on ? t.threads : 0, t.offload, t.ms};
    });
}

int cpx_tune_clear(cpx_ctx *ctx)
{
    return guarded(ctx, [&] {
        for (TuneEntry &t : ctx->tune) t = TuneEntry{};
        ctx->tuned = false;
        ctx->batch_tune = TuneEntry{};
        ctx->batch_tuned = false;
        for (uint32_t &a : ctx->batch_alpha_dec) a = 0;
    });
}

int cpx_set_p2_window(cpx_ctx *ctx, uint64_t limit)
{
    return guarded(ctx, [&] {
        if (limit < (1ull << 20)) fail(CPX_EINVAL, "limit must be at least 2^20");
        ctx->p2_table_limit = limit;
    });
}

int cpx_mem_info(cpx_ctx *ctx, uint64_t *free_bytes, uint64_t *total_bytes)
{
    return guarded(ctx, [&] {
        size_t f = 0, t = 0;
        CPX_CUDA(cudaMemGetInfo(&f, &t));
        if (free_bytes) *free_bytes = f;
        if (total_bytes) *total_bytes = t;
    });
}

int cpx_set_timing(cpx_ctx *ctx, int enable)
{
    return guarded(ctx, [&] { ctx->timing = enable != 0; });
}

int cpx_last_batch_ms(cpx_ctx *ctx, float *ms)
{
    return guarded(ctx, [&] { *ms = ctx->last_batch_ms; });
}

int cpx_flush_l2(cpx_ctx *ctx)
{
    return guarded(ctx, [&] {
        const size_t bytes = size_t(256) << 20;
        void *p = ctx->b_flush.get(bytes);
        CPX_CUDA(cudaMemsetAsync(p, (int)(ctx->launches & 0xff), bytes, ctx->stream));
        CPX_CUDA(cudaStreamSynchronize(ctx->stream));
    });
}

int cpx_last_batch_io(cpx_ctx *ctx, uint64_t *h2d_bytes, uint64_t *d2h_bytes)
{
    return guarded(ctx, [&] {
        if (h2d_bytes) *h2d_bytes = ctx->last_h2d;
        if (d2h_bytes) *d2h_bytes = ctx->last_d2h;
    });
}

int cpx_last_batch_stats(cpx_ctx *ctx, cpx_batch_stats *out)
{
    return guarded(ctx, [&] {
        if (!out) fail(CPX_EINVAL, "null output");
        *out = ctx->last_stats;
    });
}

int cpx_timer_start(cpx_ctx *ctx)
{
    return guarded(ctx, [&] { CPX_CUDA(cudaEventRecord(ctx->ev_t0, ctx->stream)); });
}

int cpx_timer_stop(cpx_ctx *ctx, float *ms)
{
    return guarded(ctx, [&] {
        CPX_CUDA(cudaEventRecord(ctx->ev_t1, ctx->stream));
        CPX_CUDA(cudaEventSynchronize(ctx->ev_t1));
        CPX_CUDA(cudaEventElapsedTime(ms, ctx->ev_t0, ctx->ev_t1));
    });
}

int cpx_last_kernel_span(cpx_ctx *ctx, int i, const char **name, float *ms)
{
    return guarded(ctx, [&] {
        if (i < 0 || i >= ctx->n_span) fail(CPX_ERANGE, "no such kernel span");
        if (name) *name = ctx->span_name[i];
        if (ms) *ms = ctx->span_ms[i];
    });
}

int cpx_last_hard_stats(cpx_ctx *ctx, float *ms, double *bytes)
{
    return guarded(ctx, [&] {
        if (ms) *ms = ctx->last_hard_ms;
        if (bytes) *bytes = ctx->last_hard_bytes;
    });
}

int cpx_iroots(cpx_u128 x, uint64_t *sqrt_x, uint64_t *cbrt_x, uint64_t *qrt_x)
{
    const u128 v = U(x);
    if (sqrt_x) *sqrt_x = cpx_isqrt(v);
    if (cbrt_x) *cbrt_x = cpx_icbrt(v);
    if (qrt_x) *qrt_x = cpx_iroot4(v);
    return CPX_OK;
}

int cpx_default_y(cpx_u128 x, uint32_t alpha_num, uint32_t alpha_den, uint64_t *y)
{
    if (!y) return CPX_EINVAL;
    *y = default_y(U(x), alpha_num, alpha_den);
    return CPX_OK;
}

uint32_t cpx_alpha_milli(cpx_u128 x) { return alpha_milli(U(x)); }

// ------------------------------------------------------------------ terms

int cpx_P2_u64(cpx_ctx *ctx, uint64_t x, uint64_t y, uint64_t *out)
{
    return guarded(ctx, [&] {
        i128 t[7];
        one(ctx, x, y, 6, TERM_P2, t);
        *out = (uint64_t)t[0];
    });
}
int cpx_P2_u128(cpx_ctx *ctx, cpx_u128 x, uint64_t y, cpx_u128 *out)
{
    return guarded(ctx, [&] {
        i128 t[7];
        one(ctx, U(x), y, 6, TERM_P2, t);
        *out = C128s(t[0]);
    });
}
int cpx_trivial_u64(cpx_ctx *ctx, uint64_t x, uint64_t y, uint64_t *out)
{
    return guarded(ctx, [&] {
        i128 t[7];
        one(ctx, x, y, 6, TERM_TRIV, t);
        *out = (uint64_t)t[2];
    });
}
int cpx_trivial_u128(cpx_ctx *ctx, cpx_u128 x, uint64_t y, cpx_u128 *out)
{
    return guarded(ctx, [&] {
        i128 t[7];
        one(ctx, U(x), y, 6, TERM_TRIV, t);
        *out = C128s(t[2]);
    });
}
int cpx_ordinary_u64(cpx_ctx *ctx, uint64_t x, uint64_t y, uint16_t c, int64_t *out)
{
    return guarded(ctx, [&] {
        i128 t[7];
        one(ctx, x, y, c, TERM_ORD, t);
        *out = (int64_t)t[1];
    });
}
int cpx_ordinary_u128(cpx_ctx *ctx, cpx_u128 x, uint64_t y, uint16_t c, cpx_u128 *out)
{
    return guarded(ctx, [&] {
        i128 t[7];
        one(ctx, U(x), y, c, TERM_ORD, t);
        *out = C128s(t[1]);
    });
}
int cpx_S2_easy_u64(cpx_ctx *ctx, uint64_t x, uint64_t y, uint16_t c, int64_t *out)
{
    return guarded(ctx, [&] {
        i128 t[7];
        one(ctx, x, y, c, TERM_EASY, t);
        *out = (int64_t)t[3];
    });
}
int cpx_S2_easy_u128(cpx_ctx *ctx, cpx_u128 x, uint64_t y, uint16_t c, cpx_u128 *out)
{
    return guarded(ctx, [&] {
        i128 t[7];
        one(ctx, U(x), y, c, TERM_EASY, t);
        *out = C128s(t[3]);
    });
}
int cpx_S2_hard_u64(cpx_ctx *ctx, uint64_t x, uint64_t y, uint16_t c, int64_t *out)
{
    return guarded(ctx, [&] {
        i128 t[7];
        one(ctx, x, y, c, TERM_HARD, t);
        *out = (int64_t)t[4];
    });
}
int cpx_S2_hard_u128(cpx_ctx *ctx, cpx_u128 x, uint64_t y, uint16_t c, cpx_u128 *out)
{
    return guarded(ctx, [&] {
        i128 t[7];
        one(ctx, U(x), y, c, TERM_HARD, t);
        *out = C128s(t[4]);
    });
}

static void fill_terms(cpx_terms *T, u128 x, uint64_t y, uint32_t c, const i128 *t)
{
    T->P2 = C128s(t[0]);
    T->ordinary = C128s(t[1]);
    T->trivial = C128s(t[2]);
    T->easy = C128s(t[3]);
    T->hard = C128s(t[4]);
    T->pi_y = C128s(t[5]);
    T->pi = C128s(t[6]);
    T->x_lo = (uint64_t)x;
    T->x_hi = (uint64_t)(x >> 64);
    T->y = y;
    T->z = y ? (uint64_t)(x / y) : 0;
    T->c = c;
    T->pad = 0;
}

int cpx_pi_u64(cpx_ctx *ctx, uint64_t x, uint64_t y, uint16_t c, uint64_t *pi, cpx_terms *terms)
{
    return guarded(ctx, [&] {
        i128 t[7];
        uint64_t yu = 0;
        one(ctx, x, y, c ? c : 6, TERM_PI, t, &yu);
        if (pi) *pi = (uint64_t)t[6];
        if (terms) fill_terms(terms, x, yu, c ? c : 6, t);
    });
}

int cpx_gourdon_u64(cpx_ctx *ctx, uint64_t x, uint64_t y, uint16_t c, cpx_gourdon_terms *out)
{
    return guarded(ctx, [&] {
        if (!out) fail(CPX_EINVAL, "null output");
        const uint64_t yu = y ? y : default_y(x, 0, 0);
        i128 t[7];
        gourdon_terms(ctx, x, yu, c ? c : 6, t);
        cpx_u128 *o[7] = {&out->A, &out->B, &out->C, &out->D, &out->phi0, &out->sigma, &out->pi};
        for (int k = 0; k < 7; k++) *o[k] = C128s(t[k]);
        out->x = x;
        out->y = yu;
    });
}

int cpx_pi_u128(cpx_ctx *ctx, cpx_u128 x, uint64_t y, uint16_t c, cpx_u128 *pi, cpx_terms *terms)
{
    return guarded(ctx, [&] {
        i128 t[7];
        uint64_t yu = 0;
        one(ctx, U(x), y, c ? c : 6, TERM_PI, t, &yu);
        if (pi) *pi = C128s(t[6]);
        if (terms) fill_terms(terms, U(x), yu, c ? c : 6, t);
    });
}

static void apply_params(BatchReq &rq, const cpx_params *params)
{
    if (!params) return;
    if (params->flags & ~(CPX_BATCH_WIDE | CPX_BATCH_GRAPH)) fail(CPX_EINVAL, "unknown cpx_params flag");
    rq.c = params->c ? params->c : 6;
    rq.alpha_num = params->alpha_num;
    rq.alpha_den = params->alpha_den;
    rq.lbits = params->hard_log2_bits;
    rq.threads = params->hard_threads;
    rq.wide = (params->flags & CPX_BATCH_WIDE) != 0;
    rq.graph = (params->flags & CPX_BATCH_GRAPH) != 0;
}

int cpx_pi_batch(cpx_ctx *ctx, const cpx_u128 *xs, size_t n, const cpx_params *params, cpx_u128 *out)
{
    return guarded(ctx, [&] {
        if (!xs || !out) fail(CPX_EINVAL, "null buffer");
        std::vector<u128> xv(n);
        for (size_t i = 0; i < n; i++) xv[i] = U(xs[i]);
        std::vector<u128> pv(n);
        BatchReq rq;
        rq.xs = xv.data();
        rq.n = n;
        apply_params(rq, params);
        rq.terms = TERM_PI;
        rq.out_pi = pv.data();
        run_batch(ctx, rq);
        for (size_t i = 0; i < n; i++) out[i] = C128(pv[i]);
    });
}

int cpx_terms_batch(cpx_ctx *ctx, const cpx_u128 *xs, const uint64_t *ys, size_t n, const cpx_params *params,
                    cpx_terms *out)
{
    return guarded(ctx, [&] {
        if (!xs || !out) fail(CPX_EINVAL, "null buffer");
        std::vector<u128> xv(n);
        std::vector<uint64_t> yv(n, 0), yu(n, 0);
        for (size_t i = 0; i < n; i++) {
            xv[i] = U(xs[i]);
            if (ys) yv[i] = ys[i];
        }
        std::vector<i128> t((size_t)n * 7);
        BatchReq rq;
        rq.xs = xv.data();
        rq.ys = yv.data();
        rq.n = n;
        apply_params(rq, params);
        rq.terms = TERM_PI;
        rq.out_terms = t.data();
        rq.out_y = yu.data();
        run_batch(ctx, rq);
        for (size_t i = 0; i < n; i++) fill_terms(out + i, xv[i], yu[i], rq.c, t.data() + 7 * i);
    });
}

// ---------------------------------------------------------- sieves and tables

static void check_range(uint64_t lo, uint64_t hi)
{
    if (lo & 1) fail(CPX_EINVAL, "lo must be even");
    if (hi <= lo) fail(CPX_EINVAL, "hi must exceed lo");
}

int cpx_gen_d_mu(cpx_ctx *ctx, uint64_t lo, uint64_t hi, int8_t **d_mu)
{
    return guarded(ctx, [&] {
        check_range(lo, hi);
        const uint64_t n = (hi - lo) / 2;
        int8_t *p = nullptr;
        CPX_CUDA(cudaMalloc(&p, n + 16));
        try {
            mulpf_sieve(ctx, lo, lo + 2 * n, p, nullptr, nullptr, nullptr);
            CPX_CUDA(cudaStreamSynchronize(ctx->stream));
        } catch (...) {
            cudaFree(p);
            throw;
        }
        *d_mu = p;
    });
}

int cpx_gen_d_lpf32(cpx_ctx *ctx, uint64_t lo, uint64_t hi, uint32_t **d_lpf)
{
    return guarded(ctx, [&] {
        check_range(lo, hi);
        if (hi > (1ull << 32)) fail(CPX_ERANGE, "32-bit lpf needs hi <= 2^32");
        const uint64_t n = (hi - lo) / 2;
        uint32_t *p = nullptr;
        CPX_CUDA(cudaMalloc(&p, (n + 4) * 4));
        try {
            mulpf_sieve(ctx, lo, lo + 2 * n, nullptr, p, nullptr, nullptr);
            CPX_CUDA(cudaStreamSynchronize(ctx->stream));
        } catch (...) {
            cudaFree(p);
            throw;
        }
        *d_lpf = p;
    });
}

int cpx_gen_d_lpf64(cpx_ctx *ctx, uint64_t lo, uint64_t hi, uint64_t **d_lpf)
{
    return guarded(ctx, [&] {
        check_range(lo, hi);
        const uint64_t n = (hi - lo) / 2;
        uint64_t *p = nullptr;
        CPX_CUDA(cudaMalloc(&p, (n + 4) * 8));
        try {
            mulpf_sieve(ctx, lo, lo + 2 * n, nullptr, nullptr, p, nullptr);
            CPX_CUDA(cudaStreamSynchronize(ctx->stream));
        } catch (...) {
            cudaFree(p);
            throw;
        }
        *d_lpf = p;
    });
}

int cpx_gen_d_mu_lpf(cpx_ctx *ctx, uint64_t lo, uint64_t hi, int8_t *d_mu, uint64_t *d_lpf)
{
    return guarded(ctx, [&] {
        check_range(lo, hi);
        mulpf_sieve(ctx, lo, lo + 2 * ((hi - lo) / 2), d_mu, nullptr, d_lpf, nullptr);
        CPX_CUDA(cudaStreamSynchronize(ctx->stream));
    });
}

int cpx_gen_h_mu(cpx_ctx *ctx, uint64_t lo, uint64_t hi, int8_t *h_mu)
{
    return guarded(ctx, [&] {
        check_range(lo, hi);
        const uint64_t n = (hi - lo) / 2;
        int8_t *p = ctx->b_win.as<int8_t>(n + 16);
        mulpf_sieve(ctx, lo, lo + 2 * n, p, nullptr, nullptr, nullptr);
        CPX_CUDA(cudaMemcpyAsync(h_mu, p, n, cudaMemcpyDeviceToHost, ctx->stream));
        CPX_CUDA(cudaStreamSynchronize(ctx->stream));
    });
}

int cpx_gen_h_lpf32(cpx_ctx *ctx, uint64_t lo, uint64_t hi, uint32_t *h_lpf)
{
    return guarded(ctx, [&] {
        check_range(lo, hi);
        if (hi > (1ull << 32)) fail(CPX_ERANGE, "32-bit lpf needs hi <= 2^32");
        const uint64_t n = (hi - lo) / 2;
        uint32_t *p = ctx->b_win.as<uint32_t>(n + 4);
        mulpf_sieve(ctx, lo, lo + 2 * n, nullptr, p, nullptr, nullptr);
        CPX_CUDA(cudaMemcpyAsync(h_lpf, p, n * 4, cudaMemcpyDeviceToHost, ctx->stream));
        CPX_CUDA(cudaStreamSynchronize(ctx->stream));
    });
}

int cpx_mutest(cpx_ctx *ctx, uint64_t top, int64_t *out)
{
    return guarded(ctx, [&] { *out = mutest(ctx, top); });
}

int cpx_pitable(cpx_ctx *ctx, uint64_t hi, uint32_t **d_out)
{
    return guarded(ctx, [&] { *d_out = pitable_dense(ctx, hi); });
}

int cpx_pitable_window(cpx_ctx *ctx, uint64_t base, uint64_t range, uint32_t *d_out, uint64_t *pi_base)
{
    return guarded(ctx, [&] {
        if (!d_out) fail(CPX_EINVAL, "null output");
        pitable_window(ctx, base, range, d_out, pi_base);
    });
}

int cpx_primes(cpx_ctx *ctx, uint64_t lo, uint64_t hi, uint64_t **d_out, uint64_t *count)
{
    return guarded(ctx, [&] {
        uint64_t *p = nullptr;
        const uint64_t n = primes_list(ctx, lo, hi, &p);
        *d_out = p;
        if (count) *count = n;
    });
}

int cpx_count_primes(cpx_ctx *ctx, uint64_t lo, uint64_t hi, uint64_t *count)
{
    return guarded(ctx, [&] { *count = count_primes(ctx, lo, hi); });
}

int cpx_phi(cpx_ctx *ctx, uint64_t x, uint32_t a, uint64_t *out)
{
    return guarded(ctx, [&] { *out = phi_count(ctx, x, a); });
}

int cpx_phi_range(cpx_ctx *ctx, uint32_t num, uint32_t a, uint32_t **d_out)
{
    return guarded(ctx, [&] { *d_out = phi_range(ctx, num, a); });
}

}  // extern "C"

// ------------------------------------------------------------------ Phisieve

struct cpx_phisieve {
    cpx_ctx *ctx = nullptr;
    uint64_t nbits = 0, nwords = 0;
    uint64_t *words = nullptr;
    uint32_t *counts = nullptr;
    uint32_t a = 0;
    uint32_t max_prime = 0;
    bool sieved = false;
};

extern "C" {

int cpx_phisieve_create(cpx_ctx *ctx, uint32_t max_prime, uint32_t bits, cpx_phisieve **out)
{
    return guarded(ctx, [&] {
        if (!out || bits == 0) fail(CPX_EINVAL, "bad Phisieve arguments");
        cpx_phisieve *ps = new cpx_phisieve();
        ps->ctx = ctx;
        ps->nbits = bits;
        ps->nwords = (bits + 63) / 64;
        ps->max_prime = max_prime;
        cudaError_t e = cudaMalloc(&ps->words, ps->nwords * 8);
        if (e == cudaSuccess) e = cudaMalloc(&ps->counts, (size_t)bits * 4);
        if (e != cudaSuccess) {
            cudaFree(ps->words);
            cudaFree(ps->counts);
            delete ps;
            cudaGetLastError();
            fail(CPX_EOOM, "Phisieve allocation failed");
        }
        ensure_primes(ctx, std::max<uint64_t>(max_prime, 64));
        *out = ps;
    });
}

int cpx_phisieve_destroy(cpx_phisieve *ps)
{
    if (!ps) return CPX_EINVAL;
    cudaFree(ps->words);
    cudaFree(ps->counts);
    delete ps;
    return CPX_OK;
}

int cpx_phisieve_first(cpx_phisieve *ps, uint16_t c)
{
    if (!ps) return CPX_EINVAL;
    return guarded(ps->ctx, [&] {
        phi_bits(ps->ctx, ps->nwords, c, ps->words);
        ps->a = c;
        counts_from_bits(ps->ctx, ps->words, ps->nwords, ps->nbits, 0, ps->counts);
        CPX_CUDA(cudaStreamSynchronize(ps->ctx->stream));
        ps->sieved = true;
    });
}

int cpx_phisieve_mark_next(cpx_phisieve *ps)
{
    if (!ps) return CPX_EINVAL;
    return guarded(ps->ctx, [&] {
        if (!ps->sieved) fail(CPX_ESTATE, "call first() before mark_next()");
        Tables &tb = ps->ctx->tab;
        while (ps->a >= tb.prm_n) ensure_primes(ps->ctx, std::max<uint64_t>(tb.prm_max * 2, 1 << 16));
        // next prime p_{a+1} = P[a]
        uint32_t p = 0;
        CPX_CUDA(cudaMemcpy(&p, tb.P + ps->a, 4, cudaMemcpyDeviceToHost));
        if (ps->a == 0) fail(CPX_ESTATE, "the odd-only sieve already excludes 2");
        phisieve_cross(ps->ctx, ps->words, ps->nbits, p);
        CPX_CUDA(cudaStreamSynchronize(ps->ctx->stream));
        ps->a++;
    });
}

int cpx_phisieve_update(cpx_phisieve *ps)
{
    if (!ps) return CPX_EINVAL;
    return guarded(ps->ctx, [&] {
        counts_from_bits(ps->ctx, ps->words, ps->nwords, ps->nbits, 0, ps->counts);
        CPX_CUDA(cudaStreamSynchronize(ps->ctx->stream));
    });
}

int cpx_phisieve_counts(cpx_phisieve *ps, uint32_t **d_counts, uint32_t *a_current)
{
    if (!ps) return CPX_EINVAL;
    if (d_counts) *d_counts = ps->counts;
    if (a_current) *a_current = ps->a;
    return CPX_OK;
}

// mark_next checks the value when it is used (a = 0, or p_{a+1} beyond 32 bits)
int cpx_phisieve_set_a(cpx_phisieve *ps, uint32_t a_current)
{
    if (!ps) return CPX_EINVAL;
    ps->a = a_current;
    return CPX_OK;
}

}  // extern "C"
