// serve.cu -- continuous batching of pi(x) requests over resident tables.
//
// No reference counterpart: the reference answers one x per
// deleglise_rivat64/128 object (src/Deleglise-Rivat/deleglise-rivat.cpp:13-80)
// on the default stream.  A server owns `lanes` worker threads; each lane is a
// context of its own (CUDA stream, batch buffers, CUDA graph) whose tables
// point at the tables of the context the server was created from.  A free
// lane takes the waiting requests in arrival order into one batch while they
// fit: at most max_batch queries, covered by the resident tables, and a
// footprint estimate within the lane's share of the free HBM.  Batches of
// different lanes run concurrently on the device, so requests that arrive
// while others are on the GPU start as soon as a lane frees up.  A request
// that needs larger tables waits until every lane is idle; the tables then
// grow once for every waiting request and the lanes see the new pointers.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <deque>
#include <thread>
#include <unordered_map>

#include "driver.h"

using Clock = std::chrono::steady_clock;

namespace {

struct Req {
    uint64_t ticket;
    u128 x;
    Clock::time_point t_arrive;
    cpx::TableNeed need;
    uint64_t foot;  // device bytes the request adds to a batch (estimate)
};

struct Result {
    u128 pi = 0;
    double latency_ms = 0.0;
    int status = CPX_OK;
};

bool covers(const cpx::TableNeed &cap, const cpx::TableNeed &n)
{
    return n.N <= cap.N && n.Y <= cap.Y && n.P <= cap.P && (n.c == 0 || n.c == cap.c);
}

cpx::TableNeed coverage(const cpx_ctx *ctx)
{
    const cpx::Tables &tb = ctx->tab;
    cpx::TableNeed c;
    c.N = tb.T ? tb.tab_n : 0;
    c.Y = tb.MU ? tb.mu_n : 0;
    c.P = tb.P ? tb.prm_max : 0;
    c.c = tb.WH ? tb.wh_c : 0;
    return c;
}

cpx::TableNeed merge(cpx::TableNeed a, const cpx::TableNeed &b)
{
    a.N = std::max(a.N, b.N);
    a.Y = std::max(a.Y, b.Y);
    a.P = std::max(a.P, b.P);
    if (b.c) a.c = b.c;
    return a;
}

}  // namespace

struct cpx_server {
    cpx_ctx *master = nullptr;
    std::vector<cpx_ctx *> lanes;
    std::vector<std::thread> workers;
    cpx_serve_config cfg = {};
    uint64_t lane_budget = 0;

    std::mutex mu;
    std::condition_variable cv_work, cv_idle, cv_done;
    std::deque<Req> pending;
    std::unordered_map<uint64_t, Result> done;
    uint64_t next_ticket = 1;
    bool stop = false, growing = false;
    int busy = 0;
    cpx::TableNeed cap;
    cpx_serve_counters st = {};
    std::string last_error;
};

namespace cpx {

static void run_lane(cpx_server *S, size_t li)
{
    cpx_ctx *L = S->lanes[li];
    const cpx_params &P = S->cfg.params;
    for (;;) {
        std::vector<Req> batch;
        {
            std::unique_lock<std::mutex> lk(S->mu);
            S->cv_work.wait(lk, [&] { return S->stop || (!S->pending.empty() && !S->growing); });
            if (S->pending.empty()) {
                if (S->stop) return;
                continue;
            }
            if (!covers(S->cap, S->pending.front().need)) {
                // grow once for every waiting request, with every lane idle
                S->growing = true;
                S->cv_idle.wait(lk, [&] { return S->busy == 0; });
                TableNeed target = S->cap;
                for (const Req &r : S->pending) target = merge(target, r.need);
                lk.unlock();
                int rc = CPX_OK;
                std::string msg;
                try {
                    std::lock_guard<std::recursive_mutex> g(S->master->mu);
                    CPX_CUDA(cudaSetDevice(S->master->device));
                    grow_tables(S->master, target);
                    CPX_CUDA(cudaStreamSynchronize(S->master->stream));
                } catch (const Error &e) {
                    rc = e.code;
                    msg = e.msg;
                } catch (const std::bad_alloc &) {
                    rc = CPX_EOOM;
                    msg = "host allocation failed";
                }
                lk.lock();
                if (rc == CPX_OK) {
                    for (cpx_ctx *l : S->lanes) l->tab = S->master->tab;
                    S->cap = coverage(S->master);
                    S->st.table_growths++;
                } else {
                    // the requests that needed the growth fail; the others go on
                    S->last_error = msg;
                    for (auto it = S->pending.begin(); it != S->pending.end();) {
                        if (!covers(S->cap, it->need)) {
                            Result &res = S->done[it->ticket];
                            res.status = rc;
                            res.latency_ms =
                                std::chrono::duration<double, std::milli>(Clock::now() - it->t_arrive).count();
                            S->st.failed++;
                            it = S->pending.erase(it);
                        } else {
                            ++it;
                        }
                    }
                    S->cv_done.notify_all();
                }
                S->growing = false;
                S->cv_work.notify_all();
                continue;
            }
            // batch window: under load (another lane busy) wait for a fuller batch
            if (S->busy > 0 && S->cfg.fill_target > 1 && S->pending.size() < S->cfg.fill_target) {
                const auto deadline = S->pending.front().t_arrive + std::chrono::microseconds(S->cfg.window_us);
                S->cv_work.wait_until(lk, deadline, [&] {
                    return S->stop || S->growing || S->busy == 0 || S->pending.size() >= S->cfg.fill_target;
                });
                if (S->pending.empty() || S->growing) continue;
            }
            uint64_t foot = 0;
            while (!S->pending.empty() && batch.size() < S->cfg.max_batch) {
                const Req &r = S->pending.front();
                if (!covers(S->cap, r.need)) break;
                if (!batch.empty() && foot + r.foot > S->lane_budget) break;
                foot += r.foot;
                batch.push_back(r);
                S->pending.pop_front();
            }
            S->busy++;
        }
        // ---- run the batch on this lane's stream
        std::vector<u128> xs(batch.size()), pis(batch.size(), 0);
        for (size_t i = 0; i < batch.size(); i++) xs[i] = batch[i].x;
        int rc = CPX_OK;
        std::string msg;
        const auto t_run = Clock::now();
        try {
            std::lock_guard<std::recursive_mutex> g(L->mu);
            CPX_CUDA(cudaSetDevice(L->device));
            BatchReq rq;
            rq.xs = xs.data();
            rq.n = xs.size();
            rq.c = P.c ? P.c : 6;
            rq.alpha_num = P.alpha_num;
            rq.alpha_den = P.alpha_den;
            rq.lbits = P.hard_log2_bits;
            rq.threads = P.hard_threads;
            rq.wide = (P.flags & CPX_BATCH_WIDE) != 0;
            rq.graph = (P.flags & CPX_BATCH_GRAPH) != 0;
            rq.terms = TERM_PI;
            rq.out_pi = pis.data();
            run_batch(L, rq);
        } catch (const Error &e) {
            rc = e.code;
            msg = e.msg;
        } catch (const std::bad_alloc &) {
            rc = CPX_EOOM;
            msg = "host allocation failed";
        }
        const auto t_end = Clock::now();
        {
            std::lock_guard<std::mutex> lk(S->mu);
            for (size_t i = 0; i < batch.size(); i++) {
                Result &res = S->done[batch[i].ticket];
                res.pi = pis[i];
                res.status = rc;
                res.latency_ms = std::chrono::duration<double, std::milli>(t_end - batch[i].t_arrive).count();
            }
            if (rc != CPX_OK) {
                S->last_error = msg;
                S->st.failed += batch.size();
            }
            S->st.completed += batch.size();
            S->st.batches++;
            S->st.max_batch_seen = std::max<uint64_t>(S->st.max_batch_seen, batch.size());
            S->st.busy_ms += std::chrono::duration<double, std::milli>(t_end - t_run).count();
            S->busy--;
        }
        S->cv_done.notify_all();
        S->cv_idle.notify_all();
        S->cv_work.notify_all();
    }
}

// Admission data of one request: its table bounds and a device footprint
// estimate (per (segment, level) outputs of the hard leaves, 8 bytes each,
// plus the per-query records).  The alpha a lane runs a request with depends
// on its batch: the per-decade tuning in batches of up to 4 queries; above
// that the batch scale, the decade's own batch scale, or the untuned alpha
// (no batch entry, few neighbours without a decade alpha, or a batch planned
// again without the batch alpha).  y and z differ with alpha, so the bounds
// cover every one of them.
static Req make_req(cpx_server *S, u128 x, Clock::time_point t)
{
    const cpx_params &P = S->cfg.params;
    const cpx_ctx *M = S->master;
    BatchReq rq;
    rq.xs = &x;
    rq.n = 1;
    rq.c = P.c ? P.c : 6;
    rq.alpha_num = P.alpha_num;
    rq.alpha_den = P.alpha_den;
    rq.terms = TERM_PI;
    rq.p2_table_limit = M->p2_table_limit;
    rq.tune = M->tuned ? M->tune : nullptr;
    std::vector<QD> qd;
    Req r;
    bool wide = false;
    compute_needs(rq, qd, r.need, wide);
    QD d = qd[0];
    auto also = [&](const BatchReq &rb) {
        std::vector<QD> qb;
        TableNeed nb;
        compute_needs(rb, qb, nb, wide);
        r.need = merge(r.need, nb);
        if (qb[0].z > d.z) d = qb[0];
    };
    if (!P.alpha_num) {
        BatchReq rb = rq;
        rb.tune = nullptr;
        also(rb);  // the untuned alpha
        if (M->batch_tuned && M->batch_tune.alpha_milli) {
            rb.alpha_scale = M->batch_tune.alpha_milli;
            also(rb);
            const uint32_t e = decade_of(x);
            if (e < kTuneDecades && M->batch_alpha_dec[e]) {
                rb.alpha_scale = M->batch_alpha_dec[e];
                also(rb);
            }
        }
    }
    r.x = x;
    r.t_arrive = t;
    uint64_t foot = 4096;
    if (!d.direct && d.r4 > 1) {
        const uint32_t lb = P.hard_log2_bits ? P.hard_log2_bits : S->master->hard_log2_bits;
        const double nseg = (double)d.z / (double)(2ull << lb) + 1.0;
        const double lr = std::log((double)d.r4);
        const double levels = lr > 1.0 ? 1.3 * (double)d.r4 / lr : 1.0;
        foot += (uint64_t)(8.0 * nseg * levels);
    }
    r.foot = foot;
    return r;
}

static uint64_t submit(cpx_server *S, u128 x, Clock::time_point t)
{
    Req r = make_req(S, x, t);
    std::lock_guard<std::mutex> lk(S->mu);
    if (S->stop) fail(CPX_ESTATE, "server is shutting down");
    r.ticket = S->next_ticket++;
    S->pending.push_back(r);
    S->st.submitted++;
    S->cv_work.notify_all();  // a lane in its batch window counts the arrivals
    return r.ticket;
}

static Result wait_for(cpx_server *S, uint64_t ticket)
{
    std::unique_lock<std::mutex> lk(S->mu);
    S->cv_done.wait(lk, [&] { return S->done.count(ticket) != 0; });
    Result r = S->done[ticket];
    S->done.erase(ticket);
    return r;
}

static void shutdown(cpx_server *S)
{
    {
        std::lock_guard<std::mutex> lk(S->mu);
        S->stop = true;
    }
    S->cv_work.notify_all();
    for (auto &t : S->workers)
        if (t.joinable()) t.join();
    S->workers.clear();
    for (cpx_ctx *l : S->lanes) {
        release_context(l);
        delete l;
    }
    S->lanes.clear();
    if (S->master) S->master->server_attached = false;
}

}  // namespace cpx

using namespace cpx;

template <class F> static int srv_guarded(cpx_server *S, F &&f)
{
    if (!S) return CPX_EINVAL;
    try {
        f();
        return CPX_OK;
    } catch (const Error &e) {
        std::lock_guard<std::mutex> lk(S->mu);
        S->last_error = e.msg;
        return e.code;
    } catch (const std::bad_alloc &) {
        std::lock_guard<std::mutex> lk(S->mu);
        S->last_error = "host allocation failed";
        return CPX_EOOM;
    }
}

static u128 U(cpx_u128 v) { return ((u128)v.hi << 64) | v.lo; }
static cpx_u128 C128(u128 v) { return cpx_u128{(uint64_t)v, (uint64_t)(v >> 64)}; }

extern "C" {

int cpx_serve_create(cpx_ctx *ctx, const cpx_serve_config *cfg, cpx_server **out)
{
    if (!ctx || !out) return CPX_EINVAL;
    *out = nullptr;
    cpx_server *S = new (std::nothrow) cpx_server();
    if (!S) return CPX_EOOM;
    try {
        std::lock_guard<std::recursive_mutex> g(ctx->mu);
        if (ctx->server_attached) fail(CPX_ESTATE, "the context already serves another server");
        DeviceGuard dg(ctx->device);
        CPX_CUDA(dg.err);
        if (cfg) S->cfg = *cfg;
        if (!S->cfg.lanes) S->cfg.lanes = 4;
        if (!S->cfg.max_batch) S->cfg.max_batch = 4096;
        if (!(S->cfg.admit_fraction > 0.0)) S->cfg.admit_fraction = 0.5;
        if (!S->cfg.fill_target) S->cfg.fill_target = 64;
        if (!S->cfg.window_us) S->cfg.window_us = 5000;
        if (S->cfg.lanes > 16) fail(CPX_EINVAL, "lanes must be in 1..16");
        if (S->cfg.admit_fraction > 0.95) fail(CPX_EINVAL, "admit_fraction must be in (0, 0.95]");
        if (S->cfg.params.flags & ~(CPX_BATCH_WIDE | CPX_BATCH_GRAPH)) fail(CPX_EINVAL, "unknown cpx_params flag");
        S->master = ctx;
        // tables for the largest x announced up front
        const u128 rx = U(S->cfg.reserve_x);
        if (rx) {
            Req r = make_req(S, rx, Clock::now());
            grow_tables(ctx, r.need);
            CPX_CUDA(cudaStreamSynchronize(ctx->stream));
        } else {
            TableNeed small;
            small.P = 1 << 16;
            small.N = 1 << 20;
            grow_tables(ctx, small);
            CPX_CUDA(cudaStreamSynchronize(ctx->stream));
        }
        S->cap = coverage(ctx);
        size_t fr = 0, tot = 0;
        CPX_CUDA(cudaMemGetInfo(&fr, &tot));
        S->lane_budget = (uint64_t)((double)fr * S->cfg.admit_fraction / S->cfg.lanes);
        for (uint32_t i = 0; i < S->cfg.lanes; i++) {
            cpx_ctx *l = new cpx_ctx();
            l->tables_borrowed = true;
            if (init_context(l, ctx->device) != CPX_OK) {
                release_context(l);
                delete l;
                fail(CPX_ECUDA, "could not create a serving lane");
            }
            l->tab = ctx->tab;
            l->hard_log2_bits = ctx->hard_log2_bits;
            l->hard_threads = ctx->hard_threads;
            l->hard_offload_min = ctx->hard_offload_min;
            l->hard_shared = ctx->hard_shared;
            l->hard_offload_bytes = ctx->hard_offload_bytes;
            for (uint32_t e = 0; e < kTuneDecades; e++) l->tune[e] = ctx->tune[e];
            l->tuned = ctx->tuned;
            l->batch_tune = ctx->batch_tune;
            l->batch_tuned = ctx->batch_tuned;
            for (uint32_t e = 0; e < kTuneDecades; e++) l->batch_alpha_dec[e] = ctx->batch_alpha_dec[e];
            S->lanes.push_back(l);
        }
        ctx->server_attached = true;
        for (size_t i = 0; i < S->lanes.size(); i++) S->workers.emplace_back(run_lane, S, i);
    } catch (const Error &e) {
        ctx->last_error = e.msg;
        shutdown(S);
        delete S;
        return e.code;
    } catch (const std::exception &e) {
        ctx->last_error = e.what();
        shutdown(S);
        delete S;
        return CPX_EOOM;
    }
    *out = S;
    return CPX_OK;
}

int cpx_serve_destroy(cpx_server *S)
{
    if (!S) return CPX_EINVAL;
    shutdown(S);
    delete S;
    return CPX_OK;
}

int cpx_serve_submit(cpx_server *S, cpx_u128 x, uint64_t *ticket)
{
    return srv_guarded(S, [&] {
        const uint64_t t = submit(S, U(x), Clock::now());
        if (ticket) *ticket = t;
    });
}

int cpx_serve_wait(cpx_server *S, uint64_t ticket, cpx_u128 *pi, double *latency_ms)
{
    return srv_guarded(S, [&] {
        {
            std::lock_guard<std::mutex> lk(S->mu);
            if (ticket == 0 || ticket >= S->next_ticket) fail(CPX_EINVAL, "unknown ticket");
        }
        const Result r = wait_for(S, ticket);
        if (pi) *pi = C128(r.pi);
        if (latency_ms) *latency_ms = r.latency_ms;
        if (r.status != CPX_OK) fail(r.status, "request failed: " + S->last_error);
    });
}

int cpx_serve_replay(cpx_server *S, const cpx_u128 *xs, const double *arrival_s, size_t n, cpx_u128 *pi,
                     double *latency_ms)
{
    return srv_guarded(S, [&] {
        if (!xs || !arrival_s || !pi) fail(CPX_EINVAL, "null buffer");
        for (size_t i = 1; i < n; i++)
            if (arrival_s[i] < arrival_s[i - 1]) fail(CPX_EINVAL, "arrival times must be non-decreasing");
        std::vector<uint64_t> tickets(n);
        const Clock::time_point t0 = Clock::now();
        for (size_t i = 0; i < n; i++) {
            const auto t = t0 + std::chrono::duration_cast<Clock::duration>(std::chrono::duration<double>(arrival_s[i]));
            std::this_thread::sleep_until(t);
            tickets[i] = submit(S, U(xs[i]), t);  // latency counts from the scheduled arrival
        }
        int first_bad = CPX_OK;
        for (size_t i = 0; i < n; i++) {
            const Result r = wait_for(S, tickets[i]);
            pi[i] = C128(r.pi);
            if (latency_ms) latency_ms[i] = r.latency_ms;
            if (r.status != CPX_OK && first_bad == CPX_OK) first_bad = r.status;
        }
        if (first_bad != CPX_OK) fail(first_bad, "a replayed request failed: " + S->last_error);
    });
}

int cpx_serve_stats(cpx_server *S, cpx_serve_counters *out)
{
    if (!S || !out) return CPX_EINVAL;
    std::lock_guard<std::mutex> lk(S->mu);
    *out = S->st;
    out->pending = S->pending.size();
    return CPX_OK;
}

const char *cpx_serve_last_error(cpx_server *S)
{
    if (!S) return "null server";
    std::lock_guard<std::mutex> lk(S->mu);
    return S->last_error.c_str();
}

}  // extern "C"
