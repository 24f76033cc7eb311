// cpx_internal.h -- private types shared by the library's translation units.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/cpx.h"
#include "cpx_int.cuh"

namespace cpx {

constexpr int kThreads = 256;
// Prime-table build: one CTA sieves 2^18 odd numbers (4096 table entries).
constexpr uint64_t kTabSegWords = 4096;
constexpr uint64_t kTabSegNumbers = kTabSegWords * 128;

struct Status {
    int code = CPX_OK;
    std::string msg;
};

// Thrown inside the library, caught at the C-ABI boundary.
struct Error {
    int code;
    std::string msg;
};

[[noreturn]] void fail(int code, const std::string &msg);
void check_cuda(cudaError_t e, const char *what);
#define CPX_CUDA(call) ::cpx::check_cuda((call), #call)
#define CPX_LAUNCH(what) ::cpx::check_cuda(cudaGetLastError(), what)

// Grow-only device buffer, allocated and freed in the order of the owning
// context's stream (a free does not wait for the other contexts' work).
struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
    cudaStream_t stream = nullptr;
    void *get(size_t need);
    void release();
    ~DevBuf() { release(); }
    template <class T> T *as(size_t n) { return static_cast<T *>(get(n * sizeof(T))); }
};

// Resident tables.  All sized to the largest request seen; grown on demand.
struct Tables {
    // compressed pi table over [0, tab_n]
    cpx_pient *T = nullptr;
    uint64_t tab_n = 0, tab_words = 0;
    // all primes <= prm_max, ascending (uint32)
    uint32_t *P = nullptr;
    uint64_t prm_n = 0, prm_max = 0;
    // packed mu*lpf for odd n <= mu_n: v = 0 if mu(n) = 0 else mu(n) * lpf(n);
    // n = 1 -> INT32_MAX.  Index (n - 1) / 2.
    int32_t *MU = nullptr;
    uint64_t mu_n = 0;
    // wheel phi table for c: W[k] = phi(2k - 1, c), k <= w_mod / 2
    uint32_t *WH = nullptr;
    uint32_t wh_c = 0;
    uint64_t wh_mod = 0, wh_tot = 0;
    uint64_t version = 0;
};

// tuned settings (0 = the context default): alpha_milli is the alpha scale
// in per mille of the reference alpha(x); lbits caps the segment bits
struct TuneEntry {
    uint32_t alpha_milli, lbits, threads, offload;
    float ms;  // sample time when tuned
};
constexpr uint32_t kTuneDecades = 40;
constexpr uint32_t kBatchEntry = 99;  // decade number of the batch entry in the JSON file
constexpr uint32_t kBatchDecade0 = 100;  // entries 100 + e: the batch alpha scale of the queries of decade e

struct Timer {
    cudaEvent_t a = nullptr, b = nullptr;
};

}  // namespace cpx

struct cpx_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    cpx::Tables tab;
    cpx::DevBuf b_scan[3];   // block sums of the three scan levels
    cpx::DevBuf b_segtot;    // per-segment totals of a table build
    cpx::DevBuf b_small;     // a few words for pi lookups and totals
    cpx::DevBuf b_tmp;       // bootstrap table, wheel flags
    cpx::DevBuf b_win;       // windowed pi tables, mu arrays, phi bitmaps
    cpx::DevBuf b_win2;      // word prefixes of phi bitmaps
    cpx::DevBuf b_work[8];   // term kernels' work arrays
    cpx::DevBuf b_flush;     // L2 flush buffer (bench only)
    cpx::DevBuf b_jobs, b_jobctl, b_snap;  // offloaded hard-leaf sets and their snapshots
    cpx::DevBuf b_levels;                  // per-level records of a part of a split query
    unsigned long long *d_acc = nullptr;  // per-query accumulators (grown)
    size_t acc_cap = 0;
    unsigned long long *h_acc = nullptr;  // pinned mirror
    size_t h_acc_cap = 0;
    std::string last_error;
    std::recursive_mutex mu;
    std::vector<uint32_t> hP;  // host mirror of tab.P (launch planning only)
    uint64_t hP_version = 0;
    bool tables_borrowed = false;  // a serving lane: tab points at the server's tables, never grown here
    bool server_attached = false;  // the context's tables serve a cpx_server
    int sm_count = 148;
    size_t smem_optin = 0;
    size_t smem_per_sm = 0;
    // tuning
    uint32_t hard_log2_bits = 18;  // hard-leaf segment size (odd numbers, bits)
    uint32_t hard_threads = 256;
    bool hard_params_set = false;      // cpx_set_hard_params was called (no size rule then)
    uint32_t hard_offload_min = 1024;  // candidates of a (sub-segment, level) sent to k_hard_leaves
    uint32_t hard_shared = 1;          // batch-shared sieve: 0 never, 1 batches, 2 always
    uint32_t hard_persist = 1;         // shared sieve as a persistent launch over a unit queue
    uint64_t hard_offload_bytes = 4ull << 30;  // snapshot pool budget of one batch
    uint64_t p2_table_limit = 1ull << 36;      // z beyond this: P2 by pi-table windows
    cpx::TuneEntry tune[cpx::kTuneDecades] = {};  // per decade (batches of up to 4 queries)
    bool tuned = false;
    cpx::TuneEntry batch_tune = {};               // larger batches
    bool batch_tuned = false;
    // alpha scale of a batch's queries by decade of x (0: the batch entry's);
    // the tuning file's entries 100 + e
    uint32_t batch_alpha_dec[cpx::kTuneDecades] = {};
    // kernel timing (CUDA events around the hard-leaf sieve)
    bool timing = false;
    cudaEvent_t ev_hard0 = nullptr, ev_hard1 = nullptr;
    float last_hard_ms = 0.f;
    cudaEvent_t ev_b0 = nullptr, ev_b1 = nullptr;  // around a batch's kernels
    cudaEvent_t ev_t0 = nullptr, ev_t1 = nullptr;  // caller stopwatch
    float last_batch_ms = 0.f;
    cudaGraphExec_t graph_exec = nullptr;  // the batch kernels of CPX_BATCH_GRAPH
    uint64_t graph_builds = 0, graph_updates = 0;
    uint64_t last_h2d = 0, last_d2h = 0;  // bytes copied by the last batch
    cpx_batch_stats last_stats = {};      // host phases of the last batch
    double last_hard_bytes = 0.0;
    uint64_t launches = 0;  // kernels launched by this context
    void *noalloc_scratch = nullptr;  // device address of cpx_mutest_noalloc's static array (first call)
    // per-kernel CUDA-event spans of the last timed batch (timing on, not a graph)
    static constexpr int kMaxSpans = 16;
    cudaEvent_t span_ev[2 * kMaxSpans] = {};
    const char *span_name[kMaxSpans] = {};
    float span_ms[kMaxSpans] = {};
    int n_span = 0;
    bool span_on = false;  // spans are being recorded for the current batch
};

namespace cpx {

// ---------------------------------------------------------------- tables
void ensure_primes(cpx_ctx *ctx, uint64_t pmax);
void ensure_pitable(cpx_ctx *ctx, uint64_t nmax);
void ensure_mulpf(cpx_ctx *ctx, uint64_t ymax);
void ensure_wheel(cpx_ctx *ctx, uint32_t c);

// builds a pi table window [128*w0, 128*(w0+nwords)) into T (pre relative to
// the window start, i.e. counts odd primes >= 128*w0), using the resident
// primes (must cover sqrt of the window top).  Returns total odd primes.
uint64_t build_pitable_window(cpx_ctx *ctx, uint64_t w0, uint64_t nwords, cpx_pient *T);

// exclusive scan of n uint64 values in place (device)
void scan_u64(cpx_ctx *ctx, uint64_t *d, uint64_t n);
// grows the scan's block-sum buffers for n values ahead of a graph capture
void scan_reserve(cpx_ctx *ctx, uint64_t n);

// Extract primes from table words [w0, w1) whose value is in [lo, hi).
uint64_t extract_primes_u64(cpx_ctx *ctx, uint64_t lo, uint64_t hi, uint64_t *d_out, uint64_t cap);

// mu / lpf sieve over odd n in [lo, hi), lo even; any of the outputs may be null.
void mulpf_sieve(cpx_ctx *ctx, uint64_t lo, uint64_t hi, int8_t *mu, uint32_t *lpf32,
                 uint64_t *lpf64, int32_t *packed);

// context set-up and tear-down shared by cpx_create/cpx_destroy and the
// serving lanes (a lane with tables_borrowed leaves the tables alone)
int init_context(cpx_ctx *ctx, int device);
void release_context(cpx_ctx *ctx);

// counts launched kernels for the gpu_launches report
inline void note_launch(cpx_ctx *ctx, uint64_t n = 1) { ctx->launches += n; }

// Brackets one kernel launch with CUDA events on the context stream when the
// batch records spans (ctx->span_on); the durations are read once the batch
// has synchronised (finish_spans).
struct KSpan {
    cpx_ctx *c;
    int i = -1;
    KSpan(cpx_ctx *ctx, const char *name) : c(ctx)
    {
        if (!c->span_on || c->n_span >= cpx_ctx::kMaxSpans) return;
        i = c->n_span++;
        c->span_name[i] = name;
        if (!c->span_ev[2 * i]) {
            cudaEventCreate(&c->span_ev[2 * i]);
            cudaEventCreate(&c->span_ev[2 * i + 1]);
        }
        cudaEventRecord(c->span_ev[2 * i], c->stream);
    }
    ~KSpan()
    {
        if (i >= 0) cudaEventRecord(c->span_ev[2 * i + 1], c->stream);
    }
    KSpan(const KSpan &) = delete;
    KSpan &operator=(const KSpan &) = delete;
};
inline void finish_spans(cpx_ctx *c)
{
    for (int i = 0; i < c->n_span; i++) {
        c->span_ms[i] = 0.f;
        cudaEventElapsedTime(&c->span_ms[i], c->span_ev[2 * i], c->span_ev[2 * i + 1]);
    }
    c->span_on = false;
}

// Makes a device current for the lifetime of the guard and gives the caller's
// current device back afterwards (entry points leave the caller's device as
// they found it).
struct DeviceGuard {
    int prev = -1;
    cudaError_t err;
    explicit DeviceGuard(int dev)
    {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        err = cudaSetDevice(dev);
    }
    ~DeviceGuard()
    {
        if (prev >= 0) cudaSetDevice(prev);
    }
    DeviceGuard(const DeviceGuard &) = delete;
    DeviceGuard &operator=(const DeviceGuard &) = delete;
};

}  // namespace cpx
