/*
 * cpx.h -- C ABI of cudapix_b200, a B200 (sm_100a) implementation of the
 * Deleglise-Rivat combinatorial prime count pi(x) with the term split of
 * curtisseizert/CUDApix.
 *
 * Every entry point returns an int status (CPX_OK = 0) and writes results
 * through out-pointers; cpx_last_error() gives the message of the last
 * failure on a context.  Device buffers handed to callers are cudaMalloc'd,
 * so the reference's `cudaFree(ptr)` keeps working; cpx_free() is the same.
 * A context owns one CUDA stream, the resident tables (compressed pi table,
 * prime list, packed mu/lpf array, wheel table) and all scratch; calls on one
 * context are serialised by a mutex.  No call resets the device.
 *
 * Reference interfaces replaced (file:line in curtisseizert/CUDApix):
 *   P2           include/P2.cuh:16-17
 *   S2_trivial   include/trivial.cuh:8,12
 *   Ordinary     include/ordinary.cuh:6-7
 *   Phi          include/phi.cuh:17-36
 *   Phisieve     include/sieve/phisieve_host.cuh:6-40
 *   PiTable / get_d_piTable   include/pitable.cuh:7,12-51
 *   mutest       include/mutest.cuh:3
 *   gen_d_lpf / gen_h_lpf / gen_d_mu / gen_h_mu / gen_d_mu_lpf
 *                include/sieve/lpf_mu.cuh:12-24
 *   S2hardHost::S2hard        include/sieve/S2_hard_host.cuh:35-36
 *   deleglise_rivat64/128::pi_deleglise_rivat
 *                include/Deleglise-Rivat/deleglise-rivat.hpp:28,64
 *   CudaSieve::getDevicePrimes / countPrimes (external CUDASieve, call sites
 *                e.g. src/P2.cu:100,103, src/Deleglise-Rivat/deleglise-rivat.cpp:33-37)
 */
#ifndef CPX_H
#define CPX_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    CPX_OK = 0,
    CPX_EINVAL = 1,   /* argument outside the supported domain */
    CPX_EOOM = 2,     /* device memory exhausted */
    CPX_ECUDA = 3,    /* CUDA runtime error */
    CPX_ETIMEOUT = 4, /* a bounded device wait gave up */
    CPX_ERANGE = 5,   /* result or size beyond a stated limit */
    CPX_ESTATE = 6    /* object used in the wrong state */
};

typedef struct cpx_ctx cpx_ctx;
/* unsigned 128-bit value split in two words */
typedef struct {
    uint64_t lo, hi;
} cpx_u128;

/* All terms of one pi(x) evaluation, signed 128-bit (two's complement in
 * lo/hi).  pi = ordinary + trivial + easy + hard + pi_y - 1 - P2. */
typedef struct {
    cpx_u128 P2, ordinary, trivial, easy, hard, pi_y, pi;
    uint64_t x_lo, x_hi, y, z;
    uint32_t c, pad;
} cpx_terms;

/* ---- context ---------------------------------------------------------- */
int cpx_create(int device, cpx_ctx **out);
int cpx_destroy(cpx_ctx *ctx);
const char *cpx_last_error(cpx_ctx *ctx);
const char *cpx_version(void);
/* the context's cudaStream_t, for callers that time or order work on it */
void *cpx_stream(cpx_ctx *ctx);
/* kernels launched by this context since creation */
uint64_t cpx_launch_count(cpx_ctx *ctx);
/* streaming multiprocessors of the context's device (0 for a null context) */
int cpx_sm_count(cpx_ctx *ctx);
int cpx_free(void *device_ptr);
/* plain device memory helpers for callers without their own CUDA runtime */
int cpx_device_alloc(size_t bytes, void **device_ptr);
int cpx_copy_to_host(void *host_dst, const void *device_src, size_t bytes);
int cpx_copy_to_device(void *device_dst, const void *host_src, size_t bytes);
/* number of CUDA devices visible (0 when there is no GPU) */
int cpx_device_count(void);
/* free and total device memory of the context's device (cudaMemGetInfo) */
int cpx_mem_info(cpx_ctx *ctx, uint64_t *free_bytes, uint64_t *total_bytes);
/* hard-leaf sieve tuning: segment = 2^log2_bits odd numbers (15..20),
 * threads per CTA in {128, 256, 512}. */
int cpx_set_hard_params(cpx_ctx *ctx, uint32_t log2_bits, uint32_t threads);
/* a (sub-segment, level) of the hard-leaf sieve with at least min_candidates
 * candidate m is answered by a separate GPU-wide leaf kernel from a snapshot
 * of the sub-segment; 0 answers every leaf inside the sieve (default 1024) */
int cpx_set_hard_offload(cpx_ctx *ctx, uint32_t min_candidates);
/* Batches share one hard-leaf sieve between their queries: the survivor
 * counts of one sweep give every (sub-segment, level) its carry, and each
 * segment is then sieved once per group of up to 32 queries, answering all
 * their leaves.  mode 0: never (one sieve per query), 1: batches of more than
 * four queries with at least eight hard-leaf queries (default), 2: always.
 * Batches holding an x >= 2^64 keep one sieve per query in every mode.
 * Results are the same in every mode.  No reference counterpart. */
int cpx_set_hard_shared(cpx_ctx *ctx, uint32_t mode);
/* P2 needs pi(x/p) up to z = x/y.  For z above `limit` (default 2^36) the
 * resident pi table stops at sqrt(x) and P2 is summed over pi-table windows
 * of 2^34 integers built one after another (the 128-bit path to 1e20). */
int cpx_set_p2_window(cpx_ctx *ctx, uint64_t limit);
/* time of the last hard-leaf sieve (CUDA events on the context stream) and
 * its algorithmic byte count (one pass over the segment bitmap per active
 * prime per segment). */
int cpx_last_hard_stats(cpx_ctx *ctx, float *ms, double *bytes);
/* Device time of the i-th timed kernel launch of the last batch run with
 * timing on (cpx_set_timing) and not as a graph: *name is the kernel (a
 * static string), *ms its CUDA-event duration on the context stream.  The
 * timed kernels are the dominant ones (k_hard_shared, k_hard, k_easy,
 * k_easy_comp, k_p2, k_sieve_counts, k_ordinary).  CPX_ERANGE past the last. */
int cpx_last_kernel_span(cpx_ctx *ctx, int i, const char **name, float *ms);
int cpx_set_timing(cpx_ctx *ctx, int enable);
/* device time of the last batch's kernels (first launch to last, CUDA events
 * on the context stream); valid when timing is enabled */
int cpx_last_batch_ms(cpx_ctx *ctx, float *ms);
/* bytes the last batch copied host->device and device->host */
int cpx_last_batch_io(cpx_ctx *ctx, uint64_t *h2d_bytes, uint64_t *d2h_bytes);

/* Host-side profile of the last batch (wall clock, milliseconds) and the
 * shape of its hard-leaf work.  No reference counterpart. */
typedef struct {
    double roots_ms;      /* per-query roots, y, validity, table bounds */
    double tables_ms;     /* growing the resident tables (0 when they suffice) */
    double plan_ms;       /* segment sizes, work-unit prefixes, leaf-set count */
    double launch_ms;     /* staging copy and kernel launches (enqueue only) */
    double wait_ms;       /* waiting for the device and reading the results */
    uint64_t queries;
    uint64_t segments;    /* hard-leaf sieve work units (CTAs) */
    uint64_t hard_jobs;   /* leaf-set slots reserved for k_hard_leaves */
    uint64_t offload_min; /* candidate threshold of an offloaded leaf set */
    uint64_t shared_groups; /* query groups sharing a sieve (0: one sieve per query) */
} cpx_batch_stats;
int cpx_last_batch_stats(cpx_ctx *ctx, cpx_batch_stats *out);
/* CUDA-event stopwatch on the context stream: start records an event; stop
 * records another, synchronises and returns the elapsed milliseconds */
int cpx_timer_start(cpx_ctx *ctx);
int cpx_timer_stop(cpx_ctx *ctx, float *ms);
/* overwrite a device buffer larger than L2 (256 MiB) on the context stream,
 * so that the next timed call starts with a cold L2 */
int cpx_flush_l2(cpx_ctx *ctx);

/* ---- parameters (host, exact integer) ---------------------------------- */
int cpx_iroots(cpx_u128 x, uint64_t *sqrt_x, uint64_t *cbrt_x, uint64_t *qrt_x);
/* y = floor(alpha * icbrt(x)) for alpha = num/den (num = 0: the reference's
 * alpha(x)), clamped to [icbrt(x), isqrt(x) - 1] (src/main.cpp:59-64). */
int cpx_default_y(cpx_u128 x, uint32_t alpha_num, uint32_t alpha_den, uint64_t *y);
/* alpha(x) of the reference (src/main.cpp:128-194) scaled by 1000; only
 * chooses y, never enters a count. */
uint32_t cpx_alpha_milli(cpx_u128 x);

/* ---- terms -------------------------------------------------------------- */
/* P2(x, y) = sum_{y < p <= sqrt x} [pi(x/p) - pi(p) + 1]      (src/P2.cu:99) */
int cpx_P2_u64(cpx_ctx *ctx, uint64_t x, uint64_t y, uint64_t *out);
int cpx_P2_u128(cpx_ctx *ctx, cpx_u128 x, uint64_t y, cpx_u128 *out);
/* trivial leaves S1 + U                                    (src/trivial.cu:31) */
int cpx_trivial_u64(cpx_ctx *ctx, uint64_t x, uint64_t y, uint64_t *out);
int cpx_trivial_u128(cpx_ctx *ctx, cpx_u128 x, uint64_t y, cpx_u128 *out);
/* ordinary leaves sum_{n <= y, lpf(n) > p_c} mu(n) phi(x/n, c), 1 <= c <= 8
 *                                                         (src/ordinary.cu:33) */
int cpx_ordinary_u64(cpx_ctx *ctx, uint64_t x, uint64_t y, uint16_t c, int64_t *out);
int cpx_ordinary_u128(cpx_ctx *ctx, cpx_u128 x, uint64_t y, uint16_t c, cpx_u128 *out);
/* easy special leaves: the non-trivial leaves (b > c, m) with
 * u = x/(p_b m) < p_b^2, whose value -mu(m) phi(u, b-1) is
 * -mu(m) (pi(u) - b + 2): prime m = q for p_b > iroot4(x) (max(p, y/p) < q <=
 * min(y, x/p^2)) and every m > x/p_b^3 for p_b <= iroot4(x) */
int cpx_S2_easy_u64(cpx_ctx *ctx, uint64_t x, uint64_t y, uint16_t c, int64_t *out);
int cpx_S2_easy_u128(cpx_ctx *ctx, cpx_u128 x, uint64_t y, uint16_t c, cpx_u128 *out);
/* hard special leaves: p_b <= iroot4(x), b > c, m <= x/p_b^3 (u >= p_b^2),
 * by the segmented phi sieve               (src/sieve/S2_hard_host.cu:172) */
int cpx_S2_hard_u64(cpx_ctx *ctx, uint64_t x, uint64_t y, uint16_t c, int64_t *out);
int cpx_S2_hard_u128(cpx_ctx *ctx, cpx_u128 x, uint64_t y, uint16_t c, cpx_u128 *out);
/* pi(x) by the term identity; terms may be NULL.  y = 0 picks the default
 * y rule; the DR domain needs icbrt(x) <= y < isqrt(x); smaller x is counted
 * directly.                   (src/Deleglise-Rivat/deleglise-rivat.cpp:50-80) */
int cpx_pi_u64(cpx_ctx *ctx, uint64_t x, uint64_t y, uint16_t c, uint64_t *pi, cpx_terms *terms);
int cpx_pi_u128(cpx_ctx *ctx, cpx_u128 x, uint64_t y, uint16_t c, cpx_u128 *pi, cpx_terms *terms);
/* pi(x) through Gourdon's decomposition, the terms of the reference's
 * GourdonVariant64 (include/Gourdon/gourdonvariant.hpp:7-56; A: src/Gourdon/A2.cu,
 * B: B.cu, C: C.cu, D = S2hard (gourdonvariant.cpp:61), Phi0: phi_0.cpp,
 * Sigma: sigma_cpu.cpp): pi = A - B + C + D + phi0 + sigma, every term signed
 * 128-bit (two's complement).  x < 2^64; y = 0 picks the default y rule; the
 * domain is icbrt(x) <= y < isqrt(x).  x* = max(iroot4(x), x/y^2) (the
 * reference's x* = iroot4(x) is exact only for y >= ~x^(3/8)). */
typedef struct {
    cpx_u128 A, B, C, D, phi0, sigma, pi;
    uint64_t x, y;
} cpx_gourdon_terms;
int cpx_gourdon_u64(cpx_ctx *ctx, uint64_t x, uint64_t y, uint16_t c, cpx_gourdon_terms *out);

/* ---- sieves and tables -------------------------------------------------- */
/* mu(n) and lpf(n) for odd n = lo + 2i + 1, i < (hi - lo) / 2, lo even.
 * lpf(1) = 0xFFFFFFFF; lpf(p) = p.  Outputs are cudaMalloc'd, caller frees.
 *                                              (src/sieve/lpf_mu.cu:199-302) */
int cpx_gen_d_mu(cpx_ctx *ctx, uint64_t lo, uint64_t hi, int8_t **d_mu);
int cpx_gen_d_lpf32(cpx_ctx *ctx, uint64_t lo, uint64_t hi, uint32_t **d_lpf);
int cpx_gen_d_lpf64(cpx_ctx *ctx, uint64_t lo, uint64_t hi, uint64_t **d_lpf);
int cpx_gen_d_mu_lpf(cpx_ctx *ctx, uint64_t lo, uint64_t hi, int8_t *d_mu, uint64_t *d_lpf);
/* host copies into caller buffers of (hi - lo) / 2 entries */
int cpx_gen_h_mu(cpx_ctx *ctx, uint64_t lo, uint64_t hi, int8_t *h_mu);
int cpx_gen_h_lpf32(cpx_ctx *ctx, uint64_t lo, uint64_t hi, uint32_t *h_lpf);
/* Mertens sum over 1 <= n < top                              (src/mutest.cu:6) */
int cpx_mutest(cpx_ctx *ctx, uint64_t top, int64_t *out);
/* The same Mertens sum without allocating any device memory; no counterpart
 * in the reference.  For callers that cannot call cudaMalloc (their device
 * memory belongs to another allocator, or cudaMalloc/cudaFree would
 * synchronise a latency-critical path).  Scratch lives in one file-scope
 * static device array of 16 MiB + 16 KiB that every GPU loading the library
 * holds until exit; top must be <= 33554432 (CPX_ERANGE otherwise).  The
 * first call on a context looks up the array's device address and keeps it
 * in the context, so make it before any stream capture on that context; after
 * a cudaDeviceReset, create new contexts (a reset also destroys their streams
 * and tables).  Calls share the array: calls that overlap on the GPU race.
 * Uses the context's stream and device; the caller's current device is left
 * as it was. */
int cpx_mutest_noalloc(cpx_ctx *ctx, uint64_t top, int64_t *out);
/* dense pi table of get_d_piTable: out[k] = pi(2k - 1), k < hi / 2, hi < 2^32
 *                                                          (src/pitable.cu:10) */
int cpx_pitable(cpx_ctx *ctx, uint64_t hi, uint32_t **d_out);
/* windowed table of PiTable: out[k] = pi(base + 2k - 1) - pi(base - 1) for
 * k < range/2 + 2 into a caller buffer; *pi_base = pi(base - 1).  base even.
 *                                                      (src/pitable.cu:27-218) */
int cpx_pitable_window(cpx_ctx *ctx, uint64_t base, uint64_t range, uint32_t *d_out,
                       uint64_t *pi_base);
/* primes in [lo, hi) (CudaSieve::getDevicePrimes); cudaMalloc'd output */
int cpx_primes(cpx_ctx *ctx, uint64_t lo, uint64_t hi, uint64_t **d_out, uint64_t *count);
/* number of primes in [lo, hi) (CudaSieve::countPrimes) */
int cpx_count_primes(cpx_ctx *ctx, uint64_t lo, uint64_t hi, uint64_t *count);
/* phi(x, a): #{1 <= n <= x : no prime factor among the first a primes}
 *                                                             (src/phi.cu:42) */
int cpx_phi(cpx_ctx *ctx, uint64_t x, uint32_t a, uint64_t *out);
/* Phi::generateRange: out[i] = phi(2i + 1, a) for i < num/2 (cudaMalloc'd)
 *                                                             (src/phi.cu:75) */
int cpx_phi_range(cpx_ctx *ctx, uint32_t num, uint32_t a, uint32_t **d_out);

/* Phisieve: odd-only bit sieve of 'bits' bits over [0, 2*bits) with a count
 * table counts[i] = phi(2i - 1, a) (exclusive scan of the bits), where a is
 * the number of primes sieved so far.     (src/sieve/phisieve_host.cu:12-89) */
typedef struct cpx_phisieve cpx_phisieve;
int cpx_phisieve_create(cpx_ctx *ctx, uint32_t max_prime, uint32_t bits, cpx_phisieve **out);
int cpx_phisieve_destroy(cpx_phisieve *ps);
int cpx_phisieve_first(cpx_phisieve *ps, uint16_t c);
int cpx_phisieve_mark_next(cpx_phisieve *ps);
int cpx_phisieve_update(cpx_phisieve *ps);
int cpx_phisieve_counts(cpx_phisieve *ps, uint32_t **d_counts, uint32_t *a_current);
/* Phisieve::set_a_current (include/sieve/phisieve_host.cuh:37): the next
 * mark_next crosses off p_{a+1}; the bitmap is left as it is. */
int cpx_phisieve_set_a(cpx_phisieve *ps, uint32_t a_current);

/* ---- batched and served evaluation -------------------------------------- */
/* cpx_params.flags */
#define CPX_BATCH_WIDE 1u  /* 128-bit kernels for every query, also when all x < 2^64 */
#define CPX_BATCH_GRAPH 2u /* run the batch's kernels as one CUDA graph launch (the
                              graph is kept in the context and updated in place) */

typedef struct {
    uint32_t alpha_num, alpha_den; /* y rule; 0/0 = reference alpha(x) */
    uint16_t c;                    /* pre-sieve primes, default 6 */
    uint16_t flags;                /* CPX_BATCH_* */
    uint32_t hard_log2_bits;       /* 0 = context default */
    uint32_t hard_threads;         /* 0 = context default */
} cpx_params;

/* pi(x_i) for n queries in one batched device pass over shared tables sized
 * to the largest query.  out[i] = pi(x_i).  No reference counterpart: the
 * reference evaluates one x per deleglise_rivat64/128 object
 * (src/deleglise-rivat.cpp:13-80). */
int cpx_pi_batch(cpx_ctx *ctx, const cpx_u128 *xs, size_t n, const cpx_params *params,
                 cpx_u128 *out);

/* ---- one query split over GPUs (hard leaves) -----------------------------
 * The hard-leaf sieve runs over segments 0 .. nseg-1 of 2^log2_bits odd
 * numbers (cpx_S2_hard_layout).  Each GPU takes a contiguous range
 * [seg_lo, seg_hi) with cpx_S2_hard_part: its local hard sum (carries from
 * below its range taken as 0 unless the level starts inside it) and, per
 * level b = c+1 .. pi(x^(1/4)), the survivors of level b-1 over its
 * segments, Sum(-mu) of its leaves, and the start carry when the level's
 * first segment is in the range.  One exchange of those records (an
 * all-gather) and cpx_S2_hard_merge, a host-only sum over the parts in
 * segment order, give S2_hard(x, y, c).  Every part must use the same
 * log2_bits and the context's threads per segment.  The plan of the
 * reference's multi-GPU notes; the reference itself runs on one GPU. */
typedef struct {
    uint64_t count;     /* survivors of level b-1 in the part's segments */
    int64_t msum;       /* Sum(-mu(m)) of the part's leaves of level b */
    uint64_t carry0;    /* start carry of the level when anchored */
    uint32_t anchored;  /* the level's first sieved segment lies in the part */
    uint32_t pad;
} cpx_hard_level;
int cpx_S2_hard_layout(cpx_ctx *ctx, cpx_u128 x, uint64_t y, uint16_t c, uint32_t log2_bits, uint64_t *nseg,
                       uint32_t *nlevels);
int cpx_S2_hard_part(cpx_ctx *ctx, cpx_u128 x, uint64_t y, uint16_t c, uint32_t log2_bits, uint64_t seg_lo,
                     uint64_t seg_hi, cpx_u128 *h_part, cpx_hard_level *levels);
/* parts[k] = (h[k], levels[k * nlevels .. ]) for ranges in segment order */
int cpx_S2_hard_merge(const cpx_u128 *h, const cpx_hard_level *levels, uint32_t nparts, uint32_t nlevels,
                      cpx_u128 *out);

/* ---- autotuning ---------------------------------------------------------
 * Candidate settings are timed on the device by coordinate descent: the cap
 * of the hard-leaf segment bits with the threads per segment, then the alpha
 * scale (per mille of the reference alpha(x)), then the offload threshold.
 * cpx_autotune tunes each decade of x in [decade_lo, decade_hi] (6..30) on
 * lone queries at 10^e and 10^(e+1/2): the plain path, applied to
 * batches of up to four queries (threads and offload of the largest query's
 * decade); it stops after the decade that passes `seconds` (0: no limit).
 * cpx_autotune_batch tunes one entry on a sample batch (>= 5 queries),
 * applied to larger batches.  Settings a request fixes win.  Results never
 * change; only the time does.  cpx_tune_get(ctx, 99, ...) reads the batch
 * entry.  No reference counterpart (its segment length and block shape are
 * fixed at compile time, src/sieve/S2_hard_device.cuh:7-22, and its alpha is
 * a formula, src/main.cpp:128-194). */
typedef struct {
    uint32_t decade;             /* 99: the batch entry */
    uint32_t alpha_scale_milli;  /* per mille of the reference alpha; 0 = 1000 */
    uint32_t log2_bits;          /* segment-bit cap; 0 = context default */
    uint32_t threads;            /* 0: not tuned */
    uint32_t offload_min;
    float ms;                    /* sample time */
} cpx_tune_entry;
int cpx_autotune(cpx_ctx *ctx, uint32_t decade_lo, uint32_t decade_hi, double seconds);
int cpx_autotune_batch(cpx_ctx *ctx, const cpx_u128 *xs, size_t n);
int cpx_tune_save(cpx_ctx *ctx, const char *path);  /* JSON */
int cpx_tune_load(cpx_ctx *ctx, const char *path);
int cpx_tune_get(cpx_ctx *ctx, uint32_t decade, cpx_tune_entry *out);
int cpx_tune_clear(cpx_ctx *ctx);

/* Exact special-leaf counts of pi(x) with y (0: the y rule), in this
 * library's split, u = x/(p_b m): trivial u < p_b; easy p_b <= u < p_b^2
 * (prime m, composite m); hard u >= p_b^2.  Replaces the leaf-count
 * estimates of src/leafcount.cpp:12-202. */
typedef struct {
    uint64_t hard, easy_composite, easy_prime, trivial;
} cpx_leaf_counts;
int cpx_leaf_count(cpx_ctx *ctx, cpx_u128 x, uint64_t y, uint16_t c, cpx_leaf_counts *out);

/* ---- serving: continuous batching over resident tables -------------------
 * A server owns `lanes` worker threads, each with its own CUDA stream, batch
 * buffers and graph; all lanes share the tables of the context the server is
 * created from (that context answers no other call while the server exists:
 * CPX_ESTATE).  A free lane takes the waiting requests in arrival order into
 * one batch while they fit: at most max_batch queries, covered by the
 * resident tables, and a summed footprint estimate within admit_fraction of
 * the free HBM (measured at creation) divided among the lanes.  Batches of
 * different lanes run concurrently on the device.  A request that needs
 * larger tables waits until every lane is idle; the tables then grow once for
 * all waiting requests.  Latencies run from arrival (submit, or the scheduled
 * arrival of a replay) to the moment the batch's results are on the host.
 * No reference counterpart: the reference answers one x per
 * deleglise_rivat64/128 object (src/Deleglise-Rivat/deleglise-rivat.cpp:13-80). */
typedef struct cpx_server cpx_server;
typedef struct {
    uint32_t lanes;         /* worker lanes (streams), 1..16; 0 = 4 */
    uint32_t max_batch;     /* queries per batch; 0 = 4096 */
    double admit_fraction;  /* share of free HBM for batch buffers, (0, 0.95]; 0 = 0.5 */
    cpx_u128 reserve_x;     /* grow the tables for x up to this at creation (0: on demand) */
    cpx_params params;      /* y rule, c, hard-leaf tuning, CPX_BATCH_* flags */
    /* Batch window: a lane that frees up while other lanes still run batches
     * waits until fill_target requests are pending, or until the oldest has
     * waited window_us, so that requests arriving under load share a batch
     * (and its hard-leaf sieve); with every lane idle it starts at once.
     * fill_target 0 = 64; window_us 0 = 5000; fill_target 1 = no window. */
    uint32_t fill_target;
    uint32_t window_us;
} cpx_serve_config;
typedef struct {
    uint64_t submitted, completed, failed, pending;
    uint64_t batches, max_batch_seen, table_growths;
    double busy_ms;         /* summed lane time spent in batches */
} cpx_serve_counters;
int cpx_serve_create(cpx_ctx *ctx, const cpx_serve_config *cfg, cpx_server **out);
/* waits for every admitted request, then stops the lanes */
int cpx_serve_destroy(cpx_server *srv);
int cpx_serve_submit(cpx_server *srv, cpx_u128 x, uint64_t *ticket);
/* blocks until the request is answered; each ticket can be waited for once */
int cpx_serve_wait(cpx_server *srv, uint64_t ticket, cpx_u128 *pi, double *latency_ms);
/* submits xs[i] at arrival_s[i] seconds after the call (non-decreasing), waits
 * for all of them; latency_ms may be NULL */
int cpx_serve_replay(cpx_server *srv, const cpx_u128 *xs, const double *arrival_s, size_t n, cpx_u128 *pi,
                     double *latency_ms);
int cpx_serve_stats(cpx_server *srv, cpx_serve_counters *out);
const char *cpx_serve_last_error(cpx_server *srv);

/* Every term for n queries in one batched pass; ys[i] = 0 (or ys = NULL)
 * selects the y rule of params.  out[i] as filled by cpx_pi_u128. */
int cpx_terms_batch(cpx_ctx *ctx, const cpx_u128 *xs, const uint64_t *ys, size_t n,
                    const cpx_params *params, cpx_terms *out);

#ifdef __cplusplus
}
#endif
#endif /* CPX_H */
