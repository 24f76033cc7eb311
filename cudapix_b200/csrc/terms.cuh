// terms.cuh -- query descriptors and launch entry points of the term kernels.
#pragma once
#include "cpx_internal.h"

namespace cpx {

// One pi(x) evaluation as the device sees it.  Roots are exact floor roots
// computed on the host.
struct __align__(16) QD {
    u128 x;
    uint64_t y, z, sx, cx, r4, tx;  // tx = isqrt(x / y): trivial-leaf bound
    uint32_t c, nb;                 // nb = pi(r4)
    uint32_t lbits, direct;         // hard segment = 2^lbits odd numbers; direct = count by table
    uint64_t nseg;                  // hard-leaf segments over [0, z]
    uint32_t p2win;                 // P2 by pi-table windows over [sqrt x, z] (z beyond the table)
    uint32_t piy;                   // pi(y) when P2 walks the prime list (Plan::p2_primes)
    uint64_t seg0;                  // first hard-leaf segment (a part of a query split over GPUs)
};

// Per level b of a query's part: survivors of level b-1 over its segments,
// Sum(-mu) of its leaves, and, when the level's first sieved segment lies in
// the part, the carry that segment starts with (anchored = 1).
struct HardLevel {
    uint64_t count;
    int64_t msum;
    uint64_t carry0;
    uint32_t anchored, pad;
};

// One level of composite easy leaves of one query: odd m = 2i + 1 with
// i in [i_lo, i_hi); work units of 1024 indices from i_base (i_lo rounded
// down to a multiple of 4), numbered from unit0.
struct __align__(16) EasyLvl {
    uint32_t q, b, p, pad;
    uint64_t i_lo, i_hi, i_base, unit0;
};

// A heavy (sub-segment, level) leaf set handed from a sieve kernel to
// k_hard_leaves: the sub-segment's bitmap and per-chunk survivor prefixes at
// level b-1 sit in snapshot slot `snap` (one slot can serve the sets of
// several queries); the leaves are m in (mlo, mhi] (prime m only when
// kind = 1).  nunits counts its k_hard_leaves work units; their offsets are
// the scanned job-unit array.  `slot` is the level output that receives
// Sum(-mu), ~0 when `carry` already counts every survivor below the
// sub-segment.
struct __align__(16) HardJob {
    uint32_t q, b, p, kind;
    uint64_t mlo, mhi, lo, slot;  // lo: first number of the warp's sub-segment
    uint64_t nunits;              // k_hard_leaves work units
    uint64_t carry;               // survivors of level b-1 below the sub-segment (in its segment, or all)
    uint64_t snap;                // snapshot slot
    uint64_t pad;
    u128 xp;
};

// Up to 32 queries of a batch whose hard leaves share one sieve (z
// descending).  Its work units are the segments [0, nseg) of the group;
// xmax and r4max = iroot4(xmax) bound the levels each segment sieves.
constexpr uint32_t kGroupMax = 32;
// Consecutive groups that share one sieve of each segment (a work unit of the
// shared sieve is a block of up to kBlockMax groups and one segment).
constexpr uint32_t kBlockMax = 8;
struct __align__(16) HardGroup {
    u128 xmax;
    uint64_t r4max, nseg;
    uint32_t n, pad[3];
    uint32_t q[kGroupMax];
};

// accumulator slots per query (each a signed 128-bit value = 2 words)
enum { ACC_P2 = 0, ACC_ORD, ACC_TRIV, ACC_EASY, ACC_HARD, ACC_PIY, ACC_PI, ACC_N };
constexpr int kAccStride = 2 * ACC_N;  // u64 words per query

// Unit prefix arrays (Q + 1 entries each, pre[0] = 0) over the queries of a
// batch, one per kernel family.
struct Plan {
    uint32_t Q = 0;
    const QD *qd = nullptr;
    const uint64_t *pre_ord = nullptr, *pre_p2 = nullptr, *pre_triv = nullptr, *pre_easy = nullptr,
                   *pre_seg = nullptr, *pre_comb = nullptr;
    uint64_t n_ord = 0, n_p2 = 0, n_triv = 0, n_easy = 0, n_seg = 0, n_comb = 0;
    uint64_t hard_entries = 0;
    uint32_t c = 6;
    bool wide = false;  // 128-bit kernels (some x >= 2^64, or requested)
    bool time_hard = false;  // CUDA events around the hard-leaf kernels
    uint32_t hard_threads = 256;
    uint32_t lbits_max = 18;
    // device work arrays
    uint32_t *seg_B = nullptr;
    uint64_t *seg_off = nullptr;
    uint32_t *hard_cnt = nullptr;
    int32_t *hard_ms = nullptr;
    unsigned long long *acc = nullptr;
    unsigned int *ticket = nullptr;
    // heavy hard-leaf sets offloaded from k_hard
    HardJob *jobs = nullptr;
    unsigned int *njobs = nullptr;   // device counter
    uint64_t *job_units = nullptr;   // max_jobs + 1 work-unit counts, scanned into offsets
    unsigned char *snap = nullptr;   // snapshot slots
    uint32_t max_jobs = 0;
    uint64_t offload_min = 0;        // candidate threshold of an offloaded leaf set (0: none)
    // composite easy leaves
    const EasyLvl *elv = nullptr;
    uint32_t n_elv = 0;
    uint64_t n_ecomp = 0;
    bool p2_primes = false;        // P2 units are the primes of (y, sqrt x] (k_p2_primes), else pi-table entries
    uint64_t *easy_off = nullptr;  // n_easy + 1 chunk offsets of the easy leaves
    void *easy_rec = nullptr;      // n_easy unit plans (EasyRec, 64 B each), or null: k_easy plans itself
    HardLevel *hard_levels = nullptr;  // per-level outputs of query 0 (a part of a split query)
    // batch-shared sieve (hard_shared.cu): one counting sweep over the
    // segments [0, sh_nseg) for xmax, carries per (sub-segment, level) in
    // rows from lvl_off, then the groups' units
    bool shared = false;
    uint32_t sh_lbits = 0, sh_nlv = 0, n_grp = 0;
    uint64_t sh_nseg = 0, sh_r4max = 0, n_gunits = 0, n_carry = 0;
    u128 sh_xmax = 0;
    const HardGroup *grp = nullptr;
    // units (n_gunits): a segment and up to kBlockMax consecutive groups,
    // seg << 32 | g0 << 4 | (n - 1), segment-major
    const uint64_t *units = nullptr;
    const uint64_t *lvl_off = nullptr;  // sh_nlv + 1 row offsets into carry
    uint64_t *carry = nullptr;
    unsigned int *nsnap = nullptr;      // device counter of snapshot slots
    void *gxp = nullptr;                // x/p per (group, level, slot): uint64 or u128 (wide)
    uint2 *gae = nullptr;               // y/p and min(y, x/p^3) per (group, level, slot)
    // persistent launch of the shared sieve: the device counter that hands
    // out the units in order (null: one CTA per unit)
    unsigned long long *unit_next = nullptr;
};

void launch_ordinary(cpx_ctx *ctx, const Plan &pl);
void launch_p2(cpx_ctx *ctx, const Plan &pl);
// P2 of one query by pi-table windows over v = x/p in [sqrt x, x/(y+1)];
// adds into the query's accumulator acc (device).  Host loop, synchronous.
void p2_windowed(cpx_ctx *ctx, const QD &d, unsigned long long *acc_q, bool wide);
void launch_trivial(cpx_ctx *ctx, const Plan &pl);
void launch_easy(cpx_ctx *ctx, const Plan &pl);
void launch_easy_comp(cpx_ctx *ctx, const Plan &pl);
void launch_hard(cpx_ctx *ctx, const Plan &pl);
void launch_finalize(cpx_ctx *ctx, const Plan &pl, u128 *d_out_pi, bool full);
size_t hard_smem_bytes(uint32_t lbits, uint32_t threads, bool wide);
// host-side set-up of the hard-leaf kernels (kernel attributes); called
// before the launches so that they can be captured in a graph
void prepare_hard(cpx_ctx *ctx, const Plan &pl);
size_t hard_snapshot_stride(uint32_t lbits_max);
// the batch-shared sieve (hard_shared.cu)
void prepare_hard_shared(cpx_ctx *ctx, const Plan &pl);
void launch_hard_shared(cpx_ctx *ctx, const Plan &pl);
size_t hard_shared_smem_bytes(uint32_t lbits, uint32_t threads);
// k_hard_leaves over the jobs of pl (hard.cu)
void launch_hard_leaves(cpx_ctx *ctx, const Plan &pl, uint32_t lbits_sub);

}  // namespace cpx
