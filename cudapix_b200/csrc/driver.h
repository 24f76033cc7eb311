// driver.h -- batch execution entry point shared by the C-ABI layer.
#pragma once
#include "cpx_internal.h"
#include "terms.cuh"

namespace cpx {

enum : unsigned {
    TERM_P2 = 1,
    TERM_ORD = 2,
    TERM_TRIV = 4,
    TERM_EASY = 8,
    TERM_HARD = 16,
    TERM_PI = 31  // every term plus the identity
};

struct BatchReq {
    const u128 *xs = nullptr;
    const uint64_t *ys = nullptr;  // per-query y (0 or null: default rule)
    size_t n = 0;
    uint32_t c = 6;
    uint32_t alpha_num = 0, alpha_den = 0;  // 0/0: reference alpha(x)
    uint32_t lbits = 0, threads = 0;        // hard-leaf tuning (0 = context default)
    unsigned terms = TERM_PI;
    uint64_t max_table_n = 1ull << 40;      // largest pi-table bound accepted
    uint64_t p2_table_limit = 1ull << 36;   // z beyond this: P2 by table windows
    u128 *out_pi = nullptr;                 // n entries
    i128 *out_terms = nullptr;              // 7 per query: P2 ord triv easy hard pi_y pi
    uint64_t *out_y = nullptr;
    uint32_t alpha_scale = 0;         // per mille of the reference alpha (0: 1000) when alpha_num = 0
    const uint32_t *alpha_scales = nullptr;  // per query, overriding alpha_scale where nonzero
    uint32_t lbits_cap = 0;           // cap of the hard-leaf segment bits (0: context default)
    const TuneEntry *tune = nullptr;  // per-decade alpha scale when alpha_num = alpha_scale = 0
    uint64_t seg_lo = 0, seg_hi = 0;  // one query's hard-leaf segments [seg_lo, seg_hi) (0, 0: all)
    HardLevel *hard_levels = nullptr; // per-level records of that part (host, nb - c entries)
    uint64_t easy_pmax = 0;           // easy leaves of the p <= easy_pmax only (0: every p <= icbrt x)
    bool wide = false;   // 128-bit kernels even when every x < 2^64
    bool graph = false;  // one CUDA graph launch for the batch's kernels
};

// table bounds of a batch: pi table to N, mu/lpf to Y, primes to P, wheel for c (0 = not needed)
struct TableNeed {
    uint64_t N = 0, Y = 0, P = 0;
    uint32_t c = 0;
};

void run_batch(cpx_ctx *ctx, const BatchReq &rq);
// Adds one part's per-level records (in segment order) to the running merge
// of a query's hard leaves split by segment ranges: carry[b] holds the
// survivors of level b-1 below the part, H the hard sum.
void merge_hard_part(std::vector<u128> &carry, i128 &H, const HardLevel *rec, uint32_t nlv);
void compute_needs(const BatchReq &rq, std::vector<QD> &qd, TableNeed &need, bool &wide);
bool tables_cover(const cpx_ctx *ctx, const TableNeed &need);
void grow_tables(cpx_ctx *ctx, const TableNeed &need);
// host mirror of the resident prime list, and pi(v) by binary search in it
const std::vector<uint32_t> &host_primes(cpx_ctx *ctx);
uint64_t host_pi(const std::vector<uint32_t> &P, uint64_t v);
// autotuning (autotune.cu)
uint32_t decade_of(u128 x);
void autotune(cpx_ctx *ctx, uint32_t e_lo, uint32_t e_hi, double seconds);
void autotune_batch(cpx_ctx *ctx, const u128 *xs, size_t n);
void tune_save(const cpx_ctx *ctx, const char *path);
void tune_load(cpx_ctx *ctx, const char *path);
// exact special-leaf counts of one query: hard, easy (composite m), easy (prime m), trivial
void leaf_counts(cpx_ctx *ctx, u128 x, uint64_t y, uint32_t c, uint64_t out[4]);
uint64_t default_y(u128 x, uint32_t num, uint32_t den);
// pi(x) through Gourdon's decomposition (gourdon.cu): A, B, C, D, Phi0, Sigma, pi
void gourdon_terms(cpx_ctx *ctx, uint64_t x, uint64_t y, uint32_t c, i128 out[7]);
uint32_t alpha_milli(u128 x);
bool dr_domain_ok(u128 x, uint64_t y, uint32_t c);

}  // namespace cpx
