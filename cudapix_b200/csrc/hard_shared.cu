// hard_shared.cu -- the hard special leaves of a batch on one shared sieve.
//
// The state of the segmented phi sieve after crossing off p_c+1 .. p_b-1 does
// not depend on x; only the leaves do.  A batch therefore sieves each
// segment once for many queries:
//  (1) k_sieve_counts sweeps the segments [0, nseg) once, for the largest x of
//      the batch, and records the survivors of level b-1 of every warp
//      sub-segment;
//  (2) k_carry_scan turns each level's row of counts into the carries
//      phi(lo_w - 1, b - 1), the survivors below each sub-segment (a level's
//      first sieved segment starts from the pi table: below p_b^2 the
//      survivors of level b-1 are 1 and the primes from p_b on);
//  (3) k_hard_shared runs one CTA per (group of up to 32 queries, segment).
//      Its warps sieve their sub-segments level by level as k_hard does; at
//      each level the lanes compute the candidate range of one query each
//      (from a per-(group, level) table of x/p, y/p and x/p^3 that
//      k_group_levels fills once per batch), answer their own query's leaves
//      when every query has few, or else the warp gathers the leaves of every
//      query and answers them 32 at a time; each leaf's -mu(m) phi(u, b-1) =
//      -mu(m) (carry + survivors of the sub-segment <= u) goes straight into
//      its query's sum: no per-segment outputs and no carry combine.
// Heavy (query, sub-segment, level) leaf sets go to k_hard_leaves with one
// snapshot per (sub-segment, level) for all queries of the group.
//
// Restates the reference's hard-leaf sieve (src/sieve/S2_hard_host.cu:49-191,
// src/sieve/S2_hard_device.cu:12-382), which sieves [0, z) once per x, for many
// x at a time.
#include <mutex>

#include "sieve.cuh"

namespace cpx {

// shared memory of k_sieve_counts: bitmap and chunk counters
__host__ __device__ __forceinline__ size_t counts_smem(uint32_t lbits)
{
    const size_t L = size_t(1) << lbits;
    return L / 8 + (((L / 128) + 15) & ~size_t(15));
}

// gathered leaves per warp: 256, or 128 for 32 warps (2^20 bits, 1024
// threads, fit 227 KB of shared memory)
__host__ __device__ __forceinline__ uint32_t leaf_cap(uint32_t threads) { return threads >= 1024 ? 128u : kLeafBuf; }

// shared memory of k_hard_shared
__host__ __device__ __forceinline__ size_t shared_smem(uint32_t lbits, uint32_t threads)
{
    size_t o = counts_smem(lbits);
    o += ((size_t(1) << lbits) / 128) * 2;         // chunk prefixes within their lane
    o += threads * 4;                              // lane prefixes
    o += (threads / 32) * leaf_cap(threads) * 8;   // gathered leaves: m, query | (mu(m) = -1) << 31
    o += (threads / 32) * kGroupMax * 16;  // x/p of the group's queries, per warp
    o += (threads / 32) * kGroupMax * 12;  // per-warp, per-query level sums and Sum(-mu)
    o += kBlockMax * kGroupMax * 12;       // per (group, slot): query, y, level threshold
    o += kBlockMax * kGroupMax * 16;       // per (group, slot): the hard sum over the unit
    return o;
}

// (1) One CTA per segment: survivors of level b-1 of each warp sub-segment w,
// for every level b the segment sieves, into row b at w - NW * first(b), where
// first(b) = p_b^2 / span is the level's first segment.
__global__ void __launch_bounds__(1024, 1) k_sieve_counts(uint64_t nseg, uint32_t lbits, u128 xmax, uint64_t r4max,
                                                       uint32_t c, const uint32_t *__restrict__ P, uint32_t np,
                                                       const uint64_t *__restrict__ lvl_off, uint32_t nlv,
                                                       uint64_t *__restrict__ cnt)
{
    extern __shared__ uint4 smem4[];
    __shared__ uint32_t s_B;
    const uint64_t seg = blockIdx.x;
    if (seg >= nseg) return;
    const uint32_t T = blockDim.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, NW = T >> 5;
    const uint32_t L = 1u << lbits, NC = L >> 7, CPT = NC / T;
    const int s = __ffs(CPT) - 1;
    const uint32_t Lw = L / NW;
    const uint64_t span = 2ull * L, lo = seg * span;
    const uint64_t lo_w = lo + 2ull * Lw * warp, hi_w = lo_w + 2ull * Lw;
    if (tid == 0) s_B = seg_levels<u128>(xmax, r4max, lo, lo + span, P, np);
    __syncthreads();
    const uint32_t B = min(s_B, c + nlv);  // rows exist up to level c + nlv
    if (B <= c) return;                    // uniform over the CTA
    uint32_t *bm = reinterpret_cast<uint32_t *>(smem4);
    uint8_t *cnt8 = reinterpret_cast<uint8_t *>(smem4) + L / 8;
    const uint32_t c0 = CPT * tid, cw0 = c0 - CPT * 32 * warp;
    uint32_t tot = __reduce_add_sync(FULL, presieve(bm, cnt8, P, c, lo, c0, CPT, s));
    __syncwarp();
    const uint64_t w = seg * NW + warp;
    for (uint32_t gb = c + 1; gb <= B; gb += 32) {
        const uint32_t nl = min(32u, B - gb + 1);
        uint32_t lp = 0, lr0 = 0, li0 = 0xFFFFFFFFu;
        if (lane < nl) {
            lp = P[gb + lane - 1];
            cross_params(lp, lo_w, hi_w, lr0, li0);
        }
        for (uint32_t k = 0; k < nl; k++) {
            const uint32_t b = gb + k;
            const uint32_t p = __shfl_sync(FULL, lp, k);
            if (lane == 0) {
                const uint64_t first = ((uint64_t)p * p) >> (lbits + 1);  // / span
                const uint64_t idx = lvl_off[b - c - 1] + (w - first * NW);
                if (idx < lvl_off[b - c]) cnt[idx] = tot;
            }
            const uint32_t cleared = cross_off(bm, cnt8, p, __shfl_sync(FULL, lr0, k), __shfl_sync(FULL, li0, k), c0,
                                               cw0, CPT, s, CPT * 32 * warp, lane, Lw);
            tot -= __reduce_add_sync(FULL, cleared);
            __syncwarp();
        }
    }
}

// (2) One CTA per level: exclusive scan of the level's row in place, from the
// carry of its first segment.
__global__ void __launch_bounds__(1024) k_carry_scan(uint32_t nlv, uint32_t c, uint64_t span,
                                                     const uint32_t *__restrict__ P, const cpx_pient *__restrict__ T,
                                                     const uint64_t *__restrict__ lvl_off, uint64_t *__restrict__ cnt)
{
    __shared__ uint64_t s_w[32];
    const uint32_t lv = blockIdx.x;
    if (lv >= nlv) return;
    const uint32_t b = c + 1 + lv;
    const uint64_t p = P[b - 1];
    const uint64_t first = (p * p) / span;
    uint64_t carry = 0;
    if (first > 0) {
        const uint64_t pl = cpx_pi_dev(T, first * span - 1);
        carry = 1 + (pl > b - 1 ? pl - (b - 1) : 0);
    }
    const uint64_t r0 = lvl_off[lv], r1 = lvl_off[lv + 1];
    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
    for (uint64_t base = r0; base < r1; base += blockDim.x) {
        const uint64_t i = base + tid;
        const uint64_t v = i < r1 ? cnt[i] : 0;
        uint64_t inc = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint64_t t = __shfl_up_sync(FULL, inc, o);
            if (lane >= (uint32_t)o) inc += t;
        }
        if (lane == 31) s_w[warp] = inc;
        __syncthreads();
        if (warp == 0) {
            uint64_t wv = lane < nw ? s_w[lane] : 0;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint64_t t = __shfl_up_sync(FULL, wv, o);
                if (lane >= (uint32_t)o) wv += t;
            }
            if (lane < nw) s_w[lane] = wv;
        }
        __syncthreads();
        const uint64_t before = warp ? s_w[warp - 1] : 0;
        if (i < r1) cnt[i] = carry + before + inc - v;
        carry += s_w[nw - 1];
        __syncthreads();
    }
}

// Quotients n / d by a sub-segment bound d >= 2^13 with rd = 1/d (double,
// once per warp): for n < 2^64 the quotient is below 2^51, so the truncated
// product n * rd (relative error at most 3 * 2^-53) is within 1 of it and the
// sign and size of the remainder n - q d fix it.  128-bit n: exact division.
struct Recip {
    uint64_t d;
    double rd;
};
template <class XT> __device__ __forceinline__ XT div_recip(XT n, const Recip &r)
{
    if ((u128)n >> 64) return cpx_qdiv(n, r.d);
    const uint64_t n64 = (uint64_t)n;
    uint64_t q = __double2ull_rz(__dmul_rn(__ull2double_rn(n64), r.rd));
    const int64_t rem = (int64_t)(n64 - q * r.d);
    if (rem < 0) q--;
    else if ((uint64_t)rem >= r.d) q++;
    return (XT)q;
}

// The per-level constants of every query of every group: x/p, y/p and
// min(y, x/p^3) at index (g nlv + b - c - 1) 32 + slot.  They do not depend
// on the segment, so k_hard_shared loads them instead of dividing.
template <class XT>
__global__ void k_group_levels(const QD *__restrict__ qd, const HardGroup *__restrict__ grp, uint32_t ngrp,
                               uint32_t nlv, uint32_t c, const uint32_t *__restrict__ P, XT *__restrict__ gxp,
                               uint2 *__restrict__ gae)
{
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (uint64_t)ngrp * nlv * 32) return;
    const uint32_t slot = (uint32_t)(i & 31), lv = (uint32_t)((i >> 5) % nlv), g = (uint32_t)((i >> 5) / nlv);
    XT xp = 0;
    uint32_t a = 0, e = 0;
    if (slot < grp[g].n) {
        const QD &d = qd[grp[g].q[slot]];
        const uint64_t p = P[c + lv];
        xp = cpx_qdiv(xload<XT>(d), p);
        a = (uint32_t)cpx_udiv_leaf(d.y, p);
        const XT t3 = cpx_qdiv(xp, p * p);
        e = (uint32_t)(t3 < (XT)d.y ? (uint64_t)t3 : d.y);
    }
    gxp[i] = xp;
    gae[i] = make_uint2(a, e);
}

// Hands the heavy leaf sets of one (sub-segment, level) to k_hard_leaves: one
// snapshot of the sub-segment (bitmap and chunk prefixes) for all of them,
// one job per set.  Every lane calls; returns whether this lane's set went
// (a set that finds no job slot left is answered in the sieve).  Rare path,
// out of line.
template <class XT>
static __device__ __noinline__ bool offload_sets(bool off_j, uint32_t lane, uint32_t qj, uint32_t b, uint32_t p,
                                                 bool prime_j, uint32_t qa_j, uint32_t mlo, uint32_t mhi,
                                                 uint64_t work, uint64_t lo_w, uint64_t C, XT xp, const uint32_t *bm,
                                                 const uint8_t *cnt8, uint32_t cw0, uint32_t c0, uint32_t CPT, int s,
                                                 uint32_t pre, HardJob *__restrict__ jobs,
                                                 unsigned int *__restrict__ njobs, uint64_t *__restrict__ job_units,
                                                 unsigned char *__restrict__ snap, unsigned int *__restrict__ nsnap,
                                                 uint32_t max_jobs, uint32_t lbits_sub)
{
    uint32_t snap_k = 0xFFFFFFFFu;
    for (unsigned offm = __ballot_sync(FULL, off_j); offm; offm &= offm - 1) {
        const uint32_t j = __ffs(offm) - 1;
        unsigned int jb = 0, sn = snap_k;
        if (lane == 0) {
            jb = atomicAdd(njobs, 1u);
            if (jb < max_jobs && sn == 0xFFFFFFFFu) sn = atomicAdd(nsnap, 1u);
        }
        jb = __shfl_sync(FULL, jb, 0);
        sn = __shfl_sync(FULL, sn, 0);
        // (a job slot taken without a snapshot keeps 0 units)
        if (jb < max_jobs && sn < max_jobs) {
            if (snap_k == 0xFFFFFFFFu) {
                snap_k = sn;
                uint4 *sb = reinterpret_cast<uint4 *>(snap + (size_t)sn * snap_stride(lbits_sub));
                uint32_t *spre = reinterpret_cast<uint32_t *>(sb + ((size_t(1) << lbits_sub) >> 7));
                snapshot_chunks(sb, spre, bm, cnt8, cw0, c0, CPT, s, pre);
            }
            if (lane == j) {
                HardJob J;
                J.q = qj;
                J.b = b;
                J.p = p;
                J.kind = prime_j ? 1u : 0u;
                J.mlo = prime_j ? qa_j : mlo;
                J.mhi = mhi;
                J.lo = lo_w;
                J.slot = ~0ull;
                J.nunits = prime_j ? (work / 8 + kJobWords - 1) / kJobWords
                                   : ((((uint64_t)mhi - 1) >> 3) - (((uint64_t)mlo + 1) >> 3) + kJobGroups) / kJobGroups;
                J.carry = C;
                J.snap = sn;
                J.pad = 0;
                J.xp = (u128)xp;
                jobs[jb] = J;
                job_units[jb] = J.nunits;
            }
        } else if (lane == j) {
            off_j = false;  // no slot left: answered here
        }
    }
    return off_j;
}

// Candidate entries (pi-table words or 4-m groups) a lane answers itself;
// above it on any lane the warp gathers the level's leaves (on the B200 the
// 4096-query batch took 49.0 / 46.0 / 41.4 / 40.9 ms of this kernel with 8 /
// 16 / 32 / 64 when each unit held one group; with blocks of groups 20.9 /
// 20.5 / 20.4 ms with 32 / 64 / 128)
constexpr uint32_t kLaneEntries = 128;

// (3) One CTA per unit: a segment and a block of up to kBlockMax groups.  Per
// level and group, the lanes hold one query each: its x/p and candidate range
// in the warp's sub-segment.  When no query has more than kLaneEntries
// candidate table entries (98% of the visits of the 4096-query batch, with
// about 1.3 entries a query), each lane answers its own query's leaves and
// adds them into the query's slot of the unit's sums.
// Otherwise the warp walks the candidates of all the group's queries as one
// sequence (pi-table words of the prime-only levels, then 4-m groups of
// packed mu*lpf of the others), 32 words at a time, each lane finding its
// word's query by a binary search over the warp's exclusive word counts; the
// leaves found go to the warp's buffer (m, query | (mu(m) = -1) << 31) and
// are answered 32 at a time.  Each lane keeps a running Sum(-mu) * count and
// Sum(-mu) for the query of its last leaf and adds them into the warp's
// per-query slots when the query changes; at the end of the level lane j
// adds slot j into its query's unit sum as sum + carry * Sum(-mu).
// The launch bounds (at most TMAX threads, at least MINB blocks per SM) set
// the register budget: 65536 / (TMAX MINB) a thread, 64 when 32 warps share
// an SM and 128 (no spills) when 16 do.  The launch takes the variant whose
// MINB blocks fit the SM's shared memory with this segment size.
#define CPX_HS_PARAMS                                                                                          \
    const QD *__restrict__ qd, const HardGroup *__restrict__ grp, const uint64_t *__restrict__ units,            \
        uint64_t total, uint32_t lbits, uint32_t c, const uint32_t *__restrict__ P, uint32_t np, \
        const int32_t *__restrict__ MU, const cpx_pient *__restrict__ Tpi, const uint64_t *__restrict__ lvl_off, \
        uint32_t nlv, const uint64_t *__restrict__ carry, unsigned long long *__restrict__ acc,                   \
        HardJob *__restrict__ jobs, unsigned int *__restrict__ njobs, uint64_t *__restrict__ job_units,          \
        unsigned char *__restrict__ snap, unsigned int *__restrict__ nsnap, uint32_t max_jobs, uint32_t lbits_sub, \
        uint32_t offload_min, const XT *__restrict__ gxp, const uint2 *__restrict__ gae
#define CPX_HS_ARGS                                                                                             \
    qd, grp, units, total, lbits, c, P, np, MU, Tpi, lvl_off, nlv, carry, acc, jobs, njobs, job_units, snap, \
        nsnap, max_jobs, lbits_sub, offload_min, gxp, gae

// one unit of the shared sieve, by one CTA: a segment and up to kBlockMax
// consecutive groups (z descending), packed as seg << 32 | g0 << 4 | (n - 1).
// The segment is sieved once for all of them, and each level answers every
// group's leaves in turn.
template <class XT> __device__ __forceinline__ void hard_shared_unit(uint64_t unit, CPX_HS_PARAMS)
{
    extern __shared__ uint4 smem4[];
    __shared__ uint32_t s_Bg[kBlockMax], s_ng[kBlockMax];
    const uint64_t ud = units[unit];
    const uint64_t seg = ud >> 32;
    const uint32_t g0 = (uint32_t)(ud >> 4) & 0x0FFFFFFFu, ngr = (uint32_t)(ud & 15) + 1;
    const uint32_t T = blockDim.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, NW = T >> 5;
    const uint32_t L = 1u << lbits, NC = L >> 7, CPT = NC / T;
    const int s = __ffs(CPT) - 1;
    const uint32_t Lw = L / NW;
    const uint64_t span = 2ull * L, lo = seg * span;
    const uint64_t lo_w = lo + 2ull * Lw * warp, hi_w = lo_w + 2ull * Lw;
    // per group: the levels the segment sieves for it (0: none, the group's
    // queries end below the segment) and its query count
    if (tid < kBlockMax) {
        uint32_t bg = 0, n = 0;
        if (tid < ngr && seg < grp[g0 + tid].nseg) {
            const HardGroup &G = grp[g0 + tid];
            bg = min(seg_levels<XT>((XT)G.xmax, G.r4max, lo, lo + span, P, np), c + nlv);
            n = G.n;
        }
        s_Bg[tid] = bg;
        s_ng[tid] = n;
    }
    __syncthreads();
    uint32_t B = 0;
    for (uint32_t g = 0; g < ngr; g++) B = max(B, s_Bg[g]);
    if (B <= c) return;  // uniform over the CTA

    unsigned char *sp = reinterpret_cast<unsigned char *>(smem4);
    uint32_t *bm = reinterpret_cast<uint32_t *>(sp);
    size_t o = L / 8;
    uint8_t *cnt8 = sp + o;
    o += ((L / 128) + 15) & ~size_t(15);
    uint16_t *pre16 = reinterpret_cast<uint16_t *>(sp + o);  // chunk prefixes within their lane
    o += (L / 128) * 2;
    uint32_t *wl = reinterpret_cast<uint32_t *>(sp + o) + 32 * warp;  // this warp's lane prefixes
    o += T * 4;
    uint2 *lbuf0 = reinterpret_cast<uint2 *>(sp + o);
    const uint32_t cap = leaf_cap(T);
    uint2 *lbuf = lbuf0 + cap * warp;
    o += NW * cap * 8;
    XT *s_xp = reinterpret_cast<XT *>(sp + o) + 32 * warp;  // x/p of each query at the current level
    o += NW * 32 * 16;
    unsigned long long *s_sum = reinterpret_cast<unsigned long long *>(sp + o) + 32 * warp;
    o += NW * 32 * 8;
    int *s_ms = reinterpret_cast<int *>(sp + o) + 32 * warp;
    o += NW * 32 * 4;
    // per (group, slot) of the block: the query, its y and its level
    // threshold, and its hard sum over the unit (two words, added by atomics)
    uint32_t *s_qj = reinterpret_cast<uint32_t *>(sp + o);
    uint32_t *s_yj = s_qj + kBlockMax * 32;
    uint32_t *s_pt = s_yj + kBlockMax * 32;
    o += kBlockMax * 32 * 12;
    unsigned long long *s_acc = reinterpret_cast<unsigned long long *>(sp + o);
    s_sum[lane] = 0;
    s_ms[lane] = 0;
    // A query has leaves in the segment at level b only if lo <= z, p^2 < hi
    // and x / (p hi) < y, i.e. p > pthr = floor(x / (y hi)) (hi the segment's
    // end; each warp's exact candidate range decides the rest); y < 2^31.
    // pthr = 0xFFFFFFFF: no leaves (lo > z, or no query in the slot).
    for (uint32_t t = tid; t < kBlockMax * 32; t += T) {
        const uint32_t g = t >> 5, j = t & 31;
        uint32_t qv = 0xFFFFFFFFu, yv = 0, pt = 0xFFFFFFFFu;
        if (g < ngr && j < s_ng[g]) {
            qv = grp[g0 + g].q[j];
            const QD &d = qd[qv];
            yv = (uint32_t)d.y;
            if (lo <= d.z) {
                const u128 tt = (u128)xload<XT>(d) / ((u128)d.y * (lo + span));
                pt = tt < 0xFFFFFFFFull ? (uint32_t)tt : 0xFFFFFFFFu;
            }
        }
        s_qj[t] = qv;
        s_yj[t] = yv;
        s_pt[t] = pt;
        s_acc[2 * t] = 0;
        s_acc[2 * t + 1] = 0;
    }
    __syncthreads();

    const uint32_t c0 = CPT * tid, cw0 = c0 - CPT * 32 * warp;
    presieve(bm, cnt8, P, c, lo, c0, CPT, s);
    __syncwarp();
    const uint64_t w = seg * NW + warp;
    auto sub_count = [&](uint64_t uu) -> uint32_t { return sub_survivors_pre(uu, lo_w, wl, pre16, bm, CPT, s, warp); };
    // the leaf quotient x/(p m) (leaf_quot: cpx_quot40 when x/p < 2^53; xvd = x/p as a double)
    // leaf quotients lie in [lo_w, hi_w): below 2^31 - 2 the 32-bit corrected
    // form (m <= y < 2^31), below 2^41 cpx_quot40 (both for x/p < 2^53)
    const bool q41 = hi_w <= (1ull << 41), q31 = hi_w <= (1ull << 31) - 2;
    auto hq = [&](XT xv, double xvd, uint64_t m) -> uint64_t {
        if (q31 && ((u128)xv >> 53) == 0)
            return cpx_quot40_small((uint64_t)xv, xvd, (uint32_t)m, cpx_rcp_approx((uint32_t)m));
        return leaf_quot(xv, xvd, m, q41);
    };
    const Recip r_lo{lo_w, lo_w ? 1.0 / (double)lo_w : 0.0}, r_hi{hi_w, 1.0 / (double)hi_w};

    for (uint32_t gb = c + 1; gb <= B; gb += 32) {
        const uint32_t nl = min(32u, B - gb + 1);
        // per lane k, level gb + k: its prime, crossing-off start and the
        // carry of the warp's sub-segment (survivors of level b - 1 below it,
        // row b of the counting sweep), all loaded at once
        uint32_t lp = 0, lr0 = 0, li0 = 0xFFFFFFFFu;
        uint64_t lC = 0;
        if (lane < nl) {
            const uint32_t bl = gb + lane;
            lp = P[bl - 1];
            cross_params(lp, lo_w, hi_w, lr0, li0);
            const uint64_t first = ((uint64_t)lp * lp) >> (lbits + 1);  // / span
            const uint64_t ci = lvl_off[bl - c - 1] + (w - first * NW);
            if (ci < lvl_off[bl - c]) lC = __ldg(carry + ci);
        }
        for (uint32_t k = 0; k < nl; k++) {
            const uint32_t b = gb + k;
            const uint32_t p = __shfl_sync(FULL, lp, k);
            const uint64_t pp = (uint64_t)p * p;
            bool built = false;  // the level's chunk and lane prefixes
            for (uint32_t g = 0; g < ngr; g++) {
            if (b > s_Bg[g]) continue;  // uniform: the group's queries end below this level here
            const uint32_t tq = 32 * g + lane;  // this lane's slot of group g
            const uint32_t qj = s_qj[tq], yj = s_yj[tq], pthr = s_pt[tq], nq = s_ng[g];
            // Candidates (mlo, mhi] of this lane's query in the warp's
            // sub-segment.  None unless some u in it satisfies u <= z,
            // u >= p^2 and x/(p hi_w) < y (else m > y).
            XT xp = 0;
            uint32_t mlo = 0, mhi = 0;
            bool act = false;
            if (hi_w > pp && p > pthr) {
                const size_t gi = ((size_t)(g0 + g) * nlv + (b - c - 1)) * 32 + lane;
                xp = gxp[gi];
                const uint2 ae = gae[gi];  // y/p, min(y, x/p^3)
                uint64_t a = ae.x;
                const XT t1 = div_recip(xp, r_hi);
                if (t1 > (XT)a) a = (uint64_t)t1;
                uint64_t e = ae.y;
                if (lo_w) {
                    const XT t2 = div_recip(xp, r_lo);
                    if (t2 < (XT)e) e = (uint64_t)t2;
                }
                mlo = (uint32_t)a;
                mhi = (uint32_t)(e > a ? e : a);
                act = e > ((pp > yj && p > a) ? (uint64_t)p : a);
            }
            const unsigned bal = __ballot_sync(FULL, act);
            if (bal) {
                if (!built) {
                    // chunk and lane prefixes of the sub-segment from the chunk counters
                    uint32_t off0;
                    warp_place(chunk_prefixes(cnt8, pre16, c0, CPT), lane, off0);
                    wl[lane] = off0;
                    built = true;
                }
                if (act) s_xp[lane] = xp;
                __syncwarp();
                const uint64_t C = __shfl_sync(FULL, lC, k);  // survivors below the sub-segment
                const bool prime_j = pp > yj;  // m must be a prime q > max(mlo, p)
                const uint32_t qa_j = mlo > p ? mlo : p;
                uint64_t work = 0;
                if (act)
                    work = prime_j ? 8 * ((((uint64_t)mhi - 1) >> 7) - (qa_j >> 7) + 1)
                                   : ((((uint64_t)mhi - 1) >> 1) - (((uint64_t)mlo + 1) >> 1) + 1);
                // heavy sets to k_hard_leaves, one snapshot for the warp's level
                bool off_j = act && max_jobs && offload_min && work >= offload_min;
                if (__any_sync(FULL, off_j))
                    off_j = offload_sets<XT>(off_j, lane, qj, b, p, prime_j, qa_j, mlo, mhi, work, lo_w, C, xp, bm, cnt8,
                                             cw0, c0, CPT, s, wl[lane], jobs, njobs, job_units, snap, nsnap, max_jobs,
                                             lbits_sub);
                const uint32_t nw_j =
                    (act && !off_j && prime_j) ? (uint32_t)((((uint64_t)mhi - 1) >> 7) - (qa_j >> 7) + 1) : 0u;
                uint32_t ng_j = 0;
                if (act && !off_j && !prime_j)
                    ng_j = (uint32_t)(((((uint64_t)mhi - 1) >> 1) >> 2) - ((((uint64_t)mlo + 1) >> 1) >> 2) + 1);
                if (!__any_sync(FULL, nw_j > kLaneEntries || ng_j > kLaneEntries)) {
                    // a sparse level (the common case: about one leaf per query;
                    // at most kLaneEntries table entries or 4-m groups each):
                    // each lane answers its own query's candidates
                    int64_t sv = 0;
                    int32_t sm = 0;
                    const double xpd = (double)(uint64_t)xp;
                    for (uint32_t k2 = 0; k2 < nw_j; k2++) {
                        const uint64_t wq = (qa_j >> 7) + k2;
                        uint64_t qb = __ldg(reinterpret_cast<const ulonglong2 *>(Tpi) + wq).x & range_mask(wq, qa_j, mhi);
                        while (qb) {
                            const int jb = __ffsll((long long)qb) - 1;
                            qb &= qb - 1;
                            sv += sub_count(hq(xp, xpd, 128 * wq + 2 * jb + 1));  // mu(q) = -1
                            sm += 1;
                        }
                    }
                    const uint64_t i_lo = ((uint64_t)mlo + 1) >> 1, i_hi = ((uint64_t)mhi - 1) >> 1;
                    for (uint32_t k2 = 0; k2 < ng_j; k2++) {
                        const uint64_t g4 = (i_lo >> 2) + k2;
                        uint32_t neg = 0;
                        uint32_t vm =
                            valid_group(__ldg(reinterpret_cast<const int4 *>(MU) + g4), g4, i_lo, i_hi, p, &neg);
                        while (vm) {
                            const int kq = __ffs(vm) - 1;
                            vm &= vm - 1;
                            const uint32_t cv = sub_count(hq(xp, xpd, 2 * (4 * g4 + kq) + 1));
                            if ((neg >> kq) & 1u) {
                                sv += cv;
                                sm += 1;
                            } else {
                                sv -= cv;
                                sm -= 1;
                            }
                        }
                    }
                    if (sv || sm) cpx_atomic_add_i128(s_acc + 2 * tq, (i128)sv + (i128)C * (i128)sm);
                    __syncwarp();
                } else {
                // running sums of the query of this lane's last leaf
                uint32_t cur = 0xFFu;
                int64_t csum = 0;
                int32_t cms = 0;
                auto put = [&](uint32_t key, uint32_t cv, bool plus) {
                    if (key != cur) {
                        if (cur != 0xFFu) {
                            atomicAdd(s_sum + cur, (unsigned long long)csum);
                            atomicAdd(s_ms + cur, cms);
                        }
                        cur = key;
                        csum = 0;
                        cms = 0;
                    }
                    if (plus) {
                        csum += cv;
                        cms += 1;
                    } else {
                        csum -= cv;
                        cms -= 1;
                    }
                };
                uint32_t nbuf = 0;
                auto flush = [&] {
                    __syncwarp();
                    for (uint32_t jj = lane; jj < nbuf; jj += 32) {
                        const uint2 e = lbuf[jj];
                        const uint32_t key = e.y & 31u;
                        const XT xk = s_xp[key];
                        put(key, sub_count(hq(xk, (double)(uint64_t)xk, e.x)), (e.y >> 31) != 0);
                    }
                    __syncwarp();
                    nbuf = 0;
                };
                // the query owning flat item f: the last lane j with ex[j] <= f
                auto owner = [&](uint32_t ex, uint32_t f) -> uint32_t {
                    uint32_t jq = 0;
#pragma unroll
                    for (uint32_t st = 16; st; st >>= 1) {
                        const uint32_t cnd = jq + st;
                        if (__shfl_sync(FULL, ex, cnd) <= f) jq = cnd;
                    }
                    return jq;
                };
                {
                    // prime-only levels: pi-table words of (max(mlo, p), mhi]
                    uint32_t ex_j;
                    const uint32_t tot_w = warp_place(nw_j, lane, ex_j);
                    for (uint32_t base = 0; base < tot_w; base += 32) {
                        const uint32_t f = base + lane;
                        const uint32_t jq = owner(ex_j, f);
                        const uint32_t exq = __shfl_sync(FULL, ex_j, jq);
                        const uint64_t qaq = __shfl_sync(FULL, qa_j, jq), mhq = __shfl_sync(FULL, mhi, jq);
                        uint64_t qb = 0, wq = 0;
                        if (f < tot_w) {
                            wq = (qaq >> 7) + (f - exq);
                            qb = __ldg(reinterpret_cast<const ulonglong2 *>(Tpi) + wq).x & range_mask(wq, qaq, mhq);
                        }
                        uint32_t off;
                        const uint32_t tot_r = warp_place((uint32_t)__popcll(qb), lane, off);
                        if (tot_r > cap) {  // a dense round: each lane answers its own word
                            const XT xq = s_xp[jq];
                            while (qb) {
                                const int jb = __ffsll((long long)qb) - 1;
                                qb &= qb - 1;
                                put(jq, sub_count(hq(xq, (double)(uint64_t)xq, 128 * wq + 2 * jb + 1)), true);  // mu(q) = -1
                            }
                            continue;
                        }
                        if (nbuf + tot_r > cap) flush();
                        uint32_t kk = nbuf + off;
                        while (qb) {
                            const int jb = __ffsll((long long)qb) - 1;
                            qb &= qb - 1;
                            lbuf[kk++] = make_uint2((uint32_t)(128 * wq + 2 * jb + 1), jq | 0x80000000u);
                        }
                        nbuf += tot_r;
                    }
                }
                {
                    // other levels: squarefree m with lpf(m) > p, 16-byte groups of packed mu*lpf
                    uint32_t ex_j;
                    const uint32_t tot_g = warp_place(ng_j, lane, ex_j);
                    for (uint32_t base = 0; base < tot_g; base += 32) {
                        const uint32_t f = base + lane;
                        const uint32_t jq = owner(ex_j, f);
                        const uint32_t exq = __shfl_sync(FULL, ex_j, jq);
                        const uint64_t mlq = __shfl_sync(FULL, mlo, jq), mhq = __shfl_sync(FULL, mhi, jq);
                        const uint64_t i_lo = (mlq + 1) >> 1, i_hi = (mhq - 1) >> 1;
                        uint32_t neg = 0, vm = 0;
                        uint64_t g4 = 0;
                        if (f < tot_g) {
                            g4 = (i_lo >> 2) + (f - exq);
                            vm = valid_group(__ldg(reinterpret_cast<const int4 *>(MU) + g4), g4, i_lo, i_hi, p, &neg);
                        }
                        uint32_t off;
                        const uint32_t tot_r = warp_place((uint32_t)__popc(vm), lane, off);
                        if (nbuf + tot_r > cap) flush();
                        uint32_t kk = nbuf + off;
                        while (vm) {
                            const int kq = __ffs(vm) - 1;
                            vm &= vm - 1;
                            lbuf[kk++] = make_uint2((uint32_t)(2 * (4 * g4 + kq) + 1), jq | (((neg >> kq) & 1u) << 31));
                        }
                        nbuf += tot_r;
                    }
                }
                flush();
                if (cur != 0xFFu) {
                    atomicAdd(s_sum + cur, (unsigned long long)csum);
                    atomicAdd(s_ms + cur, cms);
                }
                __syncwarp();
                // the level's sums of this lane's query: Sum(-mu)(carry + count)
                if (lane < nq) {
                    const i128 v = (i128)(int64_t)s_sum[lane] + (i128)C * (i128)s_ms[lane];
                    if (v) cpx_atomic_add_i128(s_acc + 2 * tq, v);
                    s_sum[lane] = 0;
                    s_ms[lane] = 0;
                }
                __syncwarp();
                }
            }
            }  // groups
            // ---- cross off p_b in the sub-segment
            cross_off(bm, cnt8, p, __shfl_sync(FULL, lr0, k), __shfl_sync(FULL, li0, k), c0, cw0, CPT, s,
                      CPT * 32 * warp, lane, Lw);
            __syncwarp();
        }
    }
    __syncthreads();  // every warp is past its levels: the block's sums are complete
    for (uint32_t t = tid; t < ngr * 32; t += T) {
        if (s_qj[t] == 0xFFFFFFFFu) continue;
        const i128 v = (i128)(((u128)s_acc[2 * t + 1] << 64) | s_acc[2 * t]);
        if (v) acc_add(acc, s_qj[t], ACC_HARD, v);
    }
}

// The kernel: one CTA per unit (next null), or a persistent grid whose CTAs
// take units in order from the device counter `next` (segment-major, so that
// the heaviest units start first and no CTA waits at the end for a late wave).
template <class XT, int TMAX, int MINB>
__global__ void __launch_bounds__(TMAX, MINB) k_hard_shared(unsigned long long *__restrict__ next, CPX_HS_PARAMS)
{
    if (!next) {
        if (blockIdx.x < total) hard_shared_unit<XT>(blockIdx.x, CPX_HS_ARGS);
        return;
    }
    __shared__ unsigned long long s_k;
    for (;;) {
        __syncthreads();  // every thread is done with the previous unit's shared memory
        if (threadIdx.x == 0) s_k = atomicAdd(next, 1ull);
        __syncthreads();
        const unsigned long long k = s_k;
        if (k >= total) return;
        hard_shared_unit<XT>(k, CPX_HS_ARGS);
    }
}

// ------------------------------------------------------------------ launchers

size_t hard_shared_smem_bytes(uint32_t lbits, uint32_t threads) { return shared_smem(lbits, threads); }

// blocks of k_hard_shared one SM's shared memory holds (1 KB of each is the
// runtime's reservation)
static int shared_blocks_per_sm(const cpx_ctx *ctx, uint32_t lbits, uint32_t threads)
{
    const size_t per = shared_smem(lbits, threads) + 1024;
    return (int)std::max<size_t>(1, (ctx->smem_per_sm ? ctx->smem_per_sm : 233472) / per);
}

template <class XT> static void shared_go(cpx_ctx *ctx, const Plan &pl)
{
    const Tables &tb = ctx->tab;
    const uint32_t T = pl.hard_threads;
    const uint32_t lbits_sub = pl.sh_lbits - (uint32_t)(__builtin_ctz(T) - 5);
    if (pl.time_hard) CPX_CUDA(cudaEventRecord(ctx->ev_hard0, ctx->stream));
    if (pl.sh_nlv) {
        {
            KSpan ks(ctx, "k_sieve_counts");
            k_sieve_counts<<<(unsigned)pl.sh_nseg, T, counts_smem(pl.sh_lbits), ctx->stream>>>(
                pl.sh_nseg, pl.sh_lbits, pl.sh_xmax, pl.sh_r4max, pl.c, tb.P, (uint32_t)tb.prm_n, pl.lvl_off,
                pl.sh_nlv, pl.carry);
        }
        CPX_LAUNCH("k_sieve_counts");
        k_carry_scan<<<pl.sh_nlv, 1024, 0, ctx->stream>>>(pl.sh_nlv, pl.c, 2ull << pl.sh_lbits, tb.P, tb.T, pl.lvl_off,
                                                           pl.carry);
        CPX_LAUNCH("k_carry_scan");
        note_launch(ctx, 2);
    }
    if (pl.max_jobs) {
        CPX_CUDA(cudaMemsetAsync(pl.njobs, 0, 2 * sizeof(uint64_t), ctx->stream));  // job and snapshot counters
        CPX_CUDA(cudaMemsetAsync(pl.job_units, 0, (pl.max_jobs + 1) * sizeof(uint64_t), ctx->stream));
    }
    XT *gxp = static_cast<XT *>(pl.gxp);
    const uint64_t ntab = (uint64_t)pl.n_grp * pl.sh_nlv * 32;
    if (ntab) {
        k_group_levels<XT><<<(unsigned)((ntab + 255) / 256), 256, 0, ctx->stream>>>(pl.qd, pl.grp, pl.n_grp,
                                                                                    pl.sh_nlv, pl.c, tb.P, gxp, pl.gae);
        CPX_LAUNCH("k_group_levels");
        note_launch(ctx);
    }
    {
        KSpan ks(ctx, "k_hard_shared");
        // minb: the variant's resident blocks per SM (its launch bound; the
        // shared memory fits them), the persistent grid's CTAs per SM
        auto go = [&](auto kern, int minb) {
            const size_t smem = shared_smem(pl.sh_lbits, T);
            unsigned grid = (unsigned)pl.n_gunits;
            if (pl.unit_next) grid = (unsigned)std::min<uint64_t>(pl.n_gunits, (uint64_t)minb * ctx->sm_count);
            kern<<<grid, T, smem, ctx->stream>>>(pl.unit_next, pl.qd, pl.grp, pl.units, pl.n_gunits, pl.sh_lbits, pl.c, tb.P,
                (uint32_t)tb.prm_n, tb.MU, tb.T, pl.lvl_off, pl.sh_nlv, pl.carry, pl.acc, pl.jobs, pl.njobs,
                pl.job_units, pl.snap, pl.nsnap, pl.max_jobs, lbits_sub,
                (uint32_t)std::min<uint64_t>(pl.offload_min, 0xFFFFFFFFull), gxp, pl.gae);
        };
        const int fit = shared_blocks_per_sm(ctx, pl.sh_lbits, T);
        if (T > 512) go(k_hard_shared<XT, 1024, 1>, 1);
        else if (T > 256) fit >= 2 ? go(k_hard_shared<XT, 512, 2>, 2) : go(k_hard_shared<XT, 512, 1>, 1);
        else fit >= 4 ? go(k_hard_shared<XT, 256, 4>, 4) : go(k_hard_shared<XT, 256, 2>, std::min(fit, 2));
    }
    CPX_LAUNCH("k_hard_shared");
    note_launch(ctx);
    if (pl.max_jobs) launch_hard_leaves(ctx, pl, lbits_sub);
    if (pl.time_hard) CPX_CUDA(cudaEventRecord(ctx->ev_hard1, ctx->stream));
}

// the largest dynamic shared memory a kernel may ask for: the device's opt-in
// maximum less the kernel's static shared memory
template <class K> static void raise_dyn_smem(K *kernel, size_t optin)
{
    cudaFuncAttributes fa;
    CPX_CUDA(cudaFuncGetAttributes(&fa, kernel));
    CPX_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(optin - fa.sharedSizeBytes)));
}

// raises the dynamic shared-memory limits once per device (see prepare_hard)
void prepare_hard_shared(cpx_ctx *ctx, const Plan &pl)
{
    if (!pl.n_gunits) return;
    if (shared_smem(pl.sh_lbits, pl.hard_threads) + 64 > ctx->smem_optin)
        fail(CPX_EINVAL, "shared hard-leaf segment needs more shared memory than a block can have");
    static std::mutex m;
    static int done_dev[2] = {-1, -1};
    std::lock_guard<std::mutex> g(m);
    const int w = pl.wide ? 1 : 0;
    if (done_dev[w] == ctx->device) return;
    raise_dyn_smem(k_sieve_counts, ctx->smem_optin);
    auto raise_all = [&](auto xt) {
        using XT = decltype(xt);
        raise_dyn_smem(k_hard_shared<XT, 1024, 1>, ctx->smem_optin);
        raise_dyn_smem(k_hard_shared<XT, 512, 1>, ctx->smem_optin);
        raise_dyn_smem(k_hard_shared<XT, 512, 2>, ctx->smem_optin);
        raise_dyn_smem(k_hard_shared<XT, 256, 2>, ctx->smem_optin);
        raise_dyn_smem(k_hard_shared<XT, 256, 4>, ctx->smem_optin);
    };
    if (pl.wide) raise_all(u128());
    else raise_all(uint64_t());
    done_dev[w] = ctx->device;
}

void launch_hard_shared(cpx_ctx *ctx, const Plan &pl)
{
    if (!pl.n_gunits) return;
    if (pl.n_gunits > 0x7FFFFFFFull || pl.sh_nseg > 0x7FFFFFFFull)
        fail(CPX_ERANGE, "too many hard-leaf segments in one launch");
    if (pl.wide) shared_go<u128>(ctx, pl);
    else shared_go<uint64_t>(ctx, pl);
}

}  // namespace cpx
