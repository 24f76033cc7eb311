// hard.cu -- hard special leaves: the segmented phi sieve.
//
// Restates the reference's hard-leaf sieve (S2hardHost / S2ctl,
// src/sieve/S2_hard_host.cu:49-191, src/sieve/S2_hard_device.cu:12-382) with
// this library's exact leaf split: a leaf (b, m) is hard when
// u = x/(p_b m) >= p_b^2, i.e. p_b <= iroot4(x) and m <= x/p_b^3; it
// contributes -mu(m) phi(u, b-1), which the sieve answers from the bitmap of
// the segment holding u plus the survivors of level b-1 below it.
//
// One CTA owns one segment of 2^lbits odd numbers n = lo + 2i + 1; each of its
// warps owns a contiguous sub-segment as a bitmap in shared memory with one
// 8-bit survivor counter per 16-byte chunk (128 numbers), and walks the levels
// b = c+1 .. B(seg) on its own, synchronising only inside the warp.  Per
// level a warp (1) records its survivor count at level b-1, (2) if its
// sub-segment holds leaves of p_b, scans the counters into lane prefixes and
// answers each leaf as lane prefix + earlier counters of the owning lane +
// popcounts in the chunk -- or, for a large candidate range, hands the level
// to k_hard_leaves with a snapshot of the sub-segment, (3) crosses off p_b,
// counting cleared bits and keeping the counters current.  The level
// parameters (x/p, candidate range, first multiple) are computed 32 levels at
// a time, one level per lane, and broadcast by shuffles.  Every 32 levels the
// CTA combines its warps: carries between sub-segments enter the hard sum and
// the per-segment (count, Sum(-mu)) pairs go to k_hard_combine, which adds the
// carries between segments.
//
// This is the sieve of lone queries and small batches.  Larger batches share
// the sieve between queries (hard_shared.cu); k_hard_leaves serves both.
#include <algorithm>
#include <mutex>

#include "sieve.cuh"

namespace cpx {

template <class XT>
__global__ void __launch_bounds__(512, 2) k_hard(const QD *__restrict__ qd, uint32_t Q,
                                              const uint64_t *__restrict__ pre_seg, uint64_t total,
                                              const uint32_t *__restrict__ seg_B,
                                              const uint64_t *__restrict__ seg_off,
                                              const uint32_t *__restrict__ P, const int32_t *__restrict__ MU,
                                              const cpx_pient *__restrict__ Tpi,
                                              uint32_t *__restrict__ out_cnt, int32_t *__restrict__ out_ms,
                                              uint64_t cap, unsigned long long *__restrict__ acc,
                                              uint32_t lbits_max, HardJob *__restrict__ jobs,
                                              unsigned int *__restrict__ njobs, uint64_t *__restrict__ job_units,
                                              unsigned char *__restrict__ snap, uint32_t max_jobs,
                                              uint32_t lbits_sub_max, uint32_t offload_min)
{
    extern __shared__ uint4 smem4[];
    const uint64_t unit = blockIdx.x;
    if (unit >= total) return;
    const uint32_t B = seg_B[unit];
    const uint32_t q = find_q(pre_seg, Q, unit);
    const QD &d = qd[q];
    const uint32_t c = d.c;
    if (B <= c) return;  // uniform over the CTA
    const uint32_t T = blockDim.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, NW = T >> 5;
    const uint32_t L = 1u << d.lbits;
    const uint32_t NC = L >> 7;    // chunks of the segment
    const uint32_t CPT = NC / T;   // chunks per lane (>= 1)
    const int s = __ffs(CPT) - 1;  // log2 CPT
    const uint32_t Lw = L / NW;    // bits of a warp's sub-segment
    const uint64_t seg = unit - pre_seg[q] + d.seg0;
    const uint64_t lo = seg * 2 * (uint64_t)L;
    const uint64_t lo_w = lo + 2 * (uint64_t)Lw * warp, hi_w = lo_w + 2 * (uint64_t)Lw;
    const bool q41 = hi_w <= (1ull << 41);  // leaf quotients lie in [lo_w, hi_w)
    const uint64_t off = seg_off[unit];
    if (off + (B - c) > cap) return;  // the host sized the ragged outputs exactly; never write past them
    const XT x = xload<XT>(d);
    const uint64_t y = d.y;

    // carve the shared block (sized for lbits_max)
    unsigned char *sp = reinterpret_cast<unsigned char *>(smem4);
    const size_t Lmax = size_t(1) << lbits_max;
    uint32_t *bm = reinterpret_cast<uint32_t *>(sp);
    size_t o = Lmax / 8;
    uint8_t *cnt8 = reinterpret_cast<uint8_t *>(sp + o);
    o += ((Lmax / 128) + 15) & ~size_t(15);
    uint32_t *loff = reinterpret_cast<uint32_t *>(sp + o);  // [NW][32] lane prefixes
    o += T * 4;
    LvlOut *area = reinterpret_cast<LvlOut *>(sp + o);      // [2][NW][32]
    o += 2 * NW * 32 * sizeof(LvlOut);
    o = (o + 15) & ~size_t(15);
    i128 *s_red = reinterpret_cast<i128 *>(sp + o);
    o += 32 * sizeof(i128);
    uint32_t *lbuf = reinterpret_cast<uint32_t *>(sp + o) + kLeafBuf * warp;  // this warp's gathered leaves
    uint32_t *wl = loff + 32 * warp;  // this warp's lane prefixes

    const uint32_t c0 = CPT * tid;  // first owned chunk (of the segment)
    const uint32_t cw0 = c0 - CPT * 32 * warp;  // first owned chunk of the sub-segment
    // ---- pre-sieve with p_2 .. p_c; chunk counters
    const uint32_t cnt0 = presieve(bm, cnt8, P, c, lo, c0, CPT, s);
    uint32_t tot = __reduce_add_sync(FULL, cnt0);  // survivors of this warp's sub-segment
    __syncwarp();

    const BoundDiv bd_lo = bound_div(lo_w), bd_hi = bound_div(hi_w);
    auto sub_count = [&](uint64_t uu) -> uint32_t { return sub_survivors(uu, lo_w, wl, cnt8, bm, CPT, s, warp); };

    int64_t S = 0;       // this lane's share of the hard sum (survivor counts within sub-segments)
    i128 Sx = 0;         // warp 0: carries between the CTA's sub-segments
    uint32_t grp = 0;
    for (uint32_t gb = c + 1; gb <= B; gb += 32, grp++) {
        const uint32_t nl = min(32u, B - gb + 1);
        // ---- level parameters, one level per lane
        LvlPar<XT> lv;
        lv.p = 0;
        lv.mlo = lv.mhi = lv.r0 = 0;
        lv.i0 = 0xFFFFFFFFu;
        lv.xp = 0;
        if (lane < nl) level_params<XT>(lv, x, y, P[gb + lane - 1], lo_w, hi_w, bd_lo, bd_hi);
        const uint32_t lp = lv.p, lmlo = lv.mlo, lmhi = lv.mhi, lr0 = lv.r0, li0 = lv.i0;
        const XT lxp = lv.xp;
        // levels of the block with candidates in the sub-segment (most levels of
        // the high segments have none: they only cross off)
        const unsigned act = __ballot_sync(FULL, lane < nl && lv.mhi > lv.mlo);
        LvlOut mine = {0, 0, 0xFFFFFFFFu, 0};
        for (uint32_t k = 0; k < nl; k++) {
            const uint32_t b = gb + k;
            const uint32_t p = __shfl_sync(FULL, lp, k);
            const uint32_t cnt_b = tot;
            int32_t ms_b = 0;
            uint32_t job_b = 0xFFFFFFFFu;
            if ((act >> k) & 1u) {
                const uint32_t mlo = __shfl_sync(FULL, lmlo, k), mhi = __shfl_sync(FULL, lmhi, k);
                XT xp;
                if (sizeof(XT) == 8) {
                    xp = (XT)__shfl_sync(FULL, (unsigned long long)lxp, k);
                } else {
                    const unsigned long long a0 = __shfl_sync(FULL, (unsigned long long)lxp, k);
                    const unsigned long long a1 = __shfl_sync(FULL, (unsigned long long)((u128)lxp >> 64), k);
                    xp = (XT)(((u128)a1 << 64) | a0);
                }
                // lane prefixes of the sub-segment from the chunk counters
                const uint32_t run = counter_sum(cnt8 + c0, CPT);
                uint32_t inc = run;
#pragma unroll
                for (int oo = 1; oo < 32; oo <<= 1) {
                    const uint32_t t = __shfl_up_sync(FULL, inc, oo);
                    if (lane >= (uint32_t)oo) inc += t;
                }
                wl[lane] = inc - run;
                __syncwarp();
                const bool prime_lvl = (uint64_t)p * p > y;
                const uint64_t qa = mlo > p ? mlo : p;
                uint64_t work;
                if (prime_lvl) work = (mhi > qa) ? 8 * ((((uint64_t)mhi - 1) >> 7) - (qa >> 7) + 1) : 0;
                else work = ((((uint64_t)mhi - 1) >> 1) - (((uint64_t)mlo + 1) >> 1) + 1);
                bool offloaded = false;
                if (max_jobs && offload_min && work >= offload_min) {
                    unsigned int j = 0;
                    if (lane == 0) j = atomicAdd(njobs, 1u);
                    j = __shfl_sync(FULL, j, 0);
                    if (j < max_jobs) {
                        offloaded = true;
                        job_b = j;
                        const size_t stride = snap_stride(lbits_sub_max);
                        uint4 *sb = reinterpret_cast<uint4 *>(snap + (size_t)j * stride);
                        uint32_t *spre = reinterpret_cast<uint32_t *>(sb + ((size_t(1) << lbits_sub_max) >> 7));
                        snapshot_chunks(sb, spre, bm, cnt8, cw0, c0, CPT, s, wl[lane]);
                        if (lane == 0) {
                            HardJob J;
                            J.q = q;
                            J.b = b;
                            J.p = p;
                            J.kind = prime_lvl ? 1u : 0u;
                            J.mlo = prime_lvl ? qa : mlo;
                            J.mhi = mhi;
                            J.lo = lo_w;
                            J.slot = off + (b - c - 1);
                            J.nunits = prime_lvl ? (work / 8 + kJobWords - 1) / kJobWords
                                                 : (((((uint64_t)mhi - 1) >> 1) >> 2) -
                                                    ((((uint64_t)mlo + 1) >> 1) >> 2) + kJobGroups) /
                                                       kJobGroups;
                            J.carry = 0;  // filled in by the group combine below
                            J.snap = j;
                            job_units[j] = J.nunits;
                            J.xp = (u128)xp;
                            jobs[j] = J;
                        }
                    }
                }
                if (!offloaded) {
                    // The lanes gather the level's leaves (m, with bit 31 set when
                    // mu(m) = -1) into the warp's buffer and answer them 32 at a time,
                    // so that a lane with many candidates does not hold up the others.
                    int32_t msl = 0;
                    uint32_t nbuf = 0;
                    const double xpd = (double)(uint64_t)xp;
                    auto flush = [&] {
                        __syncwarp();
                        for (uint32_t jj = lane; jj < nbuf; jj += 32) {
                            const uint32_t e = lbuf[jj];
                            const uint32_t cv = sub_count(leaf_quot(xp, xpd, e & 0x7FFFFFFFu, q41));
                            if (e >> 31) {
                                S += cv;
                                msl += 1;
                            } else {
                                S -= cv;
                                msl -= 1;
                            }
                        }
                        __syncwarp();
                        nbuf = 0;
                    };
                    auto place = [&](uint32_t n, uint32_t &off) -> uint32_t { return warp_place(n, lane, off); };
                    if (prime_lvl) {
                        // m must be a prime q > p: walk the pi-table bitmap of (max(mlo, p), mhi]
                        if (mhi > qa) {
                            const uint64_t w0q = qa >> 7, w1q = ((uint64_t)mhi - 1) >> 7;
                            for (uint64_t wb = w0q; wb <= w1q; wb += 32) {
                                const uint64_t wq = wb + lane;
                                uint64_t qb = 0;
                                if (wq <= w1q)
                                    qb = __ldg(reinterpret_cast<const ulonglong2 *>(Tpi) + wq).x & range_mask(wq, qa, mhi);
                                uint32_t off;
                                const uint32_t tot_r = place((uint32_t)__popcll(qb), off);
                                if (tot_r > kLeafBuf) {  // a dense round: each lane answers its own word
                                    while (qb) {
                                        const int j = __ffsll((long long)qb) - 1;
                                        qb &= qb - 1;
                                        S += sub_count(leaf_quot(xp, xpd, 128 * wq + 2 * j + 1, q41));  // mu(q) = -1
                                        msl += 1;
                                    }
                                    continue;
                                }
                                if (nbuf + tot_r > kLeafBuf) flush();
                                uint32_t kk = nbuf + off;
                                while (qb) {
                                    const int j = __ffsll((long long)qb) - 1;
                                    qb &= qb - 1;
                                    lbuf[kk++] = (uint32_t)(128 * wq + 2 * j + 1) | 0x80000000u;
                                }
                                nbuf += tot_r;
                            }
                        }
                    } else {
                        // any squarefree m with lpf(m) > p: 16-byte loads of packed mu*lpf
                        const uint64_t i_lo = ((uint64_t)mlo + 1) >> 1, i_hi = ((uint64_t)mhi - 1) >> 1;
                        for (uint64_t gb = i_lo >> 2; gb <= (i_hi >> 2); gb += 32) {
                            const uint64_t g = gb + lane;
                            uint32_t neg = 0, vm = 0;
                            if (g <= (i_hi >> 2))
                                vm = valid_group(__ldg(reinterpret_cast<const int4 *>(MU) + g), g, i_lo, i_hi, p, &neg);
                            uint32_t off;
                            const uint32_t tot_r = place((uint32_t)__popc(vm), off);
                            if (nbuf + tot_r > kLeafBuf) flush();
                            uint32_t kk = nbuf + off;
                            while (vm) {
                                const int kq = __ffs(vm) - 1;
                                vm &= vm - 1;
                                lbuf[kk++] = (uint32_t)(2 * (4 * g + kq) + 1) | (((neg >> kq) & 1u) << 31);
                            }
                            nbuf += tot_r;
                        }
                    }
                    flush();
                    ms_b = __reduce_add_sync(FULL, msl);
                }
                __syncwarp();
            }
            // ---- cross off p_b in the sub-segment
            const uint32_t cleared = cross_off<true>(bm, cnt8, p, __shfl_sync(FULL, lr0, k), __shfl_sync(FULL, li0, k), c0, cw0,
                                               CPT, s, CPT * 32 * warp, lane, Lw);
            tot -= __reduce_add_sync(FULL, cleared);
            __syncwarp();
            if (lane == k) {
                mine.cnt = cnt_b;
                mine.ms = ms_b;
                mine.job = job_b;
            }
        }
        // ---- combine the warps of the CTA for these 32 levels
        LvlOut *ar = area + (grp & 1) * NW * 32;
        ar[warp * 32 + lane] = mine;
        __syncthreads();
        if (warp == 0 && lane < nl) {
            const uint32_t b = gb + lane;
            uint64_t carry = 0;
            int32_t msum = 0;
            for (uint32_t w = 0; w < NW; w++) {
                const LvlOut e = ar[w * 32 + lane];
                Sx += (i128)carry * e.ms;
                if (e.job != 0xFFFFFFFFu) jobs[e.job].carry = carry;
                carry += e.cnt;
                msum += e.ms;
            }
            out_cnt[off + (b - c - 1)] = (uint32_t)carry;
            out_ms[off + (b - c - 1)] = msum;
        }
    }
    const i128 Sb = cpx_block_sum_i128((i128)S + Sx, s_red);
    if (tid == 0) acc_add(acc, q, ACC_HARD, Sb);
}

// Leaves of the offloaded (segment, level) sets.  A warp takes one unit: 256
// pi-table entries of prime m (prime-only levels) or 256 groups of 4 odd m
// read as packed mu*lpf (other levels).  Each leaf's survivor count is the
// job's carry plus the snapshot's chunk prefix plus popcounts inside the
// 16-byte chunk; the sums go to the query's hard-leaf accumulator and
// Sum(-mu) to the level's slot (none when slot = ~0: the carry was complete).
template <class XT>
__global__ void __launch_bounds__(kThreads) k_hard_leaves(const HardJob *__restrict__ jobs,
                                                          const unsigned int *njobs, uint32_t max_jobs,
                                                          const uint64_t *__restrict__ unit0,
                                                          const unsigned char *__restrict__ snap,
                                                          uint32_t lbits_sub, const int32_t *__restrict__ MU,
                                                          const cpx_pient *__restrict__ Tpi,
                                                          int32_t *__restrict__ out_ms,
                                                          unsigned long long *__restrict__ acc)
{
    const uint32_t n = min(*njobs, max_jobs);
    const uint64_t total = unit0[max_jobs];  // exclusive scan of the units; slots past n hold 0
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t gw = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    const size_t stride = snap_stride(lbits_sub);
    const size_t ncmax = (size_t(1) << lbits_sub) >> 7;
    __shared__ uint32_t s_leaf[kThreads / 32][kLeafBuf];
    uint32_t *lbuf = s_leaf[threadIdx.x >> 5];
    for (uint64_t unit = gw; unit < total; unit += nw) {
        uint32_t lo_j = 0, hi_j = n;  // unit0[lo_j] <= unit < unit0[hi_j]
        while (hi_j - lo_j > 1) {
            const uint32_t mid = (lo_j + hi_j) >> 1;
            if (__ldg(unit0 + mid) <= unit) lo_j = mid;
            else hi_j = mid;
        }
        const HardJob &J = jobs[lo_j];
        const uint64_t lu = unit - __ldg(unit0 + lo_j);
        const uint4 *sb = reinterpret_cast<const uint4 *>(snap + (size_t)J.snap * stride);
        const uint32_t *spre = reinterpret_cast<const uint32_t *>(sb + ncmax);
        const XT xp = (XT)J.xp;
        const double xpd = (double)(uint64_t)xp;
        const uint64_t lo = J.lo;
        const bool q41 = lo + (2ull << lbits_sub) <= (1ull << 41);  // the sub-segment ends below 2^41
        // survivors of the sub-segment with n <= uu (the carry is added per unit)
        auto count = [&](uint64_t uu) -> uint32_t {
            const uint32_t kk = (uint32_t)((uu - lo + 1) >> 1);
            if (!kk) return 0u;  // u = lo: no number of the sub-segment is <= u
            const uint32_t jb = kk - 1, w = jb >> 5, ch = w >> 2;
            return __ldg(spre + ch) + chunk_survivors(__ldg(sb + ch), jb);
        };
        int64_t S = 0;
        int32_t ms = 0;
        // leaves gathered into the warp's buffer (m, bit 31: mu(m) = -1) and
        // answered 32 at a time, as in k_hard
        uint32_t nbuf = 0;
        auto flush = [&] {
            __syncwarp();
            for (uint32_t jj = lane; jj < nbuf; jj += 32) {
                const uint32_t e = lbuf[jj];
                const uint32_t cv = count(leaf_quot(xp, xpd, e & 0x7FFFFFFFu, q41));
                if (e >> 31) {
                    S += cv;
                    ms += 1;
                } else {
                    S -= cv;
                    ms -= 1;
                }
            }
            __syncwarp();
            nbuf = 0;
        };
        auto place = [&](uint32_t cnt, uint32_t &off) -> uint32_t {
            uint32_t inc = cnt;
#pragma unroll
            for (int oo = 1; oo < 32; oo <<= 1) {
                const uint32_t t = __shfl_up_sync(FULL, inc, oo);
                if (lane >= (uint32_t)oo) inc += t;
            }
            off = inc - cnt;
            return __shfl_sync(FULL, inc, 31);
        };
        if (J.kind == 1) {
            const uint64_t qa = J.mlo, mhi = J.mhi;
            const uint64_t w0 = (qa >> 7) + lu * kJobWords, wl = (mhi - 1) >> 7;
            for (uint64_t k = 0; k < kJobWords / 32; k++) {
                if (w0 + 32 * k > wl) break;  // uniform
                const uint64_t wq = w0 + 32 * k + lane;
                uint64_t qb = 0;
                if (wq <= wl) qb = __ldg(reinterpret_cast<const ulonglong2 *>(Tpi) + wq).x & range_mask(wq, qa, mhi);
                uint32_t off;
                const uint32_t tot_r = place((uint32_t)__popcll(qb), off);
                if (tot_r > kLeafBuf) {  // a dense round: each lane answers its own word
                    while (qb) {
                        const int j = __ffsll((long long)qb) - 1;
                        qb &= qb - 1;
                        S += count(leaf_quot(xp, xpd, 128 * wq + 2 * j + 1, q41));  // mu(q) = -1
                        ms += 1;
                    }
                    continue;
                }
                if (nbuf + tot_r > kLeafBuf) flush();
                uint32_t kk = nbuf + off;
                while (qb) {
                    const int j = __ffsll((long long)qb) - 1;
                    qb &= qb - 1;
                    lbuf[kk++] = (uint32_t)(128 * wq + 2 * j + 1) | 0x80000000u;
                }
                nbuf += tot_r;
            }
        } else {
            const uint64_t i_lo = (J.mlo + 1) >> 1, i_hi = (J.mhi - 1) >> 1;
            const uint64_t g0 = (i_lo >> 2) + lu * kJobGroups, gl = i_hi >> 2;
            const uint32_t p = J.p;
            for (uint64_t k = 0; k < kJobGroups / 32; k++) {
                if (g0 + 32 * k > gl) break;  // uniform
                const uint64_t g = g0 + 32 * k + lane;
                uint32_t neg = 0, vm = 0;
                if (g <= gl) vm = valid_group(__ldg(reinterpret_cast<const int4 *>(MU) + g), g, i_lo, i_hi, p, &neg);
                uint32_t off;
                const uint32_t tot_r = place((uint32_t)__popc(vm), off);
                if (nbuf + tot_r > kLeafBuf) flush();
                uint32_t kk = nbuf + off;
                while (vm) {
                    const int kq = __ffs(vm) - 1;
                    vm &= vm - 1;
                    lbuf[kk++] = (uint32_t)(2 * (4 * g + kq) + 1) | (((neg >> kq) & 1u) << 31);
                }
                nbuf += tot_r;
            }
        }
        flush();
        const i128 Sw = cpx_warp_sum_i128((i128)S);
#pragma unroll
        for (int dd = 16; dd > 0; dd >>= 1) ms += __shfl_down_sync(FULL, ms, dd);
        if (lane == 0) {
            if (ms && J.slot != ~0ull) atomicAdd(out_ms + J.slot, ms);
            acc_add(acc, J.q, ACC_HARD, Sw + (i128)J.carry * ms);
        }
    }
}

// B(seg) of every work unit (seg_levels) and its level count max(0, B - c).
template <class XT>
__global__ void k_hard_plan(const QD *__restrict__ qd, uint32_t Q, const uint64_t *__restrict__ pre_seg,
                            uint64_t total, const uint32_t *__restrict__ P, uint32_t np,
                            uint32_t *__restrict__ seg_B, uint64_t *__restrict__ seg_lv)
{
    const uint64_t u = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= total) return;
    const uint32_t q = find_q(pre_seg, Q, u);
    const QD &d = qd[q];
    const uint64_t seg = u - pre_seg[q] + d.seg0;
    const uint64_t lo = seg * 2 * (1ull << d.lbits), hi = lo + 2 * (1ull << d.lbits);
    const uint32_t a = seg_levels<XT>(xload<XT>(d), d.r4, lo, hi, P, np);
    seg_B[u] = a;
    seg_lv[u] = a > d.c ? a - d.c : 0;
}

// H += sum over segments of carry(seg, b) * msum(seg, b); carry = count of
// survivors of level b-1 below the segment.  Level b is sieved from the first
// segment reaching p_b^2; below p_b^2 the survivors of level b-1 are 1 and the
// primes from p_b on, so the carry starts at 1 + max(0, pi(lo - 1) - (b - 1))
// from the pi table and then adds the sieved segments' counts.  One warp per
// (query, b): its lanes take 32 consecutive segments at a time and a warp
// scan of their counts gives each segment its carry.  The segments sieving
// level b are contiguous from the first one.
__global__ void k_hard_combine(const QD *__restrict__ qd, uint32_t Q, const uint64_t *__restrict__ pre_comb,
                               uint64_t total, const uint64_t *__restrict__ pre_seg,
                               const uint32_t *__restrict__ seg_B, const uint64_t *__restrict__ seg_off,
                               const uint32_t *__restrict__ cnt, const int32_t *__restrict__ ms, uint64_t cap,
                               const uint32_t *__restrict__ P, const cpx_pient *__restrict__ T,
                               unsigned long long *__restrict__ acc, HardLevel *__restrict__ lvl_out)
{
    const uint64_t u = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t lane = threadIdx.x & 31;
    if (u >= total) return;  // uniform over the warp
    const uint32_t q = find_q(pre_comb, Q, u);
    const uint64_t lvl = u - pre_comb[q];
    const QD &d = qd[q];
    const uint32_t b = d.c + 1 + (uint32_t)lvl;
    const uint64_t span = 2ull << d.lbits;
    const uint64_t p = P[b - 1];
    const uint64_t first = (p * p) / span;  // first segment with hi > p^2
    // the query's segments here are seg0 .. seg0 + n - 1 (all of them unless
    // the query is split over GPUs); carries below the part come from outside
    const uint64_t g0 = d.seg0, g1 = d.seg0 + (pre_seg[q + 1] - pre_seg[q]);
    const uint64_t fl = first > g0 ? first : g0;
    const uint64_t s0 = pre_seg[q] + (fl - g0), s1 = pre_seg[q + 1];
    const bool anchored = first >= g0 && first < g1;
    uint64_t carry = 0;
    if (anchored && first > 0) {
        const uint64_t pl = cpx_pi_dev(T, first * span - 1);
        carry = 1 + (pl > b - 1 ? pl - (b - 1) : 0);
    }
    const uint64_t carry0 = carry;
    int64_t msl = 0;
    i128 H = 0;
    for (uint64_t base = s0; base < s1; base += 32) {
        const uint64_t sg = base + lane;
        uint32_t cv = 0;
        int32_t mv = 0;
        bool act = false;
        if (sg < s1 && __ldg(seg_B + sg) >= b) {
            const uint64_t idx = __ldg(seg_off + sg) + lvl;
            if (idx < cap) {
                cv = __ldg(cnt + idx);
                mv = __ldg(ms + idx);
                act = true;
            }
        }
        const unsigned bal = __ballot_sync(FULL, act);
        const int stop = __ffs(~bal) - 1;  // first segment past the level's range (-1: none here)
        if (stop >= 0 && (int)lane >= stop) {
            cv = 0;
            mv = 0;
        }
        uint64_t inc = cv;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint64_t t = __shfl_up_sync(FULL, inc, o);
            if (lane >= (uint32_t)o) inc += t;
        }
        H += (i128)(carry + inc - cv) * (i128)mv;
        msl += mv;
        carry += __shfl_sync(FULL, inc, 31);
        if (stop >= 0) break;
    }
    H = cpx_warp_sum_i128(H);
    if (lane == 0) acc_add(acc, q, ACC_HARD, H);
    if (lvl_out && q == 0) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) msl += __shfl_down_sync(FULL, msl, o);
        if (lane == 0) lvl_out[lvl] = HardLevel{carry - carry0, msl, carry0, anchored ? 1u : 0u, 0u};
    }
}

// ------------------------------------------------------------------ launchers

size_t hard_snapshot_stride(uint32_t lbits_sub) { return snap_stride(lbits_sub); }

size_t hard_smem_bytes(uint32_t lbits, uint32_t threads, bool wide)
{
    (void)wide;
    return hard_smem(lbits, threads);
}

void launch_hard_leaves(cpx_ctx *ctx, const Plan &pl, uint32_t lbits_sub)
{
    const Tables &tb = ctx->tab;
    scan_u64(ctx, pl.job_units, pl.max_jobs + 1);
    if (pl.wide)
        k_hard_leaves<u128><<<(unsigned)ctx->sm_count * 8, kThreads, 0, ctx->stream>>>(
            pl.jobs, pl.njobs, pl.max_jobs, pl.job_units, pl.snap, lbits_sub, tb.MU, tb.T, pl.hard_ms, pl.acc);
    else
        k_hard_leaves<uint64_t><<<(unsigned)ctx->sm_count * 8, kThreads, 0, ctx->stream>>>(
            pl.jobs, pl.njobs, pl.max_jobs, pl.job_units, pl.snap, lbits_sub, tb.MU, tb.T, pl.hard_ms, pl.acc);
    CPX_LAUNCH("k_hard_leaves");
    note_launch(ctx);
}

template <class XT> static void hard_go(cpx_ctx *ctx, const Plan &pl)
{
    const Tables &tb = ctx->tab;
    k_hard_plan<XT><<<(unsigned)((pl.n_seg + 255) / 256), 256, 0, ctx->stream>>>(
        pl.qd, pl.Q, pl.pre_seg, pl.n_seg, tb.P, (uint32_t)tb.prm_n, pl.seg_B, pl.seg_off);
    CPX_LAUNCH("k_hard_plan");
    note_launch(ctx);
    scan_u64(ctx, pl.seg_off, pl.n_seg);
    const size_t smem = hard_smem(pl.lbits_max, pl.hard_threads);
    const uint32_t lbits_sub = pl.lbits_max - (uint32_t)(__builtin_ctz(pl.hard_threads) - 5);
    if (pl.time_hard) CPX_CUDA(cudaEventRecord(ctx->ev_hard0, ctx->stream));
    if (pl.max_jobs) {
        CPX_CUDA(cudaMemsetAsync(pl.njobs, 0, sizeof(unsigned int), ctx->stream));
        CPX_CUDA(cudaMemsetAsync(pl.job_units, 0, (pl.max_jobs + 1) * sizeof(uint64_t), ctx->stream));
    }
    {
        KSpan ks(ctx, "k_hard");
        k_hard<XT><<<(unsigned)pl.n_seg, pl.hard_threads, smem, ctx->stream>>>(
            pl.qd, pl.Q, pl.pre_seg, pl.n_seg, pl.seg_B, pl.seg_off, tb.P, tb.MU, tb.T, pl.hard_cnt, pl.hard_ms,
            pl.hard_entries, pl.acc, pl.lbits_max, pl.jobs, pl.njobs, pl.job_units, pl.snap, pl.max_jobs, lbits_sub,
            (uint32_t)std::min<uint64_t>(pl.offload_min, 0xFFFFFFFFull));
    }
    CPX_LAUNCH("k_hard");
    note_launch(ctx);
    if (pl.max_jobs) launch_hard_leaves(ctx, pl, lbits_sub);
    if (pl.time_hard) CPX_CUDA(cudaEventRecord(ctx->ev_hard1, ctx->stream));
    if (pl.n_comb) {
        k_hard_combine<<<(unsigned)((pl.n_comb * 32 + 255) / 256), 256, 0, ctx->stream>>>(
            pl.qd, pl.Q, pl.pre_comb, pl.n_comb, pl.pre_seg, pl.seg_B, pl.seg_off, pl.hard_cnt, pl.hard_ms,
            pl.hard_entries, tb.P, tb.T, pl.acc, pl.hard_levels);
        CPX_LAUNCH("k_hard_combine");
        note_launch(ctx);
    }
}

// The dynamic shared-memory limit of k_hard is a property of the function,
// shared by every context and thread of the process, so it is raised to the
// device's opt-in maximum once (under a lock) instead of per launch: a lane
// lowering it while another lane launches a larger segment would fail.
void prepare_hard(cpx_ctx *ctx, const Plan &pl)
{
    if (!pl.n_seg) return;
    const size_t smem = hard_smem(pl.lbits_max, pl.hard_threads);
    if (smem > ctx->smem_optin) fail(CPX_EINVAL, "hard-leaf segment needs more shared memory than a block can have");
    static std::mutex m;
    static int done_dev[2] = {-1, -1};
    std::lock_guard<std::mutex> g(m);
    const int w = pl.wide ? 1 : 0;
    if (done_dev[w] == ctx->device) return;
    if (pl.wide)
        CPX_CUDA(cudaFuncSetAttribute(k_hard<u128>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ctx->smem_optin));
    else
        CPX_CUDA(cudaFuncSetAttribute(k_hard<uint64_t>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)ctx->smem_optin));
    done_dev[w] = ctx->device;
}

void launch_hard(cpx_ctx *ctx, const Plan &pl)
{
    if (!pl.n_seg) return;
    if (pl.n_seg > 0x7FFFFFFFull) fail(CPX_ERANGE, "too many hard-leaf segments in one launch");
    if (pl.wide) hard_go<u128>(ctx, pl);
    else hard_go<uint64_t>(ctx, pl);
}

}  // namespace cpx
