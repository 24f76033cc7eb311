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
// Bitmap layout: thread t owns chunks [CPT t, CPT (t+1)); chunk c is stored at
// c ^ ((c >> log2 CPT) & 7) so the owners' 128-bit accesses are free of bank
// conflicts.  Counters are indexed by the unswizzled chunk.
#include <algorithm>
#include <mutex>

#include "kern_common.cuh"

namespace cpx {

__device__ __forceinline__ uint32_t swz(uint32_t c, int s) { return s ? (c ^ ((c >> s) & 7u)) : c; }

// bits k < 32 of a word whose first number is = r (mod p) that are multiples of p
__device__ __forceinline__ uint32_t mult_mask(uint32_t r, uint32_t p, uint32_t Mp)
{
    const uint32_t k0 = (r == 0) ? 0u : ((r & 1u) ? (p - r) >> 1 : p - (r >> 1));
    return k0 < 32 ? (Mp << k0) : 0u;
}
__device__ __forceinline__ uint32_t every_pth_bit(uint32_t p)
{
    uint32_t m = 0;
    for (uint32_t k = 0; k < 32; k += p) m |= 1u << k;
    return m;
}

// sum of the n 8-bit counters starting at c8 (c8 4-byte aligned when n >= 4)
__device__ __forceinline__ uint32_t counter_sum(const uint8_t *c8, uint32_t n)
{
    uint32_t s = 0;
    const uint32_t *cw = reinterpret_cast<const uint32_t *>(c8);
    uint32_t k = 0;
    for (; k < (n >> 2); k++) s = __dp4a(cw[k], 0x01010101u, s);
    const uint32_t rem = n & 3;
    if (rem) {
        if (reinterpret_cast<uintptr_t>(c8) & 3) {
            for (uint32_t i = 0; i < rem; i++) s += c8[4 * k + i];
        } else {
            s = __dp4a(cw[k] & ((1u << (8 * rem)) - 1u), 0x01010101u, s);
        }
    }
    return s;
}

// A level whose candidate range in a warp's sub-segment holds at least
// offload_min odd m (8 per pi-table entry for prime-only levels) is answered
// by k_hard_leaves (cpx_set_hard_offload; 0 keeps every leaf in the sieve).
constexpr uint64_t kJobWords = 256;   // pi-table entries per k_hard_leaves unit (prime levels)
constexpr uint64_t kJobGroups = 256;  // 4-m groups per k_hard_leaves unit (other levels)

// bytes of one snapshot slot of a sub-segment of 2^lbits_sub numbers:
// 16-byte bitmap chunks + 32-bit survivor prefixes
__host__ __device__ __forceinline__ size_t snap_stride(uint32_t lbits_sub)
{
    const size_t nc = (size_t(1) << lbits_sub) >> 7;
    return (nc * 20 + 255) & ~size_t(255);
}

// leaves a warp gathers before answering them 32 at a time
constexpr uint32_t kLeafBuf = 256;

struct LvlOut {
    uint32_t cnt;
    int32_t ms;
    uint32_t job;
    uint32_t pad;
};

__host__ __device__ __forceinline__ size_t hard_smem(uint32_t lbits, uint32_t threads)
{
    const size_t L = size_t(1) << lbits;
    size_t o = L / 8;                                 // bitmap
    o += ((L / 128) + 15) & ~size_t(15);              // chunk counters
    o += threads * 4;                                 // lane prefixes
    o += 2 * (threads / 32) * 32 * sizeof(LvlOut);    // per-warp level outputs, double buffered
    o = (o + 15) & ~size_t(15);
    o += 32 * sizeof(i128);                           // reductions
    o += (threads / 32) * kLeafBuf * 4;               // per-warp gathered leaves
    return o;
}

// Pre-sieve of one lane's chunks [c0, c0 + CPT) of the segment starting at lo
// with p_2 .. p_c (residue masks per 32-bit word); writes the bitmap and the
// chunk counters and returns the lane's survivors.  Runs once per segment, so
// it is kept out of line (instruction-cache footprint of the level loop).
__device__ __noinline__ uint32_t presieve(uint32_t *bm, uint8_t *cnt8, const uint32_t *__restrict__ P, uint32_t c,
                                          uint64_t lo, uint32_t c0, uint32_t CPT, int s)
{
    uint32_t pr[8], rr[8], st[8], Mp[8];
    const uint32_t np = c - 1;
    const uint32_t w0 = 4 * c0;
#pragma unroll
    for (uint32_t i = 0; i < 8; i++) {
        if (i < np) {
            pr[i] = P[i + 1];
            rr[i] = (uint32_t)(((lo + 1) % pr[i] + (64ull * w0) % pr[i]) % pr[i]);
            st[i] = 64u % pr[i];
            Mp[i] = every_pth_bit(pr[i]);
        }
    }
    uint32_t cnt0 = 0;
    for (uint32_t j = 0; j < CPT; j++) {
        uint32_t wv[4];
#pragma unroll
        for (int k = 0; k < 4; k++) {
            uint32_t m = 0;
#pragma unroll
            for (uint32_t i = 0; i < 8; i++) {
                if (i < np) {
                    m |= mult_mask(rr[i], pr[i], Mp[i]);
                    rr[i] += st[i];
                    if (rr[i] >= pr[i]) rr[i] -= pr[i];
                }
            }
            wv[k] = ~m;
        }
        const uint32_t cc = __popc(wv[0]) + __popc(wv[1]) + __popc(wv[2]) + __popc(wv[3]);
        cnt0 += cc;
        cnt8[c0 + j] = (uint8_t)cc;
        reinterpret_cast<uint4 *>(bm)[swz(c0 + j, s)] = make_uint4(wv[0], wv[1], wv[2], wv[3]);
    }
    return cnt0;
}

// Writes one lane's share of a leaf-set snapshot: its chunks of the
// sub-segment bitmap and the survivor prefix of each chunk (pre = survivors of
// the sub-segment before the lane's first chunk).  Out of line: rare path.
__device__ __noinline__ void snapshot_chunks(uint4 *sb, uint32_t *spre, const uint32_t *bm, const uint8_t *cnt8,
                                             uint32_t cw0, uint32_t c0, uint32_t CPT, int s, uint32_t pre)
{
    for (uint32_t jj = 0; jj < CPT; jj++) {
        sb[cw0 + jj] = reinterpret_cast<const uint4 *>(bm)[swz(c0 + jj, s)];
        spre[cw0 + jj] = pre;
        pre += cnt8[c0 + jj];
    }
}

// The valid m of one 16-byte group of packed mu*lpf (4 odd m, indices 4g..4g+3
// within [i_lo, i_hi]): squarefree with lpf > p.  Bit k of *neg: mu(m) = -1.
__device__ __forceinline__ uint32_t valid_group(int4 v4, uint64_t g, uint64_t i_lo, uint64_t i_hi, uint32_t p,
                                                uint32_t *neg)
{
    const int32_t vals[4] = {v4.x, v4.y, v4.z, v4.w};
    uint32_t vm = 0, ng = 0;
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const uint64_t i = 4 * g + k;
        const int32_t v = vals[k];
        const uint32_t av = (uint32_t)(v > 0 ? v : -v);
        if (i >= i_lo && i <= i_hi && v != 0 && av > p) {
            vm |= 1u << k;
            if (v < 0) ng |= 1u << k;
        }
    }
    *neg = ng;
    return vm;
}

// Parameters of one level (p = p_b) for one warp's sub-segment [lo_w, hi_w):
// xp = x/p, the candidate range (mlo, mhi] of m (m > y/p, u = xp/m in the
// sub-segment, m <= x/p^3 for a hard leaf), the residue of lo_w + 1 mod p and
// the bit of the first odd multiple of p (0xFFFFFFFF: none).  Computed for 32
// levels at a time, one per lane; out of line to keep the level loop small.
template <class XT> struct LvlPar {
    XT xp;
    uint32_t p, mlo, mhi, r0, i0;
};

template <class XT>
__device__ __noinline__ void level_params(LvlPar<XT> &o, XT x, uint64_t y, uint64_t p, uint64_t lo_w, uint64_t hi_w)
{
    const XT xp = cpx_qdiv(x, p);
    uint64_t mlo = y / p;
    const XT t1 = cpx_qdiv(xp, hi_w);
    if (t1 > (XT)mlo) mlo = (uint64_t)t1;
    uint64_t mhi = y;
    if (lo_w) {
        const XT t2 = cpx_qdiv(xp, lo_w);
        if (t2 < (XT)mhi) mhi = (uint64_t)t2;
    }
    const XT t3 = cpx_qdiv(xp, p * p);  // hard leaves only: m <= x/p^3
    if (t3 < (XT)mhi) mhi = (uint64_t)t3;
    if (mhi < mlo) mhi = mlo;
    o.p = (uint32_t)p;
    o.xp = xp;
    o.mlo = (uint32_t)mlo;
    o.mhi = (uint32_t)mhi;
    const uint64_t r0 = (lo_w + 1) - cpx_udiv_leaf(lo_w + 1, p) * p;
    o.r0 = (uint32_t)r0;
    uint64_t m = lo_w + 1 + (r0 ? p - r0 : 0);
    if ((m & 1) == 0) m += p;
    o.i0 = (m < hi_w) ? (uint32_t)((m - lo_w - 1) >> 1) : 0xFFFFFFFFu;
}

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

    // survivors of the warp's sub-segment with n <= uu (uu in [lo_w, hi_w))
    auto sub_count = [&](uint64_t uu) -> uint32_t {
        const uint32_t kk = (uint32_t)((uu - lo_w + 1) >> 1);  // bits [0, kk) of the sub-segment
        if (!kk) return 0u;
        const uint32_t jb = kk - 1, w = jb >> 5;
        const uint32_t chs = w >> 2, ow = chs >> s;      // chunk in the sub-segment, owning lane
        const uint32_t ch = chs + CPT * 32 * warp;       // chunk in the segment
        uint32_t cv = wl[ow] + counter_sum(cnt8 + ch - (chs - ow * CPT), chs - ow * CPT);
        const uint4 v4 = reinterpret_cast<const uint4 *>(bm)[swz(ch, s)];
        const uint32_t wi = w & 3, msk = (2u << (jb & 31)) - 1u;
        if (wi == 0) cv += __popc(v4.x & msk);
        else if (wi == 1) cv += __popc(v4.x) + __popc(v4.y & msk);
        else if (wi == 2) cv += __popc(v4.x) + __popc(v4.y) + __popc(v4.z & msk);
        else cv += __popc(v4.x) + __popc(v4.y) + __popc(v4.z) + __popc(v4.w & msk);
        return cv;
    };

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
        if (lane < nl) level_params<XT>(lv, x, y, P[gb + lane - 1], lo_w, hi_w);
        const uint32_t lp = lv.p, lmlo = lv.mlo, lmhi = lv.mhi, lr0 = lv.r0, li0 = lv.i0;
        const XT lxp = lv.xp;
        LvlOut mine = {0, 0, 0xFFFFFFFFu, 0};
        for (uint32_t k = 0; k < nl; k++) {
            const uint32_t b = gb + k;
            const uint32_t p = __shfl_sync(FULL, lp, k);
            const uint32_t mlo = __shfl_sync(FULL, lmlo, k), mhi = __shfl_sync(FULL, lmhi, k);
            XT xp;
            if (sizeof(XT) == 8) {
                xp = (XT)__shfl_sync(FULL, (unsigned long long)lxp, k);
            } else {
                const unsigned long long a0 = __shfl_sync(FULL, (unsigned long long)lxp, k);
                const unsigned long long a1 = __shfl_sync(FULL, (unsigned long long)((u128)lxp >> 64), k);
                xp = (XT)(((u128)a1 << 64) | a0);
            }
            const uint32_t cnt_b = tot;
            int32_t ms_b = 0;
            uint32_t job_b = 0xFFFFFFFFu;
            if (mhi > mlo) {
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
                    auto flush = [&] {
                        __syncwarp();
                        for (uint32_t jj = lane; jj < nbuf; jj += 32) {
                            const uint32_t e = lbuf[jj];
                            const uint32_t cv = sub_count((uint64_t)cpx_qdiv(xp, (uint64_t)(e & 0x7FFFFFFFu)));
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
                    // exclusive offset of this lane's n entries and the warp's total
                    auto place = [&](uint32_t n, uint32_t &off) -> uint32_t {
                        uint32_t inc = n;
#pragma unroll
                        for (int oo = 1; oo < 32; oo <<= 1) {
                            const uint32_t t = __shfl_up_sync(FULL, inc, oo);
                            if (lane >= (uint32_t)oo) inc += t;
                        }
                        off = inc - n;
                        return __shfl_sync(FULL, inc, 31);
                    };
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
                                        S += sub_count((uint64_t)cpx_qdiv(xp, 128 * wq + 2 * j + 1));  // mu(q) = -1
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
            uint32_t cleared = 0;
            if (p < 128) {
                // each lane masks its own words; p < 32 has several multiples per word
                const uint32_t Mp = every_pth_bit(p);
                const uint32_t stp = 64u % p;
                const uint32_t r0 = __shfl_sync(FULL, lr0, k);
                uint32_t r = (r0 + (64u * (cw0 * 4)) % p) % p;  // first owned word of the sub-segment
                for (uint32_t j = 0; j < CPT; j++) {
                    uint4 v = reinterpret_cast<const uint4 *>(bm)[swz(c0 + j, s)];
                    uint32_t a4[4] = {v.x, v.y, v.z, v.w};
                    uint32_t cj = 0;
#pragma unroll
                    for (int kk = 0; kk < 4; kk++) {
                        const uint32_t mk = mult_mask(r, p, Mp);
                        cj += __popc(a4[kk] & mk);
                        a4[kk] &= ~mk;
                        r += stp;
                        if (r >= p) r -= p;
                    }
                    if (cj) {
                        cnt8[c0 + j] = (uint8_t)(cnt8[c0 + j] - cj);
                        reinterpret_cast<uint4 *>(bm)[swz(c0 + j, s)] = make_uint4(a4[0], a4[1], a4[2], a4[3]);
                    }
                    cleared += cj;
                }
            } else {
                // p >= 128: the lanes of one step clear bits p apart, so they touch
                // distinct words and distinct chunk counters (plain read-modify-write)
                const uint32_t i0 = __shfl_sync(FULL, li0, k);
                if (i0 != 0xFFFFFFFFu) {
                    const uint32_t base_ch = CPT * 32 * warp;
                    for (uint64_t i = (uint64_t)i0 + (uint64_t)lane * p; i < Lw; i += 32ull * p) {
                        const uint32_t w = (uint32_t)(i >> 5), bit = 1u << (i & 31);
                        const uint32_t ch = base_ch + (w >> 2);
                        uint32_t *pw = bm + ((swz(ch, s) << 2) | (w & 3));
                        const uint32_t old = *pw;
                        if (old & bit) {
                            *pw = old & ~bit;
                            cleared++;
                            cnt8[ch] = (uint8_t)(cnt8[ch] - 1);
                        }
                    }
                }
            }
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
// snapshot's chunk prefix plus popcounts inside the 16-byte chunk; the sums go
// to the query's hard-leaf accumulator and Sum(-mu) to the level's slot.
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
        const uint4 *sb = reinterpret_cast<const uint4 *>(snap + (size_t)lo_j * stride);
        const uint32_t *spre = reinterpret_cast<const uint32_t *>(sb + ncmax);
        const XT xp = (XT)J.xp;
        const uint64_t lo = J.lo;
        auto count = [&](uint64_t uu) -> uint32_t {
            const uint32_t kk = (uint32_t)((uu - lo + 1) >> 1);
            if (!kk) return (uint32_t)J.carry;  // u = lo: no number of the sub-segment is <= u
            const uint32_t jb = kk - 1, w = jb >> 5, ch = w >> 2;
            uint32_t cv = (uint32_t)J.carry + __ldg(spre + ch);
            const uint4 v4 = __ldg(sb + ch);
            const uint32_t wi = w & 3, msk = (2u << (jb & 31)) - 1u;
            if (wi == 0) cv += __popc(v4.x & msk);
            else if (wi == 1) cv += __popc(v4.x) + __popc(v4.y & msk);
            else if (wi == 2) cv += __popc(v4.x) + __popc(v4.y) + __popc(v4.z & msk);
            else cv += __popc(v4.x) + __popc(v4.y) + __popc(v4.z) + __popc(v4.w & msk);
            return cv;
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
                const uint32_t cv = count((uint64_t)cpx_qdiv(xp, (uint64_t)(e & 0x7FFFFFFFu)));
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
                        S += count((uint64_t)cpx_qdiv(xp, 128 * wq + 2 * j + 1));  // mu(q) = -1
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
            if (ms) atomicAdd(out_ms + J.slot, ms);
            acc_add(acc, J.q, ACC_HARD, Sw);
        }
    }
}

// B(seg) = pi(min(r4, isqrt((x - 1) / lo), isqrt(hi - 1))): the levels b a
// segment sieves.  p_b^2 * lo < x bounds the levels whose leaves can reach
// the segment or a later one; p_b^2 < hi skips the levels whose leaves all lie
// above the segment, because below p_b^2 the carry phi(v, b - 1) is
// 1 + pi(v) - (b - 1) and k_hard_combine reads it from the pi table.
// Levels per segment = max(0, B - c).
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
    const XT x = xload<XT>(d);
    uint64_t v = d.r4;
    if (lo) {
        const uint64_t v1 = cpx_isqrt((u128)((x - 1) / (XT)lo));
        if (v1 < v) v = v1;
    }
    const uint64_t v2 = cpx_isqrt((u128)(hi - 1));
    if (v2 < v) v = v2;
    uint32_t a = 0, bnd = np;  // count of P[i] <= v
    while (a < bnd) {
        const uint32_t mid = (a + bnd) >> 1;
        if (P[mid] <= v) a = mid + 1;
        else bnd = mid;
    }
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
    k_hard<XT><<<(unsigned)pl.n_seg, pl.hard_threads, smem, ctx->stream>>>(
        pl.qd, pl.Q, pl.pre_seg, pl.n_seg, pl.seg_B, pl.seg_off, tb.P, tb.MU, tb.T, pl.hard_cnt, pl.hard_ms,
        pl.hard_entries, pl.acc, pl.lbits_max, pl.jobs, pl.njobs, pl.job_units, pl.snap, pl.max_jobs, lbits_sub,
        (uint32_t)std::min<uint64_t>(pl.offload_min, 0xFFFFFFFFull));
    CPX_LAUNCH("k_hard");
    note_launch(ctx);
    if (pl.max_jobs) {
        scan_u64(ctx, pl.job_units, pl.max_jobs + 1);
        k_hard_leaves<XT><<<(unsigned)ctx->sm_count * 8, kThreads, 0, ctx->stream>>>(
            pl.jobs, pl.njobs, pl.max_jobs, pl.job_units, pl.snap, lbits_sub, tb.MU, tb.T, pl.hard_ms, pl.acc);
        CPX_LAUNCH("k_hard_leaves");
        note_launch(ctx);
    }
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
