// sieve.cuh -- the segment bitmap of the hard-leaf sieve and the device
// helpers every hard-leaf kernel shares: layout, pre-sieve, cross-off, leaf
// counts, snapshots of leaf sets and the levels a segment sieves.
//
// Bitmap layout: one segment holds 2^lbits odd numbers n = lo + 2i + 1 as a
// bitmap in shared memory with one 8-bit survivor counter per 16-byte chunk
// (128 numbers).  Thread t owns chunks [CPT t, CPT (t+1)); chunk c is stored
// at c ^ ((c >> log2 CPT) & 7) so the owners' 128-bit accesses are free of
// bank conflicts.  Counters are indexed by the unswizzled chunk.  Warp w owns
// the contiguous sub-segment of chunks [32 CPT w, 32 CPT (w+1)).
#pragma once
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
static __device__ __noinline__ uint32_t presieve(uint32_t *bm, uint8_t *cnt8, const uint32_t *__restrict__ P, uint32_t c,
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
static __device__ __noinline__ void snapshot_chunks(uint4 *sb, uint32_t *spre, const uint32_t *bm, const uint8_t *cnt8,
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

// Crossing-off parameters of p for a sub-segment [lo_w, hi_w): r0 = (lo_w + 1)
// mod p and i0 = the bit of the first odd multiple of p (0xFFFFFFFF: none).
__device__ __forceinline__ void cross_params(uint64_t p, uint64_t lo_w, uint64_t hi_w, uint32_t &r0, uint32_t &i0)
{
    const uint64_t r = (lo_w + 1) - cpx_udiv_leaf(lo_w + 1, p) * p;
    r0 = (uint32_t)r;
    uint64_t m = lo_w + 1 + (r ? p - r : 0);
    if ((m & 1) == 0) m += p;
    i0 = (m < hi_w) ? (uint32_t)((m - lo_w - 1) >> 1) : 0xFFFFFFFFu;
}

// Quotients by a warp's sub-segment bounds.  A bound d at or above 2^32 would
// take the 64-bit hardware division; with rd = 1/d (double, once per warp) the
// quotient n/d < 2^32 is the truncated product n * rd, whose relative error
// (three roundings, at most 3 * 2^-53) leaves it within 1 of floor(n/d), fixed
// by the sign and size of the exact remainder n - q d.
struct BoundDiv {
    uint64_t d;
    double rd;
};
__device__ __forceinline__ BoundDiv bound_div(uint64_t d)
{
    BoundDiv b;
    b.d = d;
    b.rd = (d >> 32) ? 1.0 / (double)d : 0.0;
    return b;
}
template <class XT> __device__ __forceinline__ XT div_bound(XT n, const BoundDiv &b)
{
    if (!(b.d >> 32) || ((u128)n >> 64)) return cpx_qdiv(n, b.d);
    const uint64_t n64 = (uint64_t)n;
    uint64_t q = __double2ull_rz(__dmul_rn(__ull2double_rn(n64), b.rd));
    const int64_t r = (int64_t)(n64 - q * b.d);
    if (r < 0) q--;
    else if ((uint64_t)r >= b.d) q++;
    return (XT)q;
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
static __device__ __noinline__ void level_params(LvlPar<XT> &o, XT x, uint64_t y, uint64_t p, uint64_t lo_w,
                                                uint64_t hi_w, const BoundDiv &bl, const BoundDiv &bh)
{
    const XT xp = cpx_qdiv(x, p);
    uint64_t mlo = y / p;
    const XT t1 = div_bound(xp, bh);
    if (t1 > (XT)mlo) mlo = (uint64_t)t1;
    uint64_t mhi = y;
    if (lo_w) {
        const XT t2 = div_bound(xp, bl);
        if (t2 < (XT)mhi) mhi = (uint64_t)t2;
    }
    const XT t3 = cpx_qdiv(xp, p * p);  // hard leaves only: m <= x/p^3
    if (t3 < (XT)mhi) mhi = (uint64_t)t3;
    if (mhi < mlo) mhi = mlo;
    o.p = (uint32_t)p;
    o.xp = xp;
    o.mlo = (uint32_t)mlo;
    o.mhi = (uint32_t)mhi;
    cross_params(p, lo_w, hi_w, o.r0, o.i0);
}

// Crosses p off one warp's sub-segment of Lw bits (chunks [base_ch, base_ch +
// 32 CPT) of the segment); the lane owns chunks [c0, c0 + CPT), cw0 = c0 -
// base_ch.  Keeps the chunk counters current; returns the bits the lane cleared.
// kOwnWords: primes below 128 update each multiple's word and counter without
// a branch (measured on a B200: 4% faster for the lone-query sieve of pi(1e20)
// with 128 threads, 1% slower for the batch-shared sieve, which keeps the
// branch).
template <bool kOwnWords = false>
__device__ __forceinline__ uint32_t cross_off(uint32_t *bm, uint8_t *cnt8, uint32_t p, uint32_t r0, uint32_t i0,
                                              uint32_t c0, uint32_t cw0, uint32_t CPT, int s, uint32_t base_ch,
                                              uint32_t lane, uint32_t Lw)
{
    uint32_t cleared = 0;
    if (p < 32) {
        // each lane masks its own words: several multiples per word
        const uint32_t Mp = every_pth_bit(p);
        const uint32_t stp = 64u % p;
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
    } else if (p < 128 && kOwnWords) {
        // at most one multiple per word: each lane jumps from multiple to
        // multiple inside its own chunks (its words and counters only, so
        // without a branch).  The lane's chunks c share c >> s = c0 >> s, so
        // their swizzle is one XOR of bits 2..4 of the word index.
        if (i0 != 0xFFFFFFFFu) {
            const uint32_t b0 = cw0 * 128, b1 = b0 + CPT * 128;  // the lane's bits of the sub-segment
            uint32_t i = i0;
            if (b0 > i0) {
                // k = ceil(n / p), n = b0 - i0 < 2^21: trunc(n / p) from the
                // approximate reciprocal is within 1 of floor(n / p), so k lies in
                // [t - 1, t + 2]; step up from t - 1 while k p < n
                const int32_t n = (int32_t)(b0 - i0), pi = (int32_t)p;
                int32_t k = (int32_t)__float2uint_rz((float)n * cpx_rcp_approx(p)) - 1;
                k += k * pi < n;
                k += k * pi < n;
                k += k * pi < n;
                i = i0 + (uint32_t)k * p;
            }
            const uint32_t kx = s ? (((c0 >> s) & 7u) << 2) : 0u;
            uint32_t *bmw = bm + (base_ch << 2);
            uint8_t *cw8 = cnt8 + base_ch;
            for (; i < b1; i += p) {
                const uint32_t w = i >> 5;
                uint32_t *pw = bmw + (w ^ kx);
                const uint32_t old = *pw, hit = old & (1u << (i & 31));
                *pw = old ^ hit;
                const uint32_t h = hit ? 1u : 0u;
                cw8[w >> 2] = (uint8_t)(cw8[w >> 2] - h);
                cleared += h;
            }
        }
    } else if (p < 128) {
        // at most one multiple per word: each lane jumps from multiple to
        // multiple inside its own chunks (its counters only)
        if (i0 != 0xFFFFFFFFu) {
            const uint32_t b0 = cw0 * 128, b1 = b0 + CPT * 128;  // the lane's bits of the sub-segment
            uint32_t i = i0;
            if (b0 > i0) i = i0 + ((b0 - i0 + p - 1) / p) * p;
            for (; i < b1; i += p) {
                const uint32_t w = i >> 5, bit = 1u << (i & 31);
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
    } else if (i0 != 0xFFFFFFFFu) {
        // p >= 128: the lanes of one step clear bits p apart, so they touch
        // distinct words and distinct chunk counters (plain read-modify-write).
        // Bit indices stay in 32 bits while i0 + 32 p does (Lw <= 2^20).
        auto clear = [&](uint32_t i) {
            const uint32_t w = i >> 5, bit = 1u << (i & 31);
            const uint32_t ch = base_ch + (w >> 2);
            uint32_t *pw = bm + ((swz(ch, s) << 2) | (w & 3));
            const uint32_t old = *pw;
            if (old & bit) {
                *pw = old & ~bit;
                cleared++;
                cnt8[ch] = (uint8_t)(cnt8[ch] - 1);
            }
        };
        if (p < (1u << 26)) {
            for (uint32_t i = i0 + lane * p; i < Lw; i += 32u * p) clear(i);
        } else {
            for (uint64_t i = (uint64_t)i0 + (uint64_t)lane * p; i < Lw; i += 32ull * p) clear((uint32_t)i);
        }
    }
    return cleared;
}

// A leaf quotient x/(p m) = xp / m of a leaf in a sub-segment that ends at
// or below 2^41 (q41, so the quotient is below 2^41): cpx_quot40 when xp <
// 2^53 (xpd = xp as a double, exact), else cpx_qdiv.
template <class XT> __device__ __forceinline__ uint64_t leaf_quot(XT xp, double xpd, uint64_t m, bool q41)
{
    if (q41 && ((u128)xp >> 53) == 0) return cpx_quot40((uint64_t)xp, xpd, (uint32_t)m);
    return (uint64_t)cpx_qdiv(xp, m);
}

// Survivors among bits 0..jb of one 16-byte bitmap chunk, without a branch.
__device__ __forceinline__ uint32_t chunk_survivors(uint4 v4, uint32_t jb)
{
    const uint32_t wi = (jb >> 5) & 3, msk = (2u << (jb & 31)) - 1u;
    const uint32_t m0 = wi > 0 ? ~0u : msk;
    const uint32_t m1 = wi > 1 ? ~0u : (wi == 1 ? msk : 0u);
    const uint32_t m2 = wi > 2 ? ~0u : (wi == 2 ? msk : 0u);
    const uint32_t m3 = wi == 3 ? msk : 0u;
    return __popc(v4.x & m0) + __popc(v4.y & m1) + __popc(v4.z & m2) + __popc(v4.w & m3);
}

// Survivors of a warp's sub-segment [lo_w, lo_w + 2 Lw) with n <= uu, uu in
// [lo_w, hi_w), from the lane prefixes wl[] of the sub-segment, the chunk
// counters and the chunk's popcounts.
__device__ __forceinline__ uint32_t sub_survivors(uint64_t uu, uint64_t lo_w, const uint32_t *wl, const uint8_t *cnt8,
                                                  const uint32_t *bm, uint32_t CPT, int s, uint32_t warp)
{
    // bits [0, kk) of the sub-segment; uu - lo_w < 2^21, so its low 32 bits suffice
    const uint32_t kk = ((uint32_t)uu - (uint32_t)lo_w + 1u) >> 1;
    if (!kk) return 0u;
    const uint32_t jb = kk - 1, w = jb >> 5;
    const uint32_t chs = w >> 2, ow = chs >> s;  // chunk in the sub-segment, owning lane
    const uint32_t ch = chs + CPT * 32 * warp;   // chunk in the segment
    const uint32_t n = chs - ow * CPT;           // the owner's counters before the chunk
    uint32_t cv = wl[ow];
    if (CPT >= 4) {
        // the owner's counters as CPT/4 aligned words (CPT is a power of two);
        // a trip count uniform over the warp, the counters before the chunk
        // selected by a byte mask
        const uint32_t *cw = reinterpret_cast<const uint32_t *>(cnt8 + ch - n);
        for (uint32_t i = 0; i < (CPT >> 2); i++) {
            const int r = (int)n - 4 * (int)i;
            const uint32_t sel = r >= 4 ? 0x01010101u : (r <= 0 ? 0u : (0x01010101u & ((1u << (8 * r)) - 1u)));
            cv = __dp4a(cw[i], sel, cv);
        }
    } else {
        for (uint32_t i = 0; i < n; i++) cv += cnt8[ch - n + i];
    }
    return cv + chunk_survivors(reinterpret_cast<const uint4 *>(bm)[swz(ch, s)], jb);
}

// Survivor prefixes of one lane's chunks [c0, c0 + CPT): pre16[c0 + j] = the
// counters of chunks c0 .. c0 + j - 1 (below 2^16: CPT 128 <= 2^15 bits);
// returns the lane's total.  Built once a level that has leaves in the warp's
// sub-segment, so that a leaf count reads one prefix instead of summing the
// owner's counters.  CPT a multiple of 8: each counter word gives its four
// running sums by byte-masked dp4a.
__device__ __forceinline__ uint32_t chunk_prefixes(const uint8_t *cnt8, uint16_t *pre16, uint32_t c0, uint32_t CPT)
{
    uint32_t run = 0;
    if ((CPT & 7) == 0) {
        const uint32_t *cw = reinterpret_cast<const uint32_t *>(cnt8 + c0);
        uint4 *pw = reinterpret_cast<uint4 *>(pre16 + c0);
        for (uint32_t i = 0; i < (CPT >> 3); i++) {
            const uint32_t a = cw[2 * i], b = cw[2 * i + 1];
            uint4 o;
            o.x = run | (__dp4a(a, 0x00000001u, run) << 16);
            o.y = __dp4a(a, 0x00000101u, run) | (__dp4a(a, 0x00010101u, run) << 16);
            run = __dp4a(a, 0x01010101u, run);
            o.z = run | (__dp4a(b, 0x00000001u, run) << 16);
            o.w = __dp4a(b, 0x00000101u, run) | (__dp4a(b, 0x00010101u, run) << 16);
            run = __dp4a(b, 0x01010101u, run);
            pw[i] = o;
        }
    } else {
        for (uint32_t j = 0; j < CPT; j++) {
            pre16[c0 + j] = (uint16_t)run;
            run += cnt8[c0 + j];
        }
    }
    return run;
}

// sub_survivors from the chunk prefixes of chunk_prefixes: the owner lane's
// prefix, the chunk's prefix within the owner and the chunk's popcounts.
__device__ __forceinline__ uint32_t sub_survivors_pre(uint64_t uu, uint64_t lo_w, const uint32_t *wl,
                                                      const uint16_t *pre16, const uint32_t *bm, uint32_t CPT, int s,
                                                      uint32_t warp)
{
    // bits [0, kk) of the sub-segment; uu - lo_w < 2^21, so its low 32 bits suffice
    const uint32_t kk = ((uint32_t)uu - (uint32_t)lo_w + 1u) >> 1;
    if (!kk) return 0u;
    const uint32_t jb = kk - 1;
    const uint32_t chs = jb >> 7;               // chunk in the sub-segment
    const uint32_t ch = chs + CPT * 32 * warp;  // chunk in the segment
    return wl[chs >> s] + pre16[ch] + chunk_survivors(reinterpret_cast<const uint4 *>(bm)[swz(ch, s)], jb);
}

// B(seg) = pi(min(r4, isqrt((x - 1) / lo), isqrt(hi - 1))): the levels b a
// segment [lo, hi) sieves for an x with iroot4(x) = r4.  p_b^2 lo < x bounds
// the levels whose leaves can reach the segment or a later one; p_b^2 < hi
// skips the levels whose leaves all lie above the segment (below p_b^2 the
// carry phi(v, b - 1) is 1 + pi(v) - (b - 1), read from the pi table).
template <class XT>
__device__ __forceinline__ uint32_t seg_levels(XT x, uint64_t r4, uint64_t lo, uint64_t hi,
                                               const uint32_t *__restrict__ P, uint32_t np)
{
    uint64_t v = r4;
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
    return a;
}

// inclusive warp scan of n; returns the warp total, *off = exclusive offset
__device__ __forceinline__ uint32_t warp_place(uint32_t n, uint32_t lane, uint32_t &off)
{
    uint32_t inc = n;
#pragma unroll
    for (int oo = 1; oo < 32; oo <<= 1) {
        const uint32_t t = __shfl_up_sync(FULL, inc, oo);
        if (lane >= (uint32_t)oo) inc += t;
    }
    off = inc - n;
    return __shfl_sync(FULL, inc, 31);
}

}  // namespace cpx
