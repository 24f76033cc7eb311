// kern_common.cuh -- device helpers shared by the term kernels: query lookup
// over unit prefix arrays, per-query 128-bit accumulation, table-entry masks.
#pragma once
#include "terms.cuh"

namespace cpx {

constexpr unsigned FULL = 0xffffffffu;
static __constant__ uint32_t c_pc[9] = {1, 2, 3, 5, 7, 11, 13, 17, 19};  // p_c for c = 0..8

__device__ __forceinline__ uint32_t find_q(const uint64_t *__restrict__ pre, uint32_t Q, uint64_t u)
{
    uint32_t lo = 0, hi = Q;  // pre[lo] <= u < pre[hi]
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (__ldg(pre + mid) <= u) lo = mid;
        else hi = mid;
    }
    return lo;
}

// bits j of table entry w with a < 128w + 2j + 1 <= b
__device__ __forceinline__ uint64_t range_mask(uint64_t w, uint64_t a, uint64_t b)
{
    const uint64_t base = 128 * w;
    if (b < base + 1) return 0;
    uint64_t hiJ = (b - base - 1) >> 1;
    if (hiJ > 63) hiJ = 63;
    const uint64_t loJ = (a >= base) ? ((a - base + 1) >> 1) : 0;
    if (loJ > hiJ) return 0;
    const uint64_t upto = (hiJ == 63) ? ~0ull : ((2ull << hiJ) - 1);
    return upto & ~((1ull << loJ) - 1);
}

struct LaneAcc {
    uint32_t q = 0xFFFFFFFFu;
    i128 v = 0;
};

__device__ __forceinline__ void acc_add(unsigned long long *acc, uint32_t q, int term, i128 v)
{
    if (q != 0xFFFFFFFFu && v != 0) cpx_atomic_add_i128(acc + (uint64_t)q * kAccStride + 2 * term, v);
}

__device__ __forceinline__ void lane_switch(LaneAcc &a, uint32_t q, unsigned long long *acc, int term)
{
    if (q != a.q) {
        acc_add(acc, a.q, term, a.v);
        a.q = q;
        a.v = 0;
    }
}

// all 32 lanes must call
__device__ __forceinline__ void warp_flush(LaneAcc &a, unsigned long long *acc, int term)
{
    const uint32_t q0 = __shfl_sync(FULL, a.q, 0);
    if (__all_sync(FULL, a.q == q0)) {
        const i128 s = cpx_warp_sum_i128(a.v);
        if ((threadIdx.x & 31) == 0) acc_add(acc, q0, term, s);
    } else {
        acc_add(acc, a.q, term, a.v);
    }
    a.v = 0;
}

// Warp-contiguous partition of [0, total): each warp owns a slice and walks it
// 32 units at a time (coalesced, and queries change rarely inside a slice).
struct WarpSlice {
    uint64_t u0, u1;
};
__device__ __forceinline__ WarpSlice warp_slice(uint64_t total)
{
    const uint64_t gw = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    const uint64_t per = (total + nw - 1) / nw;
    uint64_t u0 = gw * per, u1 = u0 + per;
    if (u0 > total) u0 = total;
    if (u1 > total) u1 = total;
    return {u0, u1};
}

// cached query lookup per lane
struct QCache {
    uint32_t q = 0xFFFFFFFFu;
    uint64_t lo = 1, hi = 0;  // [lo, hi) unit range of q
};
__device__ __forceinline__ uint32_t qlookup(QCache &c, const uint64_t *pre, uint32_t Q, uint64_t u)
{
    if (u >= c.lo && u < c.hi) return c.q;
    c.q = find_q(pre, Q, u);
    c.lo = __ldg(pre + c.q);
    c.hi = __ldg(pre + c.q + 1);
    return c.q;
}

template <class XT> __device__ __forceinline__ XT xload(const QD &d) { return (XT)d.x; }

}  // namespace cpx
