// gourdon.cu -- pi(x) through Gourdon's decomposition on the GPU, the term
// split of the reference's GourdonVariant64 (include/Gourdon/gourdonvariant.hpp:7-56):
//
//   pi(x) = A - B + C + D + Phi0 + Sigma0 + ... + Sigma6
//
// with a = pi(y), b3 = pi(cbrt x), bs = pi(sqrt x), z = x/y, x* = min(max(
// iroot4(x), x/y^2), cbrt x), d = pi(x*) and cz = pi(sqrt z) held within [d, b3]:
//   A      = sum_{x* < p <= cbrt x} sum_{p < q <= sqrt(x/p)} chi(x/pq) pi(x/pq),
//            chi(n) = 2 if n < y else 1                (src/Gourdon/A2.cu:168-283)
//   B      = sum_{y < p <= sqrt x} pi(x/p)             (src/Gourdon/B.cu:16-71)
//   C      = the easy and trivial special leaves of the p_b <= x*, b > c
//                                                      (src/Gourdon/C.cu:67)
//   D      = the hard special leaves                   (src/Gourdon/gourdonvariant.cpp:61)
//   Phi0   = the ordinary leaves                       (src/Gourdon/phi_0.cpp:5-8)
//   Sigma0..6: closed forms in a, b3, bs, d, cz and three sums over the p of
//            (x*, cbrt x]                              (src/Gourdon/sigma_cpu.cpp:36-146)
// The reference fixes x* = iroot4(x), which makes the identity hold only for
// y >= ~x^(3/8); with x* = max(iroot4(x), x/y^2) every y of the
// Deleglise-Rivat domain works (for iroot4(x) < p <= x/y^2 no leaf is hard,
// so those p join C).  The reference's piGourdon returns 0 with its term
// calls commented out (src/Gourdon/gourdonvariant.cpp:37-75); this path
// computes every term.
//
// B, C, D and Phi0 come from the Deleglise-Rivat kernels (k_p2 plus a closed
// form, k_easy limited to p <= x* with k_easy_comp, the hard-leaf sieve,
// k_ordinary).  A is k_gourdon_A: warps take the p of (x*, cbrt x] one at a
// time from a device counter (largest q range first), gather the primes q of
// a run of pi-table entries into shared memory and answer them 32 at a time,
// one quotient and one table lookup per pair.  The Sigma sums and the trivial
// leaves of C are k_gourdon_sums, one thread per p.  x < 2^64, as the
// reference's GourdonVariant64.
#include "driver.h"
#include "sieve.cuh"

namespace cpx {

namespace {

enum { G_A = 0, G_S4, G_S5, G_S6, G_CT, G_N };  // 128-bit device sums
constexpr uint32_t kGABuf = 256;                // gathered q per warp

// A over the primes p = P[i], i in [i0, i1): per p the q in (p, sqrt(x/p)]
__global__ void __launch_bounds__(256) k_gourdon_A(uint64_t x, uint64_t y, const uint32_t *__restrict__ P,
                                                   uint32_t i0, uint32_t i1, const cpx_pient *__restrict__ T,
                                                   unsigned int *__restrict__ next, unsigned long long *__restrict__ acc)
{
    const uint32_t lane = threadIdx.x & 31;
    __shared__ uint32_t s_q[256 / 32][kGABuf];
    uint32_t *qbuf = s_q[threadIdx.x >> 5];
    u128 sum = 0;
    for (;;) {
        uint32_t k = 0;
        if (lane == 0) k = atomicAdd(next, 1u);
        k = __shfl_sync(FULL, k, 0);
        if (k >= i1 - i0) break;
        const uint64_t p = __ldg(P + i0 + k);
        const uint64_t xp = cpx_udiv_leaf(x, p);
        const uint64_t qhi = cpx_isqrt((u128)xp);
        if (qhi <= p) continue;  // uniform over the warp
        const uint64_t w_beg = p >> 7, w_end = ((qhi - 1) >> 7) + 1;
        uint64_t ps = 0;
        uint32_t nbuf = 0;
        auto answer = [&](uint64_t q) {
            const uint64_t u = cpx_udiv_leaf(xp, q);
            const uint64_t pu = cpx_pi_dev(T, u);
            ps += u < y ? 2 * pu : pu;
        };
        auto flush = [&] {
            __syncwarp();
            for (uint32_t j = lane; j < nbuf; j += 32) answer(qbuf[j]);
            __syncwarp();
            nbuf = 0;
        };
        for (uint64_t wb = w_beg; wb < w_end; wb += 32) {  // uniform over the warp
            const uint64_t wq = wb + lane;
            uint64_t qb = 0;
            if (wq < w_end) qb = __ldg(reinterpret_cast<const ulonglong2 *>(T) + wq).x & range_mask(wq, p, qhi);
            const uint32_t nq = (uint32_t)__popcll(qb);
            uint32_t off;
            const uint32_t tot = warp_place(nq, lane, off);
            if (tot > kGABuf) {  // dense: each lane answers its own entry
                while (qb) {
                    const int j = __ffsll((long long)qb) - 1;
                    qb &= qb - 1;
                    answer(128 * wq + 2 * j + 1);
                }
                continue;
            }
            if (nbuf + tot > kGABuf) flush();
            uint32_t kk = nbuf + off;
            while (qb) {
                const int j = __ffsll((long long)qb) - 1;
                qb &= qb - 1;
                qbuf[kk++] = (uint32_t)(128 * wq + 2 * j + 1);
            }
            nbuf += tot;
        }
        flush();
        sum += ps;
    }
    // warp total into the device sum
    const i128 t = cpx_warp_sum_i128((i128)sum);
    if (lane == 0 && t) cpx_atomic_add_i128(acc + 2 * G_A, t);
}

// One thread per p = P[i], i in [ir4, b3): for i < d the trivial leaves of C
// (x/p^2 < y: a - pi(x/p^2)); for i >= d Sigma4 (i < cz: pi(x/(p y))),
// Sigma5 (i >= cz: pi(x/p^2)) and Sigma6 (pi(isqrt(x/p))^2).
__global__ void __launch_bounds__(256) k_gourdon_sums(uint64_t x, uint64_t y, uint64_t a, const uint32_t *__restrict__ P,
                                                      uint32_t ir4, uint32_t d, uint32_t cz, uint32_t b3,
                                                      const cpx_pient *__restrict__ T,
                                                      unsigned long long *__restrict__ acc)
{
    const uint64_t i = (uint64_t)ir4 + (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    u128 s4 = 0, s5 = 0, s6 = 0, ct = 0;
    if (i < b3) {
        const uint64_t p = __ldg(P + i);
        const uint64_t xp = cpx_udiv_leaf(x, p);
        const uint64_t v2 = cpx_udiv_leaf(xp, p);  // x / p^2
        if (i < d) {
            if (v2 < y) ct = a - cpx_pi_dev(T, v2);
        } else {
            if (i < cz) s4 = cpx_pi_dev(T, xp / y);
            else s5 = cpx_pi_dev(T, v2);
            const uint64_t r = cpx_pi_dev(T, cpx_isqrt((u128)xp));
            s6 = (u128)r * r;
        }
    }
    const u128 v[4] = {s4, s5, s6, ct};
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const i128 t = cpx_warp_sum_i128((i128)v[k]);
        if ((threadIdx.x & 31) == 0 && t) cpx_atomic_add_i128(acc + 2 * (G_S4 + k), t);
    }
}

__global__ void k_gourdon_pi(const cpx_pient *__restrict__ T, uint64_t y, uint64_t sx, uint64_t *out)
{
    out[0] = cpx_pi_dev(T, y);
    out[1] = cpx_pi_dev(T, sx);
}

}  // namespace

// A, B, C, D, Phi0, Sigma, pi(x) of one x < 2^64 with y in the
// Deleglise-Rivat domain (icbrt(x) <= y < isqrt(x)).
void gourdon_terms(cpx_ctx *ctx, uint64_t x, uint64_t y, uint32_t c, i128 out[7])
{
    if (!y) y = default_y(x, 0, 0);
    if (!dr_domain_ok(x, y, c)) fail(CPX_EINVAL, "y outside the Deleglise-Rivat domain for this x");
    const uint64_t sx = cpx_isqrt(x), cx = cpx_icbrt(x), r4 = cpx_iroot4(x);
    const uint64_t z = x / y, sz = cpx_isqrt(z);
    const u128 yy = (u128)y * y;
    uint64_t xs = std::max<uint64_t>(r4, (uint64_t)((u128)x / yy));
    if (xs > cx) xs = cx;

    // B (from P2), C's easy leaves (p <= x*), D and Phi0: the Deleglise-Rivat kernels
    BatchReq rq;
    const u128 xx = x;
    rq.xs = &xx;
    rq.ys = &y;
    rq.n = 1;
    rq.c = c;
    rq.terms = TERM_P2 | TERM_ORD | TERM_EASY | TERM_HARD;
    rq.easy_pmax = xs;
    i128 t7[7];
    rq.out_terms = t7;
    run_batch(ctx, rq);

    // A and the Sigma sums read pi(v) for v <= sqrt x and the primes to cbrt x
    TableNeed need;
    need.N = sx + 2;
    need.P = cx + 1;
    grow_tables(ctx, need);
    const std::vector<uint32_t> &hP = host_primes(ctx);
    const uint32_t ir4 = (uint32_t)host_pi(hP, r4), d = (uint32_t)host_pi(hP, xs), b3 = (uint32_t)host_pi(hP, cx);
    const uint32_t cz = (uint32_t)std::min<uint64_t>(std::max<uint64_t>(host_pi(hP, sz), d), b3);

    unsigned long long *acc = ctx->b_small.as<unsigned long long>(2 * G_N + 8);
    uint64_t *d_pi = reinterpret_cast<uint64_t *>(acc + 2 * G_N);
    unsigned int *next = reinterpret_cast<unsigned int *>(acc + 2 * G_N + 4);
    CPX_CUDA(cudaMemsetAsync(acc, 0, (2 * G_N + 8) * sizeof(unsigned long long), ctx->stream));
    k_gourdon_pi<<<1, 1, 0, ctx->stream>>>(ctx->tab.T, y, sx, d_pi);
    CPX_LAUNCH("k_gourdon_pi");
    uint64_t hpi[2];
    CPX_CUDA(cudaMemcpyAsync(hpi, d_pi, sizeof(hpi), cudaMemcpyDeviceToHost, ctx->stream));
    CPX_CUDA(cudaStreamSynchronize(ctx->stream));
    const uint64_t a = hpi[0], bs = hpi[1];
    note_launch(ctx);
    if (b3 > d) {
        KSpan ks(ctx, "k_gourdon_A");
        k_gourdon_A<<<(unsigned)ctx->sm_count * 8, 256, 0, ctx->stream>>>(x, y, ctx->tab.P, d, b3, ctx->tab.T, next,
                                                                        acc);
        CPX_LAUNCH("k_gourdon_A");
        note_launch(ctx);
    }
    if (b3 > ir4) {
        k_gourdon_sums<<<(unsigned)((b3 - ir4 + 255) / 256), 256, 0, ctx->stream>>>(x, y, a, ctx->tab.P, ir4, d, cz, b3,
                                                                                    ctx->tab.T, acc);
        CPX_LAUNCH("k_gourdon_sums");
        note_launch(ctx);
    }
    unsigned long long h[2 * G_N];
    CPX_CUDA(cudaMemcpyAsync(h, acc, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
    CPX_CUDA(cudaStreamSynchronize(ctx->stream));
    auto rd = [&](int k) { return (i128)(((u128)h[2 * k + 1] << 64) | h[2 * k]); };

    const i128 A = rd(G_A);
    const i128 ia = (i128)a, ib3 = b3, ibs = (i128)bs, id = d, icz = cz;
    const i128 B = t7[0] + ibs * (ibs - 1) / 2 - ia * (ia - 1) / 2;  // P2 = B - sum_{y<p<=sqrt x} (pi(p) - 1)
    const i128 C = t7[3] + rd(G_CT);
    i128 sg = ia - 1 + ibs * (ibs - 1) / 2 - ia * (ia - 1) / 2;                              // Sigma0
    sg += (ia - ib3) * (ia - ib3 - 1) / 2;                                                    // Sigma1
    sg += ia * (ib3 - icz - icz * (icz - 3) / 2 + id * (id - 3) / 2);                          // Sigma2
    sg += ib3 * (ib3 - 1) * (2 * ib3 - 1) / 6 - ib3 - id * (id - 1) * (2 * id - 1) / 6 + id;  // Sigma3
    sg += ia * rd(G_S4) + rd(G_S5) - rd(G_S6);                                                // Sigma4..6
    out[0] = A;
    out[1] = B;
    out[2] = C;
    out[3] = t7[4];  // D
    out[4] = t7[1];  // Phi0
    out[5] = sg;
    out[6] = A - B + C + t7[4] + t7[1] + sg;
}

}  // namespace cpx
