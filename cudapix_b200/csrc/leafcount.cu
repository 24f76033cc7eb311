// leafcount.cu -- exact special-leaf counts per class for one query.
//
// The reference's leaf-count analysis (src/leafcount.cpp:12-202) estimates how
// many leaves each class holds, to weigh the work.  Here the counts are exact,
// in this library's split of the special leaves (b, m), u = x/(p_b m):
// trivial u < p_b, easy p_b <= u < p_b^2 (m prime or composite), hard
// u >= p_b^2.
//   p_b <= iroot4(x): m in (y/p, y], squarefree with lpf(m) > p; hard when
//     m <= x/p^3, else easy (none is trivial: x/p^2 >= sqrt x > y >= m).
//   iroot4(x) < p_b <= y: m = q prime in (max(p, y/p), y]; trivial when
//     q > x/p^2, else easy.
// The hard count divides the hard-leaf time into leaves per second.
#include "driver.h"
#include "kern_common.cuh"

namespace cpx {

enum { LC_HARD = 0, LC_EASY_COMP, LC_EASY_PRIME, LC_TRIVIAL, LC_N };
constexpr uint32_t kLeafChunk = 4096;  // odd m per block of k_leaf_small (16 per thread)

// Levels b = c+1 .. nb (p_b <= iroot4(x)); blockIdx.y = b - c - 1, blockIdx.x = chunk of odd m.
template <class XT>
__global__ void __launch_bounds__(256) k_leaf_small(XT x, uint64_t y, uint32_t c, const uint32_t *__restrict__ P,
                                                    const int32_t *__restrict__ MU,
                                                    unsigned long long *__restrict__ out)
{
    const uint32_t b = c + 1 + blockIdx.y;
    const uint64_t p = P[b - 1];
    const uint64_t i_lo = (y / p + 1) >> 1, i_hi = (y - 1) >> 1;  // odd m = 2i + 1 in (y/p, y]
    const uint64_t base = (i_lo & ~uint64_t(3)) + (uint64_t)blockIdx.x * kLeafChunk;
    __shared__ unsigned long long red[3][8];
    unsigned long long n_hard = 0, n_comp = 0, n_prime = 0;
    if (base <= i_hi) {
        const XT x3 = x / (XT)p / (XT)p / (XT)p;
        const uint64_t mh = x3 < (XT)y ? (uint64_t)x3 : y;  // hard: m <= x/p^3
        for (uint32_t k = 0; k < kLeafChunk / 4 / 256; k++) {
            const uint64_t g = (base >> 2) + k * 256 + threadIdx.x;
            if (4 * g > i_hi) break;
            const int4 v4 = __ldg(reinterpret_cast<const int4 *>(MU) + g);
            const int32_t vals[4] = {v4.x, v4.y, v4.z, v4.w};
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const uint64_t i = 4 * g + j;
                const int32_t v = vals[j];
                const uint32_t av = (uint32_t)(v > 0 ? v : -v);
                if (i < i_lo || i > i_hi || v == 0 || av <= p) continue;
                const uint64_t m = 2 * i + 1;
                if (m <= mh) n_hard++;
                else if ((uint64_t)av < m) n_comp++;
                else n_prime++;  // lpf(m) = m (m = 1 never lies in (y/p, y])
            }
        }
    }
    // block sums
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        n_hard += __shfl_down_sync(FULL, n_hard, o);
        n_comp += __shfl_down_sync(FULL, n_comp, o);
        n_prime += __shfl_down_sync(FULL, n_prime, o);
    }
    const uint32_t lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) {
        red[0][w] = n_hard;
        red[1][w] = n_comp;
        red[2][w] = n_prime;
    }
    __syncthreads();
    if (threadIdx.x < 3) {
        unsigned long long s = 0;
        for (int k = 0; k < 8; k++) s += red[threadIdx.x][k];
        if (s) atomicAdd(out + (threadIdx.x == 0 ? LC_HARD : threadIdx.x == 1 ? LC_EASY_COMP : LC_EASY_PRIME), s);
    }
}

// Primes p_b in (iroot4(x), y] (P indices k0 .. k1 - 1): prime q in (max(p, y/p), y],
// trivial above x/p^2, easy below; counted with the pi table.
template <class XT>
__global__ void k_leaf_large(XT x, uint64_t y, uint64_t k0, uint64_t k1, const uint32_t *__restrict__ P,
                             const cpx_pient *__restrict__ T, unsigned long long *__restrict__ out)
{
    const uint64_t k = k0 + (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    unsigned long long n_triv = 0, n_easy = 0;
    if (k < k1) {
        const uint64_t p = P[k];
        uint64_t qlo = y / p;
        if (qlo < p) qlo = p;
        const XT x2 = x / (XT)p / (XT)p;
        const uint64_t qe = x2 < (XT)y ? (uint64_t)x2 : y;  // easy: q <= x/p^2
        const uint64_t piy = cpx_pi_dev(T, y);
        if (qe > qlo) n_easy = cpx_pi_dev(T, qe) - cpx_pi_dev(T, qlo);
        const uint64_t tlo = qe > qlo ? qe : qlo;
        if (y > tlo) n_triv = piy - cpx_pi_dev(T, tlo);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        n_triv += __shfl_down_sync(FULL, n_triv, o);
        n_easy += __shfl_down_sync(FULL, n_easy, o);
    }
    if ((threadIdx.x & 31) == 0) {
        if (n_triv) atomicAdd(out + LC_TRIVIAL, n_triv);
        if (n_easy) atomicAdd(out + LC_EASY_PRIME, n_easy);
    }
}

template <class XT> static void leaf_go(cpx_ctx *ctx, const QD &d, unsigned long long *dout)
{
    const Tables &tb = ctx->tab;
    const XT x = (XT)d.x;
    const uint64_t y = d.y;
    const uint32_t nb = d.nb;  // pi(iroot4(x))
    if (nb > d.c) {
        // the largest level has the longest m range (y/p, y]
        const uint64_t p = host_primes(ctx)[nb - 1];
        const uint64_t i_lo = (y / p + 1) >> 1, i_hi = (y - 1) >> 1;
        const uint64_t nchunks = i_hi >= (i_lo & ~uint64_t(3)) ? ((i_hi - (i_lo & ~uint64_t(3))) / kLeafChunk + 1) : 0;
        if (nchunks) {
            const dim3 grid((unsigned)nchunks, nb - d.c);
            k_leaf_small<XT><<<grid, 256, 0, ctx->stream>>>(x, y, d.c, tb.P, tb.MU, dout);
            CPX_LAUNCH("k_leaf_small");
            note_launch(ctx);
        }
    }
    const uint64_t k0 = nb > d.c ? nb : d.c, k1 = host_pi(host_primes(ctx), y);
    if (k1 > k0) {
        k_leaf_large<XT><<<(unsigned)((k1 - k0 + 255) / 256), 256, 0, ctx->stream>>>(x, y, k0, k1, tb.P, tb.T, dout);
        CPX_LAUNCH("k_leaf_large");
        note_launch(ctx);
    }
}

void leaf_counts(cpx_ctx *ctx, u128 x, uint64_t y, uint32_t c, uint64_t out[4])
{
    BatchReq rq;
    rq.xs = &x;
    rq.ys = &y;
    rq.n = 1;
    rq.c = c;
    rq.terms = TERM_PI;
    std::vector<QD> qd;
    TableNeed need;
    bool wide = false;
    compute_needs(rq, qd, need, wide);
    QD &d = qd[0];
    if (d.direct) fail(CPX_EINVAL, "x is below the Deleglise-Rivat domain (no special leaves are split)");
    // the pi table to y and sqrt(x), mu/lpf to y, every prime up to y
    need.N = std::max<uint64_t>(need.N, std::max<uint64_t>(d.sx, d.y) + 2);
    need.P = std::max<uint64_t>(need.P, d.y + 1);
    need.Y = std::max<uint64_t>(need.Y, d.y + 8);
    grow_tables(ctx, need);
    d.nb = (uint32_t)host_pi(host_primes(ctx), d.r4);
    unsigned long long *dout = ctx->b_small.as<unsigned long long>(8);
    CPX_CUDA(cudaMemsetAsync(dout, 0, 8 * sizeof(unsigned long long), ctx->stream));
    if (wide) leaf_go<u128>(ctx, d, dout);
    else leaf_go<uint64_t>(ctx, d, dout);
    unsigned long long h[LC_N];
    CPX_CUDA(cudaMemcpyAsync(h, dout, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
    CPX_CUDA(cudaStreamSynchronize(ctx->stream));
    for (int k = 0; k < LC_N; k++) out[k] = h[k];
}

}  // namespace cpx
