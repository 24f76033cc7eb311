// misc.cu -- the smaller drop-in entry points: Mertens self-test, dense and
// windowed pi tables, prime lists and counts, phi(x, a), Phi::generateRange
// and the Phisieve object.
//
//   mutest                 src/mutest.cu:6-19
//   get_d_piTable/PiTable  src/pitable.cu:10-218
//   Phi                    src/phi.cu:14-109
//   Phisieve               src/sieve/phisieve_host.cu:12-89, phisieve_device.cu:9-78
//   CudaSieve getDevicePrimes / countPrimes (external)
#include <algorithm>

#include "misc.h"

namespace cpx {

// ------------------------------------------------------------------ mutest
// M(top - 1) = S(top - 1) - S((top - 1) / 2), S(v) = sum of mu(n) over odd n <= v
// (mu(2k) = -mu(k) for odd k, 0 for 4 | n).
__global__ void k_mu_sums(const int8_t *__restrict__ mu, uint64_t n_odd, uint64_t v1, uint64_t v2,
                          unsigned long long *out)
{
    int64_t s1 = 0, s2 = 0;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n_odd; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t n = 2 * i + 1;
        const int m = mu[i];
        if (n <= v1) s1 += m;
        if (n <= v2) s2 += m;
    }
    int64_t s = s1 - s2;
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) s += __shfl_down_sync(0xffffffffu, s, d);
    if ((threadIdx.x & 31) == 0 && s) atomicAdd(out, (unsigned long long)s);
}

// Mertens reduction of a caller mu array into a caller accumulator, on a
// caller stream; launches only, allocates nothing.
cudaError_t launch_mu_sums(cudaStream_t st, const int8_t *mu, uint64_t n_odd, uint64_t v1, uint64_t v2,
                           unsigned long long *acc, unsigned grid)
{
    k_mu_sums<<<grid, 256, 0, st>>>(mu, n_odd, v1, v2, acc);
    return cudaGetLastError();
}

int64_t mutest(cpx_ctx *ctx, uint64_t top)
{
    if (top <= 1) return 0;
    const uint64_t v1 = top - 1, v2 = (top - 1) / 2;
    const uint64_t n_odd = (v1 + 1) / 2;  // odd n <= v1
    int8_t *mu = ctx->b_win.as<int8_t>(n_odd + 1);
    mulpf_sieve(ctx, 0, 2 * n_odd, mu, nullptr, nullptr, nullptr);
    unsigned long long *d = ctx->b_small.as<unsigned long long>(8);
    CPX_CUDA(cudaMemsetAsync(d, 0, 8, ctx->stream));
    const unsigned grid = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((n_odd + 255) / 256, ctx->sm_count * 8));
    k_mu_sums<<<grid, 256, 0, ctx->stream>>>(mu, n_odd, v1, v2, d);
    CPX_LAUNCH("k_mu_sums");
    note_launch(ctx);
    unsigned long long h = 0;
    CPX_CUDA(cudaMemcpyAsync(&h, d, 8, cudaMemcpyDeviceToHost, ctx->stream));
    CPX_CUDA(cudaStreamSynchronize(ctx->stream));
    return (int64_t)h;
}

// --------------------------------------------------------- pi table windows

// odd primes in [128*w0, n] from a window table (prefix relative to w0)
__device__ __forceinline__ uint64_t odd_rel(const cpx_pient *__restrict__ T, uint64_t w0, uint64_t n)
{
    if (n < 128 * w0 + 1) return 0;
    const uint64_t w = (n - 1) >> 7;
    const ulonglong2 e = __ldg(reinterpret_cast<const ulonglong2 *>(T) + (w - w0));
    const uint32_t j = (uint32_t)(((n - 1) & 127) >> 1);
    return e.y + __popcll(e.x & ((2ull << j) - 1));
}

// out[k] = pi(base + 2k - 1) - pi(base - 1)   (k = 0 -> 0); base even
__global__ void k_pi_window(const cpx_pient *__restrict__ T, uint64_t w0, uint64_t base, uint64_t K,
                            uint32_t *__restrict__ out)
{
    const uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= K) return;
    if (k == 0) {
        out[0] = 0;
        return;
    }
    const uint64_t n = base + 2 * k - 1;
    uint64_t v = odd_rel(T, w0, n) - (base ? odd_rel(T, w0, base - 1) : 0);
    if (base <= 2 && n >= 2) v += 1;  // the prime 2
    out[k] = (uint32_t)v;
}

// count of primes in [lo, hi) from a window table covering them
__global__ void k_count_window(const cpx_pient *__restrict__ T, uint64_t w0, uint64_t lo, uint64_t hi,
                               unsigned long long *out)
{
    uint64_t v = odd_rel(T, w0, hi - 1) - (lo ? odd_rel(T, w0, lo - 1) : 0);
    if (lo <= 2 && 2 < hi) v += 1;
    atomicAdd(out, (unsigned long long)v);
}

// Window table over [A, B) with A = 128*w0 <= lo and B >= hi into ctx->b_win.
static cpx_pient *window_table(cpx_ctx *ctx, uint64_t lo, uint64_t hi, uint64_t *w0_out)
{
    const uint64_t w0 = lo / 128;
    const uint64_t w1 = (hi + 127) / 128 + 1;
    const uint64_t nwords = (w1 - w0 + kTabSegWords - 1) / kTabSegWords * kTabSegWords;
    ensure_primes(ctx, cpx_isqrt((u128)((w0 + nwords) * 128)) + 2);
    cpx_pient *T = ctx->b_win.as<cpx_pient>(nwords);
    build_pitable_window(ctx, w0, nwords, T);
    *w0_out = w0;
    return T;
}

constexpr uint64_t kWindowSpan = 1ull << 34;  // numbers per streamed window (2 GiB table)

uint64_t count_primes(cpx_ctx *ctx, uint64_t lo, uint64_t hi)
{
    if (hi <= lo) return 0;
    unsigned long long *d = ctx->b_small.as<unsigned long long>(8) + 1;
    CPX_CUDA(cudaMemsetAsync(d, 0, 8, ctx->stream));
    const Tables &tb = ctx->tab;
    if (tb.T && hi - 1 <= tb.tab_n) {
        k_count_window<<<1, 1, 0, ctx->stream>>>(tb.T, 0, lo, hi, d);
        CPX_LAUNCH("k_count_window");
        note_launch(ctx);
    } else {
        for (uint64_t a = lo; a < hi;) {
            const uint64_t b = (hi - a > kWindowSpan) ? a + kWindowSpan : hi;
            uint64_t w0;
            cpx_pient *T = window_table(ctx, a, b, &w0);
            k_count_window<<<1, 1, 0, ctx->stream>>>(T, w0, a, b, d);
            CPX_LAUNCH("k_count_window");
            note_launch(ctx);
            a = b;
        }
    }
    unsigned long long h = 0;
    CPX_CUDA(cudaMemcpyAsync(&h, d, 8, cudaMemcpyDeviceToHost, ctx->stream));
    CPX_CUDA(cudaStreamSynchronize(ctx->stream));
    return h;
}

void pitable_window(cpx_ctx *ctx, uint64_t base, uint64_t range, uint32_t *d_out, uint64_t *pi_base)
{
    if (base & 1) fail(CPX_EINVAL, "window base must be even");
    const uint64_t K = range / 2 + 2;
    const uint64_t top = base + 2 * K;
    const Tables &tb = ctx->tab;
    const cpx_pient *T;
    uint64_t w0 = 0;
    if (tb.T && top <= tb.tab_n) T = tb.T;
    else T = window_table(ctx, base, top, &w0);
    k_pi_window<<<(unsigned)((K + 255) / 256), 256, 0, ctx->stream>>>(T, w0, base, K, d_out);
    CPX_LAUNCH("k_pi_window");
    note_launch(ctx);
    CPX_CUDA(cudaStreamSynchronize(ctx->stream));
    if (pi_base) *pi_base = base ? count_primes(ctx, 0, base) : 0;
}

uint32_t *pitable_dense(cpx_ctx *ctx, uint64_t hi)
{
    if (hi >= (1ull << 32)) fail(CPX_ERANGE, "get_d_piTable takes a 32-bit bound");
    const uint64_t K = hi / 2;
    uint32_t *out = nullptr;
    CPX_CUDA(cudaMalloc(&out, std::max<uint64_t>(K, 1) * 4));
    if (K) {
        ensure_pitable(ctx, hi + 2);
        k_pi_window<<<(unsigned)((K + 255) / 256), 256, 0, ctx->stream>>>(ctx->tab.T, 0, 0, K, out);
        CPX_LAUNCH("k_pi_window");
        note_launch(ctx);
        CPX_CUDA(cudaStreamSynchronize(ctx->stream));
    }
    return out;
}

uint64_t primes_list(cpx_ctx *ctx, uint64_t lo, uint64_t hi, uint64_t **d_out)
{
    if (hi <= lo) {
        *d_out = nullptr;
        CPX_CUDA(cudaMalloc(d_out, 8));
        return 0;
    }
    const uint64_t cnt = count_primes(ctx, lo, hi);
    uint64_t *out = nullptr;
    CPX_CUDA(cudaMalloc(&out, std::max<uint64_t>(cnt, 1) * 8));
    uint64_t done = 0;
    try {
        for (uint64_t a = lo; a < hi;) {
            const uint64_t b = (hi - a > kWindowSpan) ? a + kWindowSpan : hi;
            uint64_t w0;
            const cpx_pient *T;
            const Tables &tb = ctx->tab;
            if (tb.T && b - 1 <= tb.tab_n) {
                T = tb.T;
                w0 = 0;
            } else {
                T = window_table(ctx, a, b, &w0);
            }
            done += extract_window(ctx, T, w0, a, b, out + done);
            a = b;
        }
    } catch (...) {
        cudaFree(out);
        throw;
    }
    CPX_CUDA(cudaStreamSynchronize(ctx->stream));
    *d_out = out;
    return done;
}

// primes of [lo, hi) from a window table; out[k] = k-th prime >= lo
__global__ void k_extract_rel(const cpx_pient *__restrict__ T, uint64_t w0, uint64_t wa, uint64_t wb, uint64_t lo,
                              uint64_t hi, uint64_t base_rel, int has2, uint64_t *__restrict__ out)
{
    const uint64_t w = wa + (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (w == wa && has2) out[0] = 2;
    if (w >= wb) return;
    const ulonglong2 e = reinterpret_cast<const ulonglong2 *>(T)[w - w0];
    uint64_t b = e.x, rank = e.y;
    while (b) {
        const int j = __ffsll((long long)b) - 1;
        b &= b - 1;
        rank++;
        const uint64_t p = 128 * w + 2 * j + 1;
        if (p >= lo && p < hi) out[has2 + rank - base_rel - 1] = p;
    }
}

__global__ void k_odd_rel_one(const cpx_pient *__restrict__ T, uint64_t w0, uint64_t n, unsigned long long *out)
{
    *out = (n == (uint64_t)-1) ? 0 : odd_rel(T, w0, n);
}

uint64_t extract_window(cpx_ctx *ctx, const cpx_pient *T, uint64_t w0, uint64_t lo, uint64_t hi, uint64_t *out)
{
    // base_rel = odd primes of the window below lo
    unsigned long long *d = ctx->b_small.as<unsigned long long>(8) + 2;
    k_odd_rel_one<<<1, 1, 0, ctx->stream>>>(T, w0, lo ? lo - 1 : (uint64_t)-1, d);
    CPX_LAUNCH("k_odd_rel_one");
    note_launch(ctx);
    unsigned long long base_rel = 0;
    CPX_CUDA(cudaMemcpyAsync(&base_rel, d, 8, cudaMemcpyDeviceToHost, ctx->stream));
    CPX_CUDA(cudaStreamSynchronize(ctx->stream));
    const int has2 = (lo <= 2 && 2 < hi) ? 1 : 0;
    const uint64_t wa = lo / 128, wb = (hi - 1) / 128 + 1;
    k_extract_rel<<<(unsigned)((wb - wa + 255) / 256), 256, 0, ctx->stream>>>(T, w0, wa, wb, lo, hi, base_rel, has2,
                                                                                out);
    CPX_LAUNCH("k_extract_rel");
    note_launch(ctx);
    // count written = has2 + odd primes in [lo, hi)
    k_odd_rel_one<<<1, 1, 0, ctx->stream>>>(T, w0, hi - 1, d);
    CPX_LAUNCH("k_odd_rel_one");
    note_launch(ctx);
    unsigned long long top_rel = 0;
    CPX_CUDA(cudaMemcpyAsync(&top_rel, d, 8, cudaMemcpyDeviceToHost, ctx->stream));
    CPX_CUDA(cudaStreamSynchronize(ctx->stream));
    return has2 + (top_rel - base_rel);
}

// ------------------------------------------------------------------ phi sieve
// Odd-only bitmap of [2*64*w0, ...): bit set iff n has no prime factor among
// p_2 .. p_a (n = 1 stays set).  One CTA per 2^18 odd numbers; p < 64 by
// residue masks per word, larger p by strided shared-memory atomicAnd.
// Either writes the words (out) or adds popcount(n <= nmax) to *count.
constexpr uint32_t kPhiSegW = 4096;  // 64-bit words per CTA

__global__ void __launch_bounds__(256) k_phi_sieve(uint64_t w0, const uint32_t *__restrict__ P, uint32_t a,
                                                   uint64_t *__restrict__ out, uint64_t nwords_out, uint64_t nmax,
                                                   unsigned long long *__restrict__ count)
{
    __shared__ uint32_t bm[2 * kPhiSegW];
    const uint32_t tid = threadIdx.x;
    const uint64_t wbase = w0 + (uint64_t)blockIdx.x * kPhiSegW;  // in 64-bit words
    const uint64_t lo = wbase * 128;
    const uint64_t hi = lo + 128ull * kPhiSegW;
    constexpr uint32_t NB = 2 * kPhiSegW * 32;
    for (uint32_t w = tid; w < 2 * kPhiSegW; w += 256) {
        // 32-bit word w covers n = lo + 64 w + 2k + 1
        uint32_t m = 0;
        for (uint32_t i = 1; i < a; i++) {
            const uint32_t p = P[i];
            if (p >= 64) break;
            const uint32_t r = (uint32_t)((lo + 64ull * w + 1) % p);
            const uint32_t k0 = (r == 0) ? 0u : ((r & 1u) ? (p - r) >> 1 : p - (r >> 1));
            for (uint32_t k = k0; k < 32; k += p) m |= 1u << k;
        }
        bm[w] = ~m;
    }
    __syncthreads();
    for (uint32_t i = 1; i < a; i++) {
        const uint64_t p = P[i];
        if (p < 64) continue;
        if (p >= hi) break;
        const uint64_t r = (lo + 1) % p;
        uint64_t m = lo + 1 + (r ? p - r : 0);
        if ((m & 1) == 0) m += p;
        if (m >= hi) continue;
        const uint64_t i0 = (m - lo - 1) >> 1;
        for (uint64_t bi = i0 + tid * p; bi < NB; bi += 256 * p) atomicAnd(&bm[bi >> 5], ~(1u << (bi & 31)));
    }
    __syncthreads();
    const uint64_t *bm64 = reinterpret_cast<const uint64_t *>(bm);
    if (out) {
        for (uint32_t w = tid; w < kPhiSegW; w += 256) {
            const uint64_t gw = wbase + w;
            if (gw - w0 < nwords_out) out[gw - w0] = bm64[w];
        }
    }
    if (count) {
        unsigned long long s = 0;
        for (uint32_t w = tid; w < kPhiSegW; w += 256) {
            const uint64_t base = 128 * (wbase + w);
            if (base + 1 > nmax) continue;
            uint64_t b = bm64[w];
            const uint64_t lim = nmax - base - 1;  // bit j valid iff 2j <= lim
            if (lim < 127) {
                const uint32_t j = (uint32_t)(lim >> 1);
                b &= (2ull << j) - 1;
            }
            s += __popcll(b);
        }
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) s += __shfl_down_sync(0xffffffffu, s, d);
        if ((tid & 31) == 0 && s) atomicAdd(count, s);
    }
}

static void ensure_nth_prime(cpx_ctx *ctx, uint32_t a)
{
    uint64_t pm = std::max<uint64_t>(ctx->tab.prm_max, 1 << 16);
    ensure_primes(ctx, pm);
    while (ctx->tab.prm_n <= a) {
        pm *= 2;
        ensure_primes(ctx, pm);
    }
}

uint64_t phi_count(cpx_ctx *ctx, uint64_t x, uint32_t a)
{
    if (a == 0 || x == 0) return x;
    ensure_nth_prime(ctx, a);
    const uint64_t nw = x / 128 + 1;
    const uint64_t nseg = (nw + kPhiSegW - 1) / kPhiSegW;
    unsigned long long *d = ctx->b_small.as<unsigned long long>(8) + 3;
    CPX_CUDA(cudaMemsetAsync(d, 0, 8, ctx->stream));
    for (uint64_t s0 = 0; s0 < nseg; s0 += 1u << 30) {
        const uint64_t ns = std::min<uint64_t>(nseg - s0, 1u << 30);
        k_phi_sieve<<<(unsigned)ns, 256, 0, ctx->stream>>>(s0 * kPhiSegW, ctx->tab.P, a, nullptr, 0, x, d);
        CPX_LAUNCH("k_phi_sieve");
        note_launch(ctx);
    }
    unsigned long long h = 0;
    CPX_CUDA(cudaMemcpyAsync(&h, d, 8, cudaMemcpyDeviceToHost, ctx->stream));
    CPX_CUDA(cudaStreamSynchronize(ctx->stream));
    return h;
}

// counts[i] = prefix(word of i) + popcount of the lower bits, exclusive
// (inclusive = 1 adds bit i itself)
__global__ void k_expand_counts(const uint64_t *__restrict__ words, const uint64_t *__restrict__ wpre, uint64_t nbits,
                                int inclusive, uint32_t *__restrict__ out)
{
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nbits) return;
    const uint64_t w = i >> 6;
    const uint32_t j = i & 63;
    const uint64_t m = inclusive ? ((j == 63) ? ~0ull : ((2ull << j) - 1)) : ((1ull << j) - 1);
    out[i] = (uint32_t)(wpre[w] + __popcll(words[w] & m));
}

__global__ void k_popc_words(const uint64_t *__restrict__ words, uint64_t n, uint64_t *__restrict__ out)
{
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = __popcll(words[i]);
}

// bits over odd numbers [0, 2*nbits), crossed by p_2..p_a, into words (nwords)
void phi_bits(cpx_ctx *ctx, uint64_t nwords, uint32_t a, uint64_t *words)
{
    if (a >= 1) ensure_nth_prime(ctx, a);
    const uint64_t nseg = (nwords + kPhiSegW - 1) / kPhiSegW;
    if (nseg > 0x7FFFFFFFull) fail(CPX_ERANGE, "phi sieve too large");
    k_phi_sieve<<<(unsigned)nseg, 256, 0, ctx->stream>>>(0, ctx->tab.P, a == 0 ? 1 : a, words, nwords, 0, nullptr);
    CPX_LAUNCH("k_phi_sieve");
    note_launch(ctx);
}

void counts_from_bits(cpx_ctx *ctx, const uint64_t *words, uint64_t nwords, uint64_t nbits, int inclusive,
                      uint32_t *out)
{
    uint64_t *wpre = ctx->b_win2.as<uint64_t>(nwords + 1);
    k_popc_words<<<(unsigned)((nwords + 255) / 256), 256, 0, ctx->stream>>>(words, nwords, wpre);
    CPX_LAUNCH("k_popc_words");
    note_launch(ctx);
    scan_u64(ctx, wpre, nwords);
    k_expand_counts<<<(unsigned)((nbits + 255) / 256), 256, 0, ctx->stream>>>(words, wpre, nbits, inclusive, out);
    CPX_LAUNCH("k_expand_counts");
    note_launch(ctx);
}

uint32_t *phi_range(cpx_ctx *ctx, uint32_t num, uint32_t a)
{
    const uint64_t nbits = num / 2;
    uint32_t *out = nullptr;
    CPX_CUDA(cudaMalloc(&out, std::max<uint64_t>(nbits, 1) * 4));
    if (!nbits) return out;
    const uint64_t nwords = (nbits + 63) / 64;
    uint64_t *words = ctx->b_win.as<uint64_t>(nwords);
    phi_bits(ctx, nwords, a, words);
    counts_from_bits(ctx, words, nwords, nbits, 1, out);
    CPX_CUDA(cudaStreamSynchronize(ctx->stream));
    return out;
}

// ------------------------------------------------------------------ Phisieve

__global__ void k_cross_global(uint64_t *words, uint64_t nbits, uint64_t p)
{
    // odd multiples n = p, 3p, ... ; bit (n - 1) / 2
    const uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;  // multiple index
    const uint64_t n = p * (2 * k + 1);
    const uint64_t i = (n - 1) >> 1;
    if (i >= nbits) return;
    atomicAnd(reinterpret_cast<unsigned long long *>(words) + (i >> 6), ~(1ull << (i & 63)));
}

void phisieve_cross(cpx_ctx *ctx, uint64_t *words, uint64_t nbits, uint64_t p)
{
    const uint64_t nmult = (2 * nbits / p + 1) / 2 + 1;
    k_cross_global<<<(unsigned)((nmult + 255) / 256), 256, 0, ctx->stream>>>(words, nbits, p);
    CPX_LAUNCH("k_cross_global");
    note_launch(ctx);
}

}  // namespace cpx
