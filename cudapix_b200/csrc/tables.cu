// tables.cu -- device tables shared by every term: prime list, compressed pi
// table, packed mu/lpf array, wheel phi table.
//
// Replaces the reference's table builders and its CUDASieve dependency:
//   CudaSieve::getDevicePrimes/countPrimes/genDeviceBitSieve (external; call
//     sites e.g. src/P2.cu:100,103, src/sieve/S2_hard_host.cu:64-65)
//   get_d_piTable / PiTable / transposePrimes      src/pitable.cu:10-218
//   lpf_kernel / mu_kernel / gen_d_*                src/sieve/lpf_mu.cu:25-302
//   Phisieve wheel count table                      src/sieve/phisieve_host.cu:48-56
//
// Layout in HBM (see cpx_int.cuh): the pi table is one 16-byte entry per 128
// integers {64-bit odd-number bitmap, odd primes below the entry}, so pi(n)
// costs one 16-byte load and a popcount, and a table to N takes N/8 bytes.
#include <mutex>
#include <algorithm>

#include "cpx_internal.h"

namespace cpx {

// ------------------------------------------------------------------ errors

void fail(int code, const std::string &msg) { throw Error{code, msg}; }

void check_cuda(cudaError_t e, const char *what)
{
    if (e == cudaSuccess) return;
    int code = (e == cudaErrorMemoryAllocation) ? CPX_EOOM : CPX_ECUDA;
    if (e == cudaErrorMemoryAllocation) cudaGetLastError();  // clear the sticky-free error
    fail(code, std::string(what) + ": " + cudaGetErrorString(e));
}

// Grows by at least half its size: a run of queries of rising size then
// reallocates a few times instead of at every new maximum (each reallocation
// frees, which waits for the device, and maps fresh memory).
void *DevBuf::get(size_t need)
{
    if (need <= bytes && p) return p;
    const size_t grown = bytes + bytes / 2;
    release();
    size_t n = std::max<size_t>(std::max(need, grown), 256);
    n = (n + 255) & ~size_t(255);
    if (stream) CPX_CUDA(cudaMallocAsync(&p, n, stream));
    else CPX_CUDA(cudaMalloc(&p, n));
    bytes = n;
    return p;
}

void DevBuf::release()
{
    if (p) {
        if (stream) cudaFreeAsync(p, stream);
        else cudaFree(p);
    }
    p = nullptr;
    bytes = 0;
}

// ------------------------------------------------------------------- scans

constexpr int kScanItems = 4;  // per thread
constexpr int kScanBlock = kThreads * kScanItems;

__global__ void __launch_bounds__(kThreads) k_scan_block(uint64_t *d, uint64_t n, uint64_t *sums)
{
    __shared__ uint64_t wsum[kThreads / 32];
    const uint64_t base = (uint64_t)blockIdx.x * kScanBlock + threadIdx.x * kScanItems;
    uint64_t v[kScanItems], t = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; i++) {
        v[i] = (base + i < n) ? d[base + i] : 0;
        t += v[i];
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    uint64_t inc = t;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint64_t u = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += u;
    }
    if (lane == 31) wsum[w] = inc;
    __syncthreads();
    uint64_t woff = 0;
    for (int k = 0; k < w; k++) woff += wsum[k];
    uint64_t run = woff + inc - t;
#pragma unroll
    for (int i = 0; i < kScanItems; i++) {
        if (base + i < n) d[base + i] = run;
        run += v[i];
    }
    if (threadIdx.x == kThreads - 1) sums[blockIdx.x] = run;
}

__global__ void k_scan_add(uint64_t *d, uint64_t n, const uint64_t *sums)
{
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) d[i] += sums[i / kScanBlock];
}

static void scan_u64_rec(cpx_ctx *ctx, uint64_t *d, uint64_t n, int depth)
{
    if (n == 0) return;
    uint64_t nb = (n + kScanBlock - 1) / kScanBlock;
    if (depth > 2) fail(CPX_ERANGE, "scan too large");
    uint64_t *sums = ctx->b_scan[depth].as<uint64_t>(nb + 1);
    k_scan_block<<<(unsigned)nb, kThreads, 0, ctx->stream>>>(d, n, sums);
    CPX_LAUNCH("k_scan_block");
    note_launch(ctx);
    if (nb > 1) {
        scan_u64_rec(ctx, sums, nb, depth + 1);
        k_scan_add<<<(unsigned)((n + 255) / 256), 256, 0, ctx->stream>>>(d, n, sums);
        CPX_LAUNCH("k_scan_add");
        note_launch(ctx);
    }
}

void scan_u64(cpx_ctx *ctx, uint64_t *d, uint64_t n) { scan_u64_rec(ctx, d, n, 0); }

void scan_reserve(cpx_ctx *ctx, uint64_t n)
{
    for (int depth = 0; depth < 3 && n > 0; depth++) {
        const uint64_t nb = (n + kScanBlock - 1) / kScanBlock;
        ctx->b_scan[depth].as<uint64_t>(nb + 1);
        if (nb <= 1) break;
        n = nb;
    }
}

// ---------------------------------------------------- bootstrap: trial division

// Table entries for [0, 65536) by trial division (one entry per thread, one
// CTA of 512 threads), the seed of every larger sieve.
__global__ void __launch_bounds__(512) k_trial_table(cpx_pient *T)
{
    __shared__ uint64_t wsum[16];
    const uint32_t w = threadIdx.x;
    uint64_t bits = 0;
    for (uint32_t j = 0; j < 64; j++) {
        uint32_t n = 128 * w + 2 * j + 1;
        bool pr = n >= 3;
        for (uint32_t d = 3; pr && d * d <= n; d += 2)
            if (n % d == 0) pr = false;
        if (pr) bits |= 1ull << j;
    }
    uint64_t c = __popcll(bits), inc = c;
    const int lane = threadIdx.x & 31, wi = threadIdx.x >> 5;
    for (int o = 1; o < 32; o <<= 1) {
        uint64_t u = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += u;
    }
    if (lane == 31) wsum[wi] = inc;
    __syncthreads();
    uint64_t off = 0;
    for (int k = 0; k < wi; k++) off += wsum[k];
    T[w].bits = bits;
    T[w].pre = off + inc - c;
}

// ------------------------------------------------------ segmented prime sieve

// Odd primes 3..31 are removed with per-word residue masks; 37..8191 by all
// threads together (one prime at a time, strided multiples, shared-memory
// atomicAnd); larger primes one per thread.
constexpr int kSmallCnt = 10;  // 3 .. 31
__constant__ uint32_t c_small[kSmallCnt] = {3, 5, 7, 11, 13, 17, 19, 23, 29, 31};
constexpr uint32_t kCoopMax = 1017;  // primes in [37, 8192)

__device__ __forceinline__ uint32_t first_odd_multiple_idx(uint64_t lo, uint64_t hi, uint64_t p,
                                                            bool from_square)
{
    // bit index of the first odd multiple m of p with m >= lo + 1 (and, for
    // prime sieving, m >= p^2); 0xFFFFFFFF if none below hi.  (lo + 1) mod p
    // by the reciprocal quotient (p < 2^32), not the 64-bit division routine
    uint64_t r = (lo + 1) - cpx_udiv_leaf(lo + 1, p) * p;
    uint64_t m = lo + 1 + (r ? p - r : 0);
    if ((m & 1) == 0) m += p;
    if (from_square && m < p * p) m = p * p;
    if (m >= hi) return 0xFFFFFFFFu;
    return (uint32_t)((m - lo - 1) >> 1);
}

// One CTA sieves MUL table blocks of kTabSegWords entries (2^18 odd numbers
// each) with MUL x 256 threads and writes, per block, its entries (prefix
// relative to the block) and its total.  A CTA pays the start offset of every
// sieving prime once for all its numbers, so MUL = 4 (2^20 odd numbers, 128 KB
// of dynamic shared memory) spreads that cost over four times the numbers
// for the large windows of P2 beyond the resident table.
template <int MUL>
__global__ void __launch_bounds__(kThreads * MUL) k_sieve_table(uint64_t w0, const uint32_t *__restrict__ sp,
                                                                uint32_t nsp, uint32_t ncoop,
                                                                cpx_pient *__restrict__ T,
                                                                uint64_t *__restrict__ segtot)
{
    constexpr uint32_t NT = kThreads * MUL;
    constexpr uint32_t NW32 = kTabSegWords * 2 * MUL;  // 8192 MUL words = 2^18 MUL bits
    constexpr uint32_t NBITS = NW32 * 32;
    extern __shared__ uint32_t bm[];  // NW32 words
    __shared__ uint32_t off[kCoopMax];
    __shared__ uint32_t pat[160];
    __shared__ uint32_t lomod[kSmallCnt];
    __shared__ uint64_t wsum[NT / 32];
    const uint32_t tid = threadIdx.x;
    const uint64_t wbase = w0 + (uint64_t)blockIdx.x * kTabSegWords * MUL;
    const uint64_t lo = wbase * 128, hi = lo + kTabSegNumbers * MUL;

    // residue masks: pat[o_p + r] = bits k < 32 with (r + 2k) % p == 0
    if (tid < 158) {
        uint32_t o = 0, i = 0;
        while (tid >= o + c_small[i]) o += c_small[i++];
        uint32_t p = c_small[i], r = tid - o, m = 0;
        for (uint32_t k = 0; k < 32; k++)
            if ((r + 2 * k) % p == 0) m |= 1u << k;
        pat[tid] = m;
    }
    if (tid < kSmallCnt) lomod[tid] = (uint32_t)((lo + 1) % c_small[tid]);
    for (uint32_t k = tid; k < ncoop; k += NT)
        off[k] = first_odd_multiple_idx(lo, hi, sp[k], true);
    __syncthreads();

    {
        uint32_t r[kSmallCnt], step[kSmallCnt], base[kSmallCnt];
        uint32_t o = 0;
#pragma unroll
        for (int i = 0; i < kSmallCnt; i++) {
            const uint32_t p = c_small[i];
            r[i] = (lomod[i] + (64u * tid) % p) % p;
            step[i] = (64u * NT) % p;
            base[i] = o;
            o += p;
        }
        for (uint32_t w = tid; w < NW32; w += NT) {
            uint32_t m = 0;
#pragma unroll
            for (int i = 0; i < kSmallCnt; i++) {
                m |= pat[base[i] + r[i]];
                r[i] += step[i];
                if (r[i] >= c_small[i]) r[i] -= c_small[i];
            }
            bm[w] = ~m;
        }
    }
    __syncthreads();

    for (uint32_t k = 0; k < ncoop; k++) {
        const uint32_t i0 = off[k];
        if (i0 == 0xFFFFFFFFu) continue;
        const uint32_t p = sp[k];
        for (uint32_t i = i0 + tid * p; i < NBITS; i += NT * p) atomicAnd(&bm[i >> 5], ~(1u << (i & 31)));
    }
    for (uint32_t k = ncoop + tid; k < nsp; k += NT) {
        const uint64_t p = sp[k];
        if (p * p >= hi) break;
        uint32_t i0 = first_odd_multiple_idx(lo, hi, p, true);
        if (i0 == 0xFFFFFFFFu) continue;
        for (uint64_t i = i0; i < NBITS; i += p) atomicAnd(&bm[i >> 5], ~(1u << (i & 31)));
    }
    __syncthreads();
    if (lo == 0 && tid == 0) {
        // 1 is not prime; the residue masks removed 3..31 themselves
        uint32_t v = bm[0] & ~1u;
        v |= (1u << 1) | (1u << 2) | (1u << 3) | (1u << 5) | (1u << 6) | (1u << 8) | (1u << 9) |
             (1u << 11) | (1u << 14) | (1u << 15);
        bm[0] = v;
    }
    __syncthreads();

    // per-warp popcount totals, then a warp-level scan writing {bits, prefix}
    // with prefixes relative to the warp's table block (8 warps a block)
    const int lane = tid & 31, wi = tid >> 5;
    const uint64_t *bm64 = reinterpret_cast<const uint64_t *>(bm);
    constexpr uint32_t PER_WARP = kTabSegWords / (kThreads / 32);  // 512
    uint64_t s = 0;
    for (uint32_t i = 0; i < PER_WARP / 32; i++) s += __popcll(bm64[wi * PER_WARP + 32 * i + lane]);
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) s += __shfl_down_sync(0xffffffffu, s, d);
    if (lane == 0) wsum[wi] = s;
    __syncthreads();
    const int blk = wi / (kThreads / 32);
    uint64_t run = 0;
    for (int k = blk * (kThreads / 32); k < wi; k++) run += wsum[k];
    for (uint32_t i = 0; i < PER_WARP / 32; i++) {
        const uint32_t wl = wi * PER_WARP + 32 * i + lane;
        const uint64_t b = bm64[wl];
        const uint64_t c = __popcll(b);
        uint64_t inc = c;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint64_t u = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= o) inc += u;
        }
        ulonglong2 e;
        e.x = b;
        e.y = run + inc - c;
        reinterpret_cast<ulonglong2 *>(T)[wbase - w0 + wl] = e;
        run += __shfl_sync(0xffffffffu, inc, 31);
    }
    if (tid < MUL) {
        uint64_t t = 0;
        for (int k = 0; k < kThreads / 32; k++) t += wsum[tid * (kThreads / 32) + k];
        segtot[(uint64_t)blockIdx.x * MUL + tid] = t;
    }
}

__global__ void k_table_fix(cpx_pient *T, uint64_t nwords, const uint64_t *segpre)
{
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nwords) T[i].pre += segpre[i / kTabSegWords];
}

// total odd primes of a window: segpre[nseg-1] + segtot[nseg-1]
__global__ void k_window_total(const uint64_t *segpre, const cpx_pient *T, uint64_t nwords, uint64_t *out)
{
    const cpx_pient e = T[nwords - 1];
    *out = e.pre + __popcll(e.bits);
}

// Extraction: primes p in [lo, hi) from table words; out[pi(p) - base - 1] = p.
template <class OutT>
__global__ void k_extract(const cpx_pient *__restrict__ T, uint64_t w_lo, uint64_t w_hi, uint64_t lo,
                          uint64_t hi, const uint64_t *__restrict__ d_base, OutT *__restrict__ out)
{
    const uint64_t w = w_lo + (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t base = *d_base;  // pi(lo - 1)
    if (w == w_lo && lo <= 2 && 2 < hi) out[0] = 2;
    if (w >= w_hi) return;
    cpx_pient e = T[w];
    uint64_t b = e.bits;
    uint64_t rank = e.pre;  // odd primes before this word
    while (b) {
        const int j = __ffsll((long long)b) - 1;
        b &= b - 1;
        rank++;
        const uint64_t p = 128 * w + 2 * j + 1;
        if (p >= lo && p < hi) out[rank + 1 - base - 1] = (OutT)p;
    }
}

// pi(n) for a small array of n (n within the table)
__global__ void k_pi_many(const cpx_pient *__restrict__ T, const uint64_t *n, uint64_t *out, int k)
{
    const int i = threadIdx.x;
    if (i < k) out[i] = cpx_pi_dev(T, n[i]);
}

// ------------------------------------------------------------ table drivers

static uint64_t roundup(uint64_t a, uint64_t b) { return (a + b - 1) / b * b; }

static void sync(cpx_ctx *ctx) { CPX_CUDA(cudaStreamSynchronize(ctx->stream)); }

// sieve table words [w0, w0 + nwords) into T (prefix relative to the window)
// with the resident prime list, which must reach sqrt of the window top.
uint64_t build_pitable_window(cpx_ctx *ctx, uint64_t w0, uint64_t nwords, cpx_pient *T)
{
    Tables &tb = ctx->tab;
    nwords = roundup(nwords, kTabSegWords);
    const uint64_t top = (w0 + nwords) * 128;
    if (tb.prm_max < cpx_isqrt((u128)(top - 1)))
        fail(CPX_ESTATE, "prime list does not reach sqrt of the table window");
    const uint64_t nseg = nwords / kTabSegWords;
    if (nseg == 0) return 0;
    if (nseg > 0x7FFFFFFFull) fail(CPX_ERANGE, "pi table window too large");
    uint64_t *segtot = ctx->b_segtot.as<uint64_t>(nseg + 1);
    // sieving primes P[11..] = 37, 41, ...; the kernel stops at p^2 >= segment top
    const uint32_t nsp_all = (uint32_t)(tb.prm_n > 11 ? tb.prm_n - 11 : 0);
    const uint32_t ncoop = std::min<uint32_t>(kCoopMax, nsp_all);
    // four table blocks a CTA when the window is large and a multiple of four blocks
    constexpr int kMul = 4;
    const size_t smem4 = kTabSegWords * 2 * kMul * 4;
    if (nseg % kMul == 0 && nseg >= (uint64_t)kMul * ctx->sm_count && ctx->smem_optin >= smem4 + 8192) {
        static std::mutex m;
        static int done_dev = -1;
        {
            std::lock_guard<std::mutex> g(m);
            if (done_dev != ctx->device) {
                CPX_CUDA(cudaFuncSetAttribute(k_sieve_table<kMul>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              (int)smem4));
                done_dev = ctx->device;
            }
        }
        k_sieve_table<kMul><<<(unsigned)(nseg / kMul), kThreads * kMul, smem4, ctx->stream>>>(w0, tb.P + 11, nsp_all,
                                                                                              ncoop, T, segtot);
    } else {
        k_sieve_table<1><<<(unsigned)nseg, kThreads, kTabSegWords * 2 * 4, ctx->stream>>>(w0, tb.P + 11, nsp_all,
                                                                                         ncoop, T, segtot);
    }
    CPX_LAUNCH("k_sieve_table");
    note_launch(ctx);
    scan_u64(ctx, segtot, nseg);
    k_table_fix<<<(unsigned)((nwords + 255) / 256), 256, 0, ctx->stream>>>(T, nwords, segtot);
    CPX_LAUNCH("k_table_fix");
    note_launch(ctx);
    uint64_t *d_total = ctx->b_small.as<uint64_t>(8) + 7;
    k_window_total<<<1, 1, 0, ctx->stream>>>(segtot, T, nwords, d_total);
    CPX_LAUNCH("k_window_total");
    note_launch(ctx);
    uint64_t h_total = 0;
    CPX_CUDA(cudaMemcpyAsync(&h_total, d_total, 8, cudaMemcpyDeviceToHost, ctx->stream));
    sync(ctx);
    return h_total;
}

static void bootstrap_primes(cpx_ctx *ctx)
{
    Tables &tb = ctx->tab;
    cpx_pient *T0 = ctx->b_tmp.as<cpx_pient>(512);
    k_trial_table<<<1, 512, 0, ctx->stream>>>(T0);
    CPX_LAUNCH("k_trial_table");
    note_launch(ctx);
    cpx_pient last;
    CPX_CUDA(cudaMemcpyAsync(&last, T0 + 511, sizeof(last), cudaMemcpyDeviceToHost, ctx->stream));
    sync(ctx);
    const uint64_t n = 1 + last.pre + __builtin_popcountll(last.bits);  // pi(65535)
    uint32_t *P = nullptr;
    CPX_CUDA(cudaMalloc(&P, n * 4));
    uint64_t *d_zero = ctx->b_small.as<uint64_t>(8);
    CPX_CUDA(cudaMemsetAsync(d_zero, 0, 8, ctx->stream));
    k_extract<uint32_t><<<2, 256, 0, ctx->stream>>>(T0, 0, 512, 0, 65536, d_zero, P);
    CPX_LAUNCH("k_extract");
    note_launch(ctx);
    sync(ctx);
    if (tb.P) cudaFree(tb.P);
    tb.P = P;
    tb.prm_n = n;
    tb.prm_max = 65535;
}

void ensure_primes(cpx_ctx *ctx, uint64_t pmax)
{
    Tables &tb = ctx->tab;
    if (tb.P && tb.prm_max >= pmax) return;
    if (!tb.P) bootstrap_primes(ctx);
    if (tb.prm_max >= pmax) return;
    if (pmax >= 0xFFFFFFF0ull) fail(CPX_ERANGE, "prime list bound beyond 32 bits");
    // sieve [0, pmax] into a temporary table, then extract every prime
    const uint64_t nwords = roundup(pmax / 128 + 1, kTabSegWords);
    ensure_primes(ctx, cpx_isqrt((u128)(nwords * 128 - 1)) + 1);
    cpx_pient *Tt = nullptr;
    CPX_CUDA(cudaMalloc(&Tt, nwords * sizeof(cpx_pient)));
    uint64_t nodd = 0;
    try {
        build_pitable_window(ctx, 0, nwords, Tt);
        // pi(pmax)
        uint64_t *d_n = ctx->b_small.as<uint64_t>(8);
        uint64_t h_n[2] = {pmax, 0};
        CPX_CUDA(cudaMemcpyAsync(d_n, h_n, 8, cudaMemcpyHostToDevice, ctx->stream));
        k_pi_many<<<1, 32, 0, ctx->stream>>>(Tt, d_n, d_n + 1, 1);
        CPX_LAUNCH("k_pi_many");
        note_launch(ctx);
        CPX_CUDA(cudaMemcpyAsync(&nodd, d_n + 1, 8, cudaMemcpyDeviceToHost, ctx->stream));
        sync(ctx);
        uint32_t *P = nullptr;
        CPX_CUDA(cudaMalloc(&P, nodd * 4));
        CPX_CUDA(cudaMemsetAsync(d_n, 0, 8, ctx->stream));
        const uint64_t wh = pmax / 128 + 1;
        k_extract<uint32_t><<<(unsigned)((wh + 255) / 256), 256, 0, ctx->stream>>>(Tt, 0, wh, 0, pmax + 1,
                                                                                    d_n, P);
        CPX_LAUNCH("k_extract");
        note_launch(ctx);
        sync(ctx);
        cudaFree(tb.P);
        tb.P = P;
        tb.prm_n = nodd;
        tb.prm_max = pmax;
    } catch (...) {
        cudaFree(Tt);
        throw;
    }
    cudaFree(Tt);
}

void ensure_pitable(cpx_ctx *ctx, uint64_t nmax)
{
    Tables &tb = ctx->tab;
    if (tb.T && tb.tab_n >= nmax) return;
    // grow geometrically so that a stream of slowly growing requests does not
    // rebuild every time
    uint64_t want = std::max<uint64_t>(nmax, tb.tab_n + tb.tab_n / 2);
    want = std::max<uint64_t>(want, 1ull << 20);
    const uint64_t nwords = roundup(want / 128 + 1, kTabSegWords);
    ensure_primes(ctx, cpx_isqrt((u128)(nwords * 128 - 1)) + 1);
    if (tb.T) {
        cudaFree(tb.T);
        tb.T = nullptr;
        tb.tab_n = 0;
    }
    CPX_CUDA(cudaMalloc(&tb.T, nwords * sizeof(cpx_pient)));
    build_pitable_window(ctx, 0, nwords, tb.T);
    tb.tab_words = nwords;
    tb.tab_n = nwords * 128 - 1;
    tb.version++;
}

uint64_t extract_primes_u64(cpx_ctx *ctx, uint64_t lo, uint64_t hi, uint64_t *d_out, uint64_t cap)
{
    Tables &tb = ctx->tab;
    if (hi <= lo) return 0;
    ensure_pitable(ctx, hi);
    uint64_t *d_n = ctx->b_small.as<uint64_t>(8);
    uint64_t h_n[2] = {lo ? lo - 1 : 0, hi - 1};
    CPX_CUDA(cudaMemcpyAsync(d_n, h_n, 16, cudaMemcpyHostToDevice, ctx->stream));
    k_pi_many<<<1, 32, 0, ctx->stream>>>(tb.T, d_n, d_n + 2, 2);
    CPX_LAUNCH("k_pi_many");
    note_launch(ctx);
    uint64_t res[2];
    CPX_CUDA(cudaMemcpyAsync(res, d_n + 2, 16, cudaMemcpyDeviceToHost, ctx->stream));
    sync(ctx);
    const uint64_t cnt = res[1] - res[0];
    if (!d_out) return cnt;
    if (cnt > cap) fail(CPX_ERANGE, "prime output buffer too small");
    const uint64_t w_lo = lo / 128, w_hi = (hi - 1) / 128 + 1;
    const uint64_t nw = w_hi - w_lo;
    k_extract<uint64_t><<<(unsigned)((nw + 255) / 256), 256, 0, ctx->stream>>>(tb.T, w_lo, w_hi, lo, hi,
                                                                               d_n + 2, d_out);
    CPX_LAUNCH("k_extract");
    note_launch(ctx);
    return cnt;
}

// ----------------------------------------------------------- mu / lpf sieve

// odd numbers per CTA: 8 bytes of shared state each for 32-bit words, 12 for 64-bit
template <class W> struct MuSeg { static constexpr uint32_t N = sizeof(W) == 4 ? 4096 : 2048; };

// Mitchell's approximation of log2(v), v >= 1, in units of 2^-16: the bit
// position of the leading one plus the next 16 bits read as a fraction.  It
// never exceeds log2(v) and falls short of it by less than 0.0861 + 2^-16.
__device__ __forceinline__ uint32_t mitchell_log2_q16(uint64_t v)
{
    const int e = 63 - __clzll((long long)v);
    const uint64_t frac = ((v << (63 - e)) << 1) >> 48;
    return ((uint32_t)e << 16) | (uint32_t)frac;
}

// Per odd n of the segment (sieving primes p with p^2 < hi):
//   s_lpf: the smallest prime factor found (atomicMin);
//   s_acc: bits 0..23 the sum of mitchell_log2_q16(p) over the distinct
//          prime factors found, bits 24..29 their count, bit 31 a square
//          factor (one atomicAdd and, for multiples of p^2, one atomicOr).
// An odd n < hi has at most one prime factor q that is not found (q^2 >= hi),
// and only then is the log sum short of mitchell_log2_q16(n) by log2(q) > 1.49
// less the approximation errors; without it the sum exceeds the log of n by at
// most 15 x 0.0862 < 1.3 (an odd n < 2^64 has at most 15 distinct prime
// factors).  So "cofactor" is exactly: log of n minus the sum > 1.4.
// The reference multiplies the prime factors into a word with a
// compare-and-swap loop (src/sieve/lpf_mu.cu:89-108); the log sum needs none.
constexpr uint32_t kCofactorQ16 = 91750;  // 1.4 in units of 2^-16
template <class W>
__global__ void __launch_bounds__(kThreads) k_mulpf(uint64_t lo0, uint64_t hi_all, const uint32_t *__restrict__ P,
                                                    uint32_t np, uint32_t nsmall, int8_t *__restrict__ mu,
                                                    uint32_t *__restrict__ lpf32, uint64_t *__restrict__ lpf64,
                                                    int32_t *__restrict__ packed)
{
    constexpr uint32_t kMuSeg = MuSeg<W>::N;
    __shared__ W s_lpf[kMuSeg];
    __shared__ uint32_t s_acc[kMuSeg];
    const uint32_t tid = threadIdx.x;
    const uint64_t lo = lo0 + (uint64_t)blockIdx.x * 2 * kMuSeg;
    const uint64_t hi = lo + 2 * kMuSeg;  // exclusive
    for (uint32_t i = tid; i < kMuSeg; i += kThreads) {
        s_lpf[i] = (W)~(W)0;
        s_acc[i] = 0;
    }
    __syncthreads();
    auto square_flags = [&](uint64_t p, uint32_t t0, uint32_t step) {
        const uint64_t p2 = p * p;
        if (p2 >= hi) return;
        uint64_t r = (lo + 1) % p2;
        uint64_t m = lo + 1 + (r ? p2 - r : 0);
        if ((m & 1) == 0) m += p2;
        for (m += (uint64_t)t0 * 2 * p2; m < hi; m += (uint64_t)step * 2 * p2)
            atomicOr(&s_acc[(m - lo - 1) >> 1], 0x80000000u);
    };
    // primes from P[1] (3) while p^2 < hi; the first nsmall by all threads
    for (uint32_t k = 1; k < np && k <= nsmall; k++) {
        const uint64_t p = P[k];
        if (p * p >= hi) break;
        uint32_t i0 = first_odd_multiple_idx(lo, hi, p, false);
        if (i0 == 0xFFFFFFFFu) continue;
        const uint32_t add = mitchell_log2_q16(p) + (1u << 24);
        for (uint32_t i = i0 + tid * (uint32_t)p; i < kMuSeg; i += kThreads * (uint32_t)p) {
            atomicMin(&s_lpf[i], (W)p);
            atomicAdd(&s_acc[i], add);
        }
        square_flags(p, tid, kThreads);
    }
    for (uint32_t k = nsmall + 1 + tid; k < np; k += kThreads) {
        const uint64_t p = P[k];
        if (p * p >= hi) break;
        uint32_t i0 = first_odd_multiple_idx(lo, hi, p, false);
        if (i0 == 0xFFFFFFFFu) continue;
        const uint32_t add = mitchell_log2_q16(p) + (1u << 24);
        for (uint32_t i = i0; i < kMuSeg; i += (uint32_t)p) {
            atomicMin(&s_lpf[i], (W)p);
            atomicAdd(&s_acc[i], add);
        }
        square_flags(p, 0, 1);
    }
    __syncthreads();
    for (uint32_t i = tid; i < kMuSeg; i += kThreads) {
        const uint64_t n = lo + 2 * i + 1;
        const uint64_t gi = (n - lo0 - 1) >> 1;
        if (n >= hi_all) break;
        int m;
        uint64_t l;
        if (n == 1) {
            m = 1;
            l = 0xFFFFFFFFull;
        } else {
            const uint32_t a = s_acc[i];
            l = (s_lpf[i] == (W)~(W)0) ? n : (uint64_t)s_lpf[i];
            if (a & 0x80000000u) m = 0;
            else {
                const bool cofactor = mitchell_log2_q16(n) > (a & 0xFFFFFFu) + kCofactorQ16;
                const uint32_t k = ((a >> 24) & 0x3Fu) + (cofactor ? 1u : 0u);
                m = (k & 1) ? -1 : 1;
            }
        }
        if (mu) mu[gi] = (int8_t)m;
        if (lpf32) lpf32[gi] = (uint32_t)l;
        if (lpf64) lpf64[gi] = l;
        if (packed) packed[gi] = (n == 1) ? 0x7FFFFFFF : (m == 0 ? 0 : m * (int32_t)l);
    }
}

// mu of the odd n in [lo, hi) (hi <= 2^32) into a caller buffer with a
// caller prime list, on a caller stream; launches only, allocates nothing.
cudaError_t launch_mu_only(cudaStream_t st, uint64_t lo, uint64_t hi, const uint32_t *P, uint32_t np,
                           int8_t *mu)
{
    const uint64_t seg = MuSeg<unsigned int>::N;
    const uint64_t nblk = (hi - lo + 2 * seg - 1) / (2 * seg);
    if (nblk == 0) return cudaSuccess;
    const uint32_t nsmall = np > 54 ? 53 : (np ? np - 1 : 0);
    k_mulpf<unsigned int><<<(unsigned)nblk, kThreads, 0, st>>>(lo, hi, P, np, nsmall, mu, nullptr, nullptr,
                                                                nullptr);
    return cudaGetLastError();
}

void mulpf_sieve(cpx_ctx *ctx, uint64_t lo, uint64_t hi, int8_t *mu, uint32_t *lpf32, uint64_t *lpf64,
                 int32_t *packed)
{
    if (lo & 1) fail(CPX_EINVAL, "mu/lpf: lo must be even");
    if (hi <= lo) return;
    ensure_primes(ctx, cpx_isqrt(hi) + 2);
    const Tables &tb = ctx->tab;
    const bool w32 = hi <= 0xFFFFFFFFull;
    const uint64_t seg = w32 ? MuSeg<unsigned int>::N : MuSeg<unsigned long long>::N;
    const uint64_t nblk = (hi - lo + 2 * seg - 1) / (2 * seg);
    if (nblk == 0) return;
    if (nblk > 0x7FFFFFFFull) fail(CPX_ERANGE, "mu/lpf range too large");
    // primes below 256 go through the all-threads loop
    uint32_t nsmall = 0;
    {
        static const uint32_t small_cnt = 53;  // primes < 256 after 2 ... 251 is the 54th prime
        nsmall = (uint32_t)std::min<uint64_t>(small_cnt, tb.prm_n ? tb.prm_n - 1 : 0);
    }
    if (w32) {
        k_mulpf<unsigned int><<<(unsigned)nblk, kThreads, 0, ctx->stream>>>(lo, hi, tb.P, (uint32_t)tb.prm_n, nsmall, mu,
                                                                         lpf32, lpf64, packed);
    } else {
        k_mulpf<unsigned long long><<<(unsigned)nblk, kThreads, 0, ctx->stream>>>(
            lo, hi, tb.P, (uint32_t)tb.prm_n, nsmall, mu, lpf32, lpf64, packed);
    }
    CPX_LAUNCH("k_mulpf");
    note_launch(ctx);
}

void ensure_mulpf(cpx_ctx *ctx, uint64_t ymax)
{
    Tables &tb = ctx->tab;
    if (tb.MU && tb.mu_n >= ymax) return;
    if (ymax >= 0x7FFFFFFFull) fail(CPX_ERANGE, "y beyond 2^31 is not supported by the packed mu/lpf table");
    uint64_t want = std::max<uint64_t>(ymax, tb.mu_n + tb.mu_n / 2);
    want = std::max<uint64_t>(want, 1 << 16);
    want = std::min<uint64_t>(want, 0x7FFFFFFEull);
    const uint64_t len = want / 2 + 1;  // odd n <= want -> index (n-1)/2
    if (tb.MU) {
        cudaFree(tb.MU);
        tb.MU = nullptr;
        tb.mu_n = 0;
    }
    CPX_CUDA(cudaMalloc(&tb.MU, len * 4));
    mulpf_sieve(ctx, 0, 2 * len, nullptr, nullptr, nullptr, tb.MU);
    tb.mu_n = 2 * len - 1;
    tb.version++;
}

// ------------------------------------------------------------- wheel table

__global__ void k_wheel_flags(uint64_t *f, uint64_t half, uint32_t c, const uint32_t *P)
{
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= half) return;
    const uint64_t n = 2 * i + 1;
    uint64_t ok = 1;
    for (uint32_t k = 1; k < c; k++)
        if (n % P[k] == 0) ok = 0;
    f[i] = ok;
}

__global__ void k_wheel_pack(const uint64_t *f, uint64_t cnt, uint32_t *W)
{
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < cnt) W[i] = (uint32_t)f[i];
}

void ensure_wheel(cpx_ctx *ctx, uint32_t c)
{
    Tables &tb = ctx->tab;
    if (c < 1 || c > 8) fail(CPX_EINVAL, "c must be in 1..8");
    if (tb.WH && tb.wh_c == c) return;
    ensure_primes(ctx, 64);
    static const uint64_t primorial[9] = {1, 2, 6, 30, 210, 2310, 30030, 510510, 9699690};
    static const uint64_t totient[9] = {1, 1, 2, 8, 48, 480, 5760, 92160, 1658880};
    const uint64_t W = primorial[c], half = W / 2;
    uint64_t *f = ctx->b_tmp.as<uint64_t>(half + 2);
    k_wheel_flags<<<(unsigned)((half + 1 + 255) / 256), 256, 0, ctx->stream>>>(f, half + 1, c, tb.P);
    CPX_LAUNCH("k_wheel_flags");
    note_launch(ctx);
    scan_u64(ctx, f, half + 1);
    if (tb.WH) cudaFree(tb.WH);
    tb.WH = nullptr;
    CPX_CUDA(cudaMalloc(&tb.WH, (half + 1) * 4));
    k_wheel_pack<<<(unsigned)((half + 1 + 255) / 256), 256, 0, ctx->stream>>>(f, half + 1, tb.WH);
    CPX_LAUNCH("k_wheel_pack");
    note_launch(ctx);
    CPX_CUDA(cudaStreamSynchronize(ctx->stream));
    tb.wh_c = c;
    tb.wh_mod = W;
    tb.wh_tot = totient[c];
}

}  // namespace cpx
