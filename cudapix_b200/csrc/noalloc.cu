// noalloc.cu -- cpx_mutest_noalloc: the Mertens self-test (cpx_mutest) for
// callers that cannot allocate device memory.
//
// Some callers cannot call cudaMalloc: their device memory is owned by another
// allocator (a framework's caching allocator or a fixed pool that has reserved
// the GPU), or they run on a latency-critical path where cudaMalloc/cudaFree
// would synchronise the device.  cpx_mutest allocates its scratch (the mu array
// of the odd numbers below top, and the reduction accumulator) in the context's
// grow-only buffers; this variant keeps that scratch in one file-scope static
// device array instead, so a call allocates nothing.
//
// The static array is 16 MiB + 16 KiB, held on every GPU that loads the
// library until the process exits.  Its layout:
//   [0, 8)                  the 64-bit reduction accumulator (cleared by every call)
//   [256, 256 + 4112)       the 1028 primes below 8192 (rewritten by every call)
//   [16384, 16384 + 2^24)   mu(n) of the odd n below top, one byte each
// so top may be at most 2^25 = 33554432.  Every call shares the array and it
// keeps the last call's contents; calls that overlap on the GPU (on different
// streams, contexts or threads) race on it.
//
// In host code the name g_noalloc_scratch is only a host-side stand-in for the
// device array: a kernel given it would fault or, where the GPU can reach host
// memory, silently use the wrong memory.  So the first call on each context,
// with the context's device current, asks the runtime for the array's device
// address (cudaGetSymbolAddress), keeps it in the context and passes it to the
// kernels.  Make that first call on a context before any stream capture.
// cudaDeviceReset destroys every context's stream and tables along with the
// array: destroy the contexts before a reset and create new ones after it (a
// new context looks the address up again).  The caller's current device is
// left as it was.
#include <algorithm>

#include "misc.h"

namespace cpx {

cudaError_t launch_mu_only(cudaStream_t st, uint64_t lo, uint64_t hi, const uint32_t *P, uint32_t np,
                           int8_t *mu);
cudaError_t launch_mu_sums(cudaStream_t st, const int8_t *mu, uint64_t n_odd, uint64_t v1, uint64_t v2,
                           unsigned long long *acc, unsigned grid);

namespace {

constexpr size_t kAccOff = 0;
constexpr size_t kPrimeOff = 256;
constexpr uint32_t kNumPrimes = 1028;  // primes below 8192, 2 included
constexpr size_t kMuOff = 16384;
constexpr uint64_t kMaxOdd = 1ull << 24;  // mu entries
constexpr uint64_t kMaxTop = 2 * kMaxOdd;  // 33554432
constexpr size_t kScratchBytes = kMuOff + kMaxOdd;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

// primes below 8192, ascending, by trial division in one CTA of 1024 threads
// (4 odd candidates per thread, block scan for the output positions)
__global__ void __launch_bounds__(1024) k_noalloc_primes(uint32_t *out)
{
    __shared__ uint32_t wsum[32];
    const uint32_t t = threadIdx.x, lane = t & 31, w = t >> 5;
    uint32_t f[4], c = 0;
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const uint32_t n = 2 * (4 * t + k) + 1;  // odd n < 8192
        bool pr = n >= 3;
        for (uint32_t d = 3; pr && d * d <= n; d += 2)
            if (n % d == 0) pr = false;
        f[k] = pr;
        c += pr;
    }
    uint32_t inc = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t v = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= (uint32_t)o) inc += v;
    }
    if (lane == 31) wsum[w] = inc;
    __syncthreads();
    uint32_t pos = 1 + inc - c;  // out[0] = 2
    for (uint32_t i = 0; i < w; i++) pos += wsum[i];
#pragma unroll
    for (int k = 0; k < 4; k++)
        if (f[k]) out[pos++] = 2 * (4 * t + k) + 1;
    if (t == 0) out[0] = 2;
}

}  // namespace
}  // namespace cpx

extern "C" int cpx_mutest_noalloc(cpx_ctx *ctx, uint64_t top, int64_t *out)
{
    using namespace cpx;
    if (!ctx || !out) return CPX_EINVAL;
    std::lock_guard<std::recursive_mutex> lk(ctx->mu);
    auto err = [&](int code, const std::string &m) {
        ctx->last_error = m;
        return code;
    };
    if (top > kMaxTop)
        return err(CPX_ERANGE, "cpx_mutest_noalloc: top must be <= 33554432 (the 16 MiB static scratch)");
    DeviceGuard dg(ctx->device);
    if (dg.err != cudaSuccess)
        return err(CPX_ECUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(dg.err));
    if (!ctx->noalloc_scratch) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p)
            return err(CPX_ECUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        ctx->noalloc_scratch = p;
    }
    unsigned char *base = static_cast<unsigned char *>(ctx->noalloc_scratch);
    *out = 0;
    if (top <= 1) {
        ctx->last_error.clear();
        return CPX_OK;
    }
    unsigned long long *acc = reinterpret_cast<unsigned long long *>(base + kAccOff);
    uint32_t *P = reinterpret_cast<uint32_t *>(base + kPrimeOff);
    int8_t *mu = reinterpret_cast<int8_t *>(base + kMuOff);
    const uint64_t v1 = top - 1, v2 = (top - 1) / 2;
    const uint64_t n_odd = (v1 + 1) / 2;  // odd n <= top - 1
    cudaStream_t st = ctx->stream;
    cudaError_t e = cudaMemsetAsync(acc, 0, 8, st);
    if (e == cudaSuccess) {
        k_noalloc_primes<<<1, 1024, 0, st>>>(P);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = launch_mu_only(st, 0, 2 * n_odd, P, kNumPrimes, mu);
    if (e == cudaSuccess) {
        const unsigned grid = (unsigned)std::max<uint64_t>(
            1, std::min<uint64_t>((n_odd + 255) / 256, (uint64_t)ctx->sm_count * 8));
        e = launch_mu_sums(st, mu, n_odd, v1, v2, acc, grid);
    }
    unsigned long long h = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h, acc, 8, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return err(CPX_ECUDA, std::string("cpx_mutest_noalloc: ") + cudaGetErrorString(e));
    ctx->launches += 3;
    *out = (int64_t)h;
    ctx->last_error.clear();
    return CPX_OK;
}
