// misc.h -- helpers behind the smaller drop-in entry points.
#pragma once
#include "cpx_internal.h"

namespace cpx {

int64_t mutest(cpx_ctx *ctx, uint64_t top);
uint64_t count_primes(cpx_ctx *ctx, uint64_t lo, uint64_t hi);
void pitable_window(cpx_ctx *ctx, uint64_t base, uint64_t range, uint32_t *d_out, uint64_t *pi_base);
uint32_t *pitable_dense(cpx_ctx *ctx, uint64_t hi);
uint64_t primes_list(cpx_ctx *ctx, uint64_t lo, uint64_t hi, uint64_t **d_out);
uint64_t extract_window(cpx_ctx *ctx, const cpx_pient *T, uint64_t w0, uint64_t lo, uint64_t hi, uint64_t *out);
uint64_t phi_count(cpx_ctx *ctx, uint64_t x, uint32_t a);
uint32_t *phi_range(cpx_ctx *ctx, uint32_t num, uint32_t a);
void phi_bits(cpx_ctx *ctx, uint64_t nwords, uint32_t a, uint64_t *words);
void counts_from_bits(cpx_ctx *ctx, const uint64_t *words, uint64_t nwords, uint64_t nbits, int inclusive,
                      uint32_t *out);
void phisieve_cross(cpx_ctx *ctx, uint64_t *words, uint64_t nbits, uint64_t p);

}  // namespace cpx
