// census_wide.cu -- the census for primes 2^32 <= p < 2^33 (and any smaller
// odd prime), the reference's 33-bit domain (src/census/math33.hpp:13-37,
// reproducibility/gpu_method/source/engine33): the same kernels and host
// plan as census.cu, compiled for 64-bit prime words (Montgomery products
// with R = 2^64; table numerators, planes, run lengths and canonical
// witnesses stay 32-bit).  Records are cz_profile64 (p as 64 bits).
#define CZ_WIDE 1
#include "core.cuh"

extern "C" {

int cz_open64(const cz_config *cfg, cz_handle64 **out) { return handle_open(cfg, out); }

void cz_close64(cz_handle64 *h) { handle_close(h); }

const char *cz_last_error64(const cz_handle64 *h) { return h ? h->err.c_str() : "null handle"; }

uint32_t cz_count_profiles64(const uint64_t *primes, uint32_t n) {
    for (uint32_t i = 0; i < n; ++i)
        if (primes[i] >= PW_LIMIT) return 0u;
    return count_profiles(primes, n);
}

int cz_census64(cz_handle64 *h, const uint64_t *primes, uint32_t n, uint32_t flags, cz_profile64 *out,
                uint32_t out_cap, uint32_t *a4_out, cz_stats *stats) {
    if (!h) return CZ_EINVAL;
    for (uint32_t i = 0; i < n && primes; ++i)
        if (primes[i] >= PW_LIMIT) { h->err = "prime at or above 2^33: " + std::to_string(primes[i]); return CZ_EINVAL; }
    return census_entry(h, primes, n, flags, out, out_cap, a4_out, stats);
}

}  // extern "C"
