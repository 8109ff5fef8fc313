// sieve.cuh -- segmented prime sieve on the device for census requests.
//
// A request asks for the first `count` primes >= lo (< 2^32).  The reference
// sieves bounded intervals on the host (src/census/prime_sieve.cpp:8-22, width
// <= 2e6); here one CTA per request window [lo, lo + width) marks the odd
// composites in a shared-memory bitmap with the primes <= sqrt(hi) of the
// static small-prime table, then writes the primes in increasing order with a
// block-wide prefix sum.  The host sizes width from the prime number theorem
// and widens a window that came up short.
#pragma once
#include "common.cuh"

namespace cz {

constexpr int SIEVE_THREADS = 1024;
constexpr u32 SIEVE_MAX_WIDTH = 1u << 21;          // numbers per window (odd-only bitmap 128 KiB)

struct SieveReq {
    u32 lo;          // window start
    u32 width;       // window width (<= SIEVE_MAX_WIDTH), lo + width <= 2^32
    u32 count;       // primes wanted
    u32 out_off;     // first output slot
    u32 found;       // primes written (device)
    u32 pad[3];
};

__global__ void __launch_bounds__(SIEVE_THREADS, 1)
sieve_kernel(SieveReq *reqs, u32 nreq, const u32 *small_primes, u32 n_small, u32 *out) {
    extern __shared__ u32 bits[];                   // bit i: number lo0 + 2i is composite
    __shared__ u32 warp_sum[SIEVE_THREADS / 32];
    __shared__ u32 s_base;
    for (u32 rq = blockIdx.x; rq < nreq; rq += gridDim.x) {
        SieveReq R = reqs[rq];
        const u64 lo = R.lo, hi = lo + R.width;     // [lo, hi)
        const u64 lo0 = lo | 1ull;                  // first odd number >= lo
        const u32 nodd = hi > lo0 ? (u32)((hi - lo0 + 1ull) / 2ull) : 0u;
        const u32 nwords = (nodd + 31u) / 32u;
        for (u32 i = threadIdx.x; i < nwords; i += blockDim.x) bits[i] = 0u;
        __syncthreads();
        // odd primes q with q*q < hi (the table holds every prime below 2^20 + 8192 > 2^16):
        // the first 256 (many multiples each) are swept by the whole block, one
        // prime at a time; the rest (few multiples) take one thread each
        for (u32 k = 1; k < n_small && k < 257u; ++k) {
            const u64 q = small_primes[k];
            if (q * q >= hi) break;
            u64 first = q * q > lo0 ? q * q : ((lo0 + q - 1ull) / q) * q;
            if (!(first & 1ull)) first += q;        // odd multiples only
            for (u64 m = first + 2ull * q * threadIdx.x; m < hi; m += 2ull * q * blockDim.x) {
                const u32 i = (u32)((m - lo0) >> 1);
                atomicOr(&bits[i >> 5], 1u << (i & 31u));
            }
        }
        for (u32 k = 257u + threadIdx.x; k < n_small; k += blockDim.x) {
            const u64 q = small_primes[k];
            if (q * q >= hi) break;
            u64 first = q * q > lo0 ? q * q : ((lo0 + q - 1ull) / q) * q;
            if (!(first & 1ull)) first += q;
            for (u64 m = first; m < hi; m += 2ull * q) {
                const u32 i = (u32)((m - lo0) >> 1);
                atomicOr(&bits[i >> 5], 1u << (i & 31u));
            }
        }
        __syncthreads();
        // ordered compaction: thread t owns odd numbers [t*per, (t+1)*per)
        const u32 per = (nodd + blockDim.x - 1) / blockDim.x;
        const u32 a = min(nodd, threadIdx.x * per), b = min(nodd, a + per);
        u32 cnt = 0;
        for (u32 i = a; i < b; ++i) {
            const u64 v = lo0 + 2ull * i;
            if (v >= 3 && !((bits[i >> 5] >> (i & 31u)) & 1u)) ++cnt;
        }
        const bool two = (lo <= 2 && hi > 2);       // the only even prime
        // block exclusive scan of cnt
        const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
        u32 incl = cnt;
        for (int o = 1; o < 32; o <<= 1) {
            const u32 y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
            if (lane >= o) incl += y;
        }
        if (lane == 31) warp_sum[w] = incl;
        __syncthreads();
        if (threadIdx.x == 0) {
            u32 run = two ? 1u : 0u;
            for (int i = 0; i < (int)(blockDim.x / 32); ++i) { const u32 t = warp_sum[i]; warp_sum[i] = run; run += t; }
            s_base = run;                           // total primes in the window
        }
        __syncthreads();
        u32 pos = warp_sum[w] + incl - cnt;
        if (two && threadIdx.x == 0 && R.count > 0) out[R.out_off] = 2u;
        for (u32 i = a; i < b; ++i) {
            const u64 v = lo0 + 2ull * i;
            if (v >= 3 && !((bits[i >> 5] >> (i & 31u)) & 1u)) {
                if (pos < R.count) out[R.out_off + pos] = (u32)v;
                ++pos;
            }
        }
        if (threadIdx.x == 0) reqs[rq].found = s_base < R.count ? s_base : R.count;
        __syncthreads();
    }
}

}  // namespace cz
