// finalize.cuh -- per-prime setup and per-profile finalisation kernels.
//
// setup_kernel: Montgomery constants, deterministic primality (the worker's
// "worker primality" check, src/census/worker32.cu:18), a root z of exact order
// m = lcm(r) (frozen_entry.cu:18-24), the label of -1, and the r-th roots of
// unity omega^j = z^(j m / r) used by direct colour evaluation.
//
// finalize_kernel: M and witness from the packed key, L by direct powers from
// x = 2 (the reference's prefix verification, worker32.cu:38), optional direct
// certification of the witness run (certify_witness, B2/src/advance.cpp:7-13),
// K by the scientific contract (docs/METHODS.md:11-18) and the output record.
#pragma once
#include "labels.cuh"

namespace CZ_NS {

// deterministic Miller-Rabin with bases 2, 3, 5, 7, 11: no strong pseudoprime
// to all five below 2.15e12, so exact for every n < 2^33 (host and device:
// the serving runtime refuses a caller's non-prime before any device work)
__host__ __device__ inline bool is_prime_word(pw_t n) {
    if (n < 2u) return false;
    const u32 bases[5] = {2, 3, 5, 7, 11};
    for (int i = 0; i < 5; ++i) {
        if (n == bases[i]) return true;
        if (n % bases[i] == 0u) return false;
    }
    const Mont M = make_mont(n);
    pw_t d = n - 1u;
    u32 s = 0;
    while (!(d & 1u)) { d >>= 1; ++s; }
    const pw_t mone = n - M.one;          // Montgomery form of -1
    for (int i = 0; i < 5; ++i) {
        pw_t x = mpow(to_mont((pw_t)bases[i], M), d, M);
        if (x == M.one || x == mone) continue;
        bool pass = false;
        for (u32 j = 1; j < s; ++j) {
            x = mmul(x, x, M);
            if (x == mone) { pass = true; break; }
            if (x == M.one) return false;
        }
        if (!pass) return false;
    }
    return true;
}

__global__ void setup_kernel(PrimeDesc *primes, ProfDesc *profs, ProfState *state, u32 n) {
    const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    PrimeDesc P = primes[i];
    u32 status = 0;
    if (!is_prime_word(P.p)) status |= ST_ROOT;
    if (P.p > 2u) {
        const Mont M = make_mont(P.p);
        P.ninv = M.ninv; P.one = M.one; P.r2 = M.r2;
        if (P.m > 1u) {
            P.z = find_root_of_order(M, P.p, P.m, P.e);
            if (!P.z) status |= ST_ROOT;
        } else {
            P.z = M.one;
        }
        P.sigma = (P.e & 1u) ? P.m / 2u : 0u;
        for (u32 s = 0; s < P.nprof; ++s) {
            ProfDesc &D = profs[P.first_prof + s];
            const pw_t w = mpow(P.z, (pw_t)(P.m / D.r), M);
            pw_t v = M.one;
            for (u32 j = 0; j < 9; ++j) {
                D.omega[j] = j < D.r ? v : 0u;
                v = mmul(v, w, M);
            }
            ProfState &S = state[P.first_prof + s];
            S.best = 0; S.claim = 0; S.seed = 0; S.firstnz = 0xFFFFFFFFu;
            S.status = 0; S.active = 0; S.done = 0; S.staged16 = 0; S.words = 0; S.completions = 0; S.tests = 0;
        }
    }
    P.status = status;
    primes[i] = P;
}

// mirrors cz_profile (32-bit words) or cz_profile64 (64-bit words) in
// include/rabung_census.h; the canonical witness is at most (p-1)/2 < 2^32
struct OutRecord {
    pw_t p;
    u32 r, M, L, witness, status;
#if CZ_WIDE
    u32 reserved;
#endif
    unsigned long long K;
};

__device__ __forceinline__ u32 colour_pow(pw_t x, const Mont &M, pw_t ex, const pw_t *om, u32 r) {
    const pw_t y = mpow(to_mont(x, M), ex, M);
    for (u32 j = 0; j < r; ++j)
        if (om[j] == y) return j;
    return 0xFFFFFFFFu;
}

// the record of profile g: M and witness from its best key, L (dense: from the
// scan; sparse: by direct powers), optional certification, K.  The key and
// status words are read through volatile loads: in the serving runtime the
// last CTA leaving a profile finalises it while other CTAs' atomics on them
// have just completed.
__device__ inline void finalize_one(const PrimeDesc *primes, const ProfDesc *profs, const ProfState *state,
                                    const u32 *dense_prefix, u32 g, u32 verify, OutRecord *out) {
    const ProfDesc D = profs[g];
    const PrimeDesc P = primes[D.prime];
    const unsigned long long best = *(const volatile unsigned long long *)&state[g].best;
    const u32 sstatus = *(const volatile u32 *)&state[g].status;
    const Mont M{P.p, P.ninv, P.one, P.r2};
    const pw_t p = P.p, ex = (p - 1u) / D.r;
    const u32 r = D.r;
    u32 status = P.status | sstatus;
    const u32 Mlen = key_len(best), w = key_witness(best);
    if (best == 0ull && !(D.qspec && P.route == 2u)) status |= ST_VERIFY;
    if (P.route == 2u && D.qspec && Mlen < D.qspec) status |= ST_SPEC;
    u32 L;
    if (P.route == 1u) {
        L = dense_prefix[g];
    } else {
        L = 1;                                   // colour(1) = 0
        while (L + 1u < p && colour_pow((pw_t)L + 1u, M, ex, D.omega, r) == 0u) {
            ++L;
            if (L > 4096u) { status |= ST_PREFIX; break; }
        }
    }
    if (verify && !(status & (ST_ROOT | ST_LABEL)) && Mlen > 0u && Mlen <= 4096u) {
        // the run [w, w+M-1] (or its mirror) is monochromatic and maximal
        const pw_t wx = w;
        const u32 c0 = colour_pow(wx, M, ex, D.omega, r);
        bool ok = c0 != 0xFFFFFFFFu && (u64)w + Mlen - 1u <= (u64)p - 1u;
        for (u32 k = 1; ok && k < Mlen; ++k) ok = colour_pow(wx + k, M, ex, D.omega, r) == c0;
        if (ok && w > 1u) ok = colour_pow(wx - 1u, M, ex, D.omega, r) != c0;
        if (ok && (u64)w + Mlen <= (u64)p - 1u) ok = colour_pow(wx + Mlen, M, ex, D.omega, r) != c0;
        u32 pl = 1;                              // prefix re-check from the scan result
        if (ok && P.route == 1u) {
            while (pl + 1u < p && pl <= L && colour_pow((pw_t)pl + 1u, M, ex, D.omega, r) == 0u) ++pl;
            ok = pl == L;
        }
        if (!ok) status |= ST_VERIFY;
    }
    OutRecord o;
    o.p = p; o.r = r; o.M = Mlen; o.L = L; o.witness = w; o.status = status;
#if CZ_WIDE
    o.reserved = 0u;
#endif
    const u64 b = ((((u64)p - 1u) / 2u) % r == 0u) ? 2ull * L + 2ull : (u64)L + 2ull;
    o.K = (u64)Mlen + 1ull > b ? (u64)Mlen + 1ull : b;
    out[D.out_slot] = o;
}

__global__ void finalize_kernel(const PrimeDesc *primes, const ProfDesc *profs, const ProfState *state,
                                const u32 *dense_prefix, u32 nprof, u32 verify, OutRecord *out) {
    const u32 g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g < nprof) finalize_one(primes, profs, state, dense_prefix, g, verify, out);
}

}  // namespace CZ_NS
