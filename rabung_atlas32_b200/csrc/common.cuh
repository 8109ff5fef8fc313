// common.cuh -- shared types and Montgomery arithmetic for the B200 (sm_100a)
// census kernels.
//
// The kernels are compiled for one prime word width per translation unit:
//   CZ_WIDE 0 (default): p < 2^32, pw_t = uint32_t, namespace cz;
//   CZ_WIDE 1:           p < 2^33, pw_t = uint64_t, namespace cz64.
// Only quantities of the size of p (p itself, residues, exponents, roots)
// take pw_t; table numerators, run lengths, labels and canonical witnesses
// (at most (p-1)/2 < 2^32) stay 32-bit in both.
//
// Montgomery product for an odd modulus p, R = 2^32 (32-bit words; the
// reference's kit::mont, src/census/engine32/src/mont32.hpp:9-10) or R = 2^64
// (64-bit words, p < 2^33; the reference's wide33::mont,
// src/census/math33.hpp:13-28): a*b*R^-1 mod p, formed from the two high
// products and the carry of the low half (lo(t) + lo(m p) == 0 mod R, so the
// carry is lo(t) != 0).  Four integer multiplies (mul.lo, mul.hi, mul.lo,
// mul.hi) of the word width per product.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

typedef uint32_t u32;
typedef uint64_t u64;
typedef int64_t i64;
typedef int32_t i32;

#define CZ_HD __host__ __device__ __forceinline__

#ifndef CZ_WIDE
#define CZ_WIDE 0
#endif
#if CZ_WIDE
#define CZ_NS cz64
#else
#define CZ_NS cz
#endif

namespace CZ_NS {

#if CZ_WIDE
typedef u64 pw_t;                   // prime-sized word: p < 2^33
#else
typedef u32 pw_t;                   // prime-sized word: p < 2^32
#endif

struct Mont {
    pw_t p;      // odd modulus
    pw_t ninv;   // -p^-1 mod R
    pw_t one;    // R mod p
    pw_t r2;     // R^2 mod p
};

// -p^-1 mod R by Newton steps (p*p == 1 mod 8; each step doubles the bits: 3 -> 96)
CZ_HD pw_t neg_inverse(pw_t p) {
    pw_t x = p;
    for (int i = 0; i < 5; ++i) x *= (pw_t)2 - p * x;
    return (pw_t)0 - x;
}

CZ_HD Mont make_mont(pw_t p) {
    Mont m;
    m.p = p;
    m.ninv = neg_inverse(p);
#if CZ_WIDE
    u64 R = (0ull - p) % p;                     // 2^64 mod p
    u64 r2 = R;
    for (int i = 0; i < 64; ++i) { r2 <<= 1; if (r2 >= p) r2 -= p; }   // 2^128 mod p (p < 2^33: no overflow)
    m.one = R;
    m.r2 = r2;
#else
    u64 R = (u64(1) << 32) % p;
    m.one = (u32)R;
    m.r2 = (u32)((R * R) % p);
#endif
    return m;
}

#ifdef __CUDA_ARCH__
CZ_HD u32 umulhi(u32 a, u32 b) { return __umulhi(a, b); }
CZ_HD u64 umulhi(u64 a, u64 b) { return __umul64hi(a, b); }
#else
CZ_HD u32 umulhi(u32 a, u32 b) { return (u32)(((u64)a * b) >> 32); }
CZ_HD u64 umulhi(u64 a, u64 b) { return (u64)(((unsigned __int128)a * b) >> 64); }
#endif

#if CZ_WIDE
// a*b*2^-64 mod p for a, b < p < 2^33: hi + mhi + carry < 2p, no overflow
CZ_HD u64 mmul(u64 a, u64 b, u64 p, u64 ninv) {
    const u64 tlo = a * b;
    const u64 thi = umulhi(a, b);
    const u64 m = tlo * ninv;
    const u64 mhi = umulhi(m, p);
    const u64 u = thi + mhi + (tlo != 0ull);
    return u >= p ? u - p : u;
}
#else
// a*b*2^-32 mod p for a, b < p
CZ_HD u32 mmul(u32 a, u32 b, u32 p, u32 ninv) {
    u32 tlo = a * b;
    u32 thi = umulhi(a, b);
    u32 m = tlo * ninv;
    u32 mhi = umulhi(m, p);
    u64 u = (u64)thi + mhi + (tlo != 0u);
    return u >= p ? (u32)(u - p) : (u32)u;
}
#endif

CZ_HD pw_t mmul(pw_t a, pw_t b, const Mont &M) { return mmul(a, b, M.p, M.ninv); }
CZ_HD pw_t to_mont(pw_t x, const Mont &M) { return mmul(x, M.r2, M); }
CZ_HD pw_t from_mont(pw_t x, const Mont &M) { return mmul(x, (pw_t)1, M); }

CZ_HD int top_bit(u32 e) {
#ifdef __CUDA_ARCH__
    return 31 - __clz(e);
#else
    return 31 - __builtin_clz(e);
#endif
}
CZ_HD int top_bit(u64 e) {
#ifdef __CUDA_ARCH__
    return 63 - __clzll((long long)e);
#else
    return 63 - __builtin_clzll(e);
#endif
}

// two left-to-right binary powers with one exponent, interleaved: two
// independent multiply chains per thread
CZ_HD void mpow2(pw_t a, pw_t b, pw_t e, const Mont &M, pw_t &ra, pw_t &rb) {
    if (e == 0) { ra = rb = M.one; return; }
    const int top = top_bit(e);
    pw_t va = a, vb = b;
    for (int i = top - 1; i >= 0; --i) {
        va = mmul(va, va, M);
        vb = mmul(vb, vb, M);
        if ((e >> i) & 1u) { va = mmul(va, a, M); vb = mmul(vb, b, M); }
    }
    ra = va;
    rb = vb;
}

// left-to-right binary power of a Montgomery residue
CZ_HD pw_t mpow(pw_t a, pw_t e, const Mont &M) {
    if (e == 0) return M.one;
    const int top = top_bit(e);
    pw_t v = a;
    for (int i = top - 1; i >= 0; --i) {
        v = mmul(v, v, M);
        if ((e >> i) & 1u) v = mmul(v, a, M);
    }
    return v;
}

CZ_HD u32 gcd32(u32 a, u32 b) {
    while (b) { u32 t = a % b; a = b; b = t; }
    return a;
}

CZ_HD u32 lcm_of_mask(u32 mask) {
    u32 m = 1;
    for (u32 r = 2; r <= 9; ++r)
        if (mask & (1u << (r - 2))) m = m / gcd32(m, r) * r;
    return m;
}

CZ_HD u32 mask_of(pw_t p) {
    u32 m = 0;
    for (u32 r = 2; r <= 9; ++r)
        if ((p - 1u) % r == 0u) m |= 1u << (r - 2);
    return m;
}

CZ_HD u32 planes_for(u32 r) { return r <= 2 ? 1u : r <= 4 ? 2u : r <= 8 ? 3u : 4u; }
CZ_HD u32 planes_stored(u32 r) { return r <= 2 ? 1u : r <= 4 ? 2u : 4u; }

// packed reduction key: longer run first, then least canonical witness
CZ_HD u64 pack_key(u32 len, u32 witness) { return ((u64)len << 32) | (u64)(0xFFFFFFFFu - witness); }
CZ_HD u32 key_len(u64 k) { return (u32)(k >> 32); }
CZ_HD u32 key_witness(u64 k) { return 0xFFFFFFFFu - (u32)k; }

// ---- per-prime and per-profile descriptors shared by host and device ----

struct PrimeDesc {
    pw_t p;
    u32 mask;
    u32 m;           // lcm of admissible r
    pw_t e;          // (p-1)/m
    pw_t ninv, one, r2;
    pw_t z;          // Montgomery form of an element of exact order m
    u32 sigma;       // label of -1 modulo m (0 or m/2)
    u32 B;           // signed table radius (sparse)
    u32 K0;          // base view: index of n is n + 32*K0 + 31
    u32 nwords;      // base view words per plane
    u32 K2;          // odd view: index of n = 2i+1 is i + 32*K2
    u32 nwords2;     // odd view words per plane
    u32 first_prof;  // index of this prime's first profile
    u32 nprof;
    u32 route;       // 1 dense, 2 sparse
    u32 status;      // error bits set by kernels
};

struct ProfDesc {
    u32 prime;       // index into PrimeDesc
    u32 r;
    u32 np;          // bit planes
    u32 npp;         // planes as stored (np padded to 1, 2 or 4), interleaved
    u32 Q;           // cover window cap
    u32 D;           // cover denominators 1..D
    u32 out_slot;    // index in the caller's output array
    u64 plane_off;   // word offset of plane 0 in the plane pool
    pw_t omega[9];   // Montgomery omega^j, omega = z^(m/r), j < r
    u32 local;       // index of the prime within its route's list
    u32 qspec;       // speculative threshold (0: none); exact if the best run reaches it
    u32 tpref;       // preferred anchor stages (sparse filter)
    u32 req;         // serving: the request slot this profile belongs to
};

// device-written per-profile results
struct ProfState {
    unsigned long long best;  // packed key of the best completed run
    unsigned long long claim; // sparse filter: next work item, current epoch and its threshold
    u32 seed;                 // longest monochromatic stretch seen in [1, B]
    u32 firstnz;              // least n >= 1 with colour != 0 (prefix + 1)
    u32 status;
    u32 active;               // serving: CTAs working on the profile now
    u32 done;                 // serving: 1 once its record is final
    u32 staged16;             // sparse filter: plane bytes staged into shared memory, / 16
    unsigned long long words;       // filter words visited
    unsigned long long completions; // exact completions run
    unsigned long long tests;       // plane-window comparisons (stage x plane) executed
};

enum : u32 {
    ST_OK = 0,
    ST_ROOT = 1u << 0,       // no element of exact order m found
    ST_LABEL = 1u << 1,      // a power missed the root table
    ST_SEED = 1u << 2,       // seed too short for a certified threshold
    ST_PREFIX = 1u << 3,     // prefix ran past the table
    ST_VERIFY = 1u << 4,     // direct-power certification failed
    ST_A4 = 1u << 5,         // point count not certified
    ST_QUEUE = 1u << 6,      // candidate buffer overflow
    ST_COVER = 1u << 7,      // cover certificate out of domain
    ST_SPEC = 1u << 8,       // best run below the speculative threshold: re-run without it
};

}  // namespace CZ_NS
