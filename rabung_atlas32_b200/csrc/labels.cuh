// labels.cuh -- discrete-log labels of m-th roots of unity.
//
// For a prime p and m = lcm of the admissible orders r (m | p-1, m <= 2520),
// x^((p-1)/m) is an m-th root of unity z^j for a fixed z of exact order m;
// j is the label of x and colour_r(x) = j mod r (the reference's
// character_root + sorted root table, src/census/engine32/src/frozen_entry.cu:18-24,
// 158-167).  Here the m roots live in a shared-memory open-addressing hash
// keyed by their Montgomery value, so a lookup is ~1-2 probes instead of a
// 12-step binary search.
#pragma once
#include "common.cuh"

namespace CZ_NS {

// smallest power-of-two slot count >= 3m/2 (m <= 2520 -> <= 4096 slots)
CZ_HD u32 hash_slots(u32 m) {
    u32 s = 8;
    while (2 * s < 3 * m) s <<= 1;
    return s;
}

CZ_HD u32 hash_slot(u32 key, u32 bits) { return (key * 0x9E3779B1u) >> (32 - bits); }
CZ_HD u32 hash_slot(u64 key, u32 bits) { return hash_slot((u32)key ^ (u32)(key >> 32) * 0x85EBCA6Bu, bits); }

// element of exact order m: z = a^((p-1)/m) with z^(m/q) != 1 for each prime
// q | m (the reference's character_root; only m is factored).
CZ_HD pw_t find_root_of_order(const Mont &M, pw_t p, u32 m, pw_t e) {
    if (m == 1) return M.one;
    for (u32 a = 2; a < p && a < 100000u; ++a) {
        pw_t z = mpow(to_mont((pw_t)a, M), e, M);
        bool ok = true;
        const u32 qs[4] = {2, 3, 5, 7};
        for (int i = 0; i < 4; ++i)
            if (m % qs[i] == 0 && mpow(z, m / qs[i], M) == M.one) { ok = false; break; }
        if (ok) return z;
    }
    return 0;
}

// Block-cooperative build of the root hash for one prime in shared memory.
// keys[] must hold hash_slots(m) prime-sized words, labels[] as many u16.
// All threads of the block call this; ends with __syncthreads().
__device__ __forceinline__ pw_t cas_key(pw_t *a, pw_t expect, pw_t v) {
#if CZ_WIDE
    return (pw_t)atomicCAS(reinterpret_cast<unsigned long long *>(a), (unsigned long long)expect,
                           (unsigned long long)v);
#else
    return atomicCAS(a, expect, v);
#endif
}

__device__ inline void build_root_hash(pw_t *keys, unsigned short *labels, u32 slots,
                                       const Mont &M, pw_t z, u32 m) {
    for (u32 i = threadIdx.x; i < slots; i += blockDim.x) keys[i] = 0u;
    __syncthreads();
    u32 bits = 31 - __clz(slots);
    for (u32 j = threadIdx.x; j < m; j += blockDim.x) {
        pw_t v = mpow(z, (pw_t)j, M);     // Montgomery z^j (never 0: a unit)
        u32 h = hash_slot(v, bits);
        for (u32 probe = 0; probe < slots; ++probe) {
            pw_t old = cas_key(&keys[h], (pw_t)0, v);
            if (old == 0u) { labels[h] = (unsigned short)j; break; }
            h = (h + 1) & (slots - 1);
        }
    }
    __syncthreads();
}

// label of a Montgomery m-th root of unity; 0xFFFF on a miss
__device__ __forceinline__ u32 lookup_label(const pw_t *keys, const unsigned short *labels,
                                            u32 slots, pw_t v) {
    u32 bits = 31 - __clz(slots);
    u32 h = hash_slot(v, bits);
    for (u32 probe = 0; probe < slots; ++probe) {
        pw_t k = keys[h];
        if (k == v) return labels[h];
        if (k == 0u) return 0xFFFFu;
        h = (h + 1) & (slots - 1);
    }
    return 0xFFFFu;
}

// exact floor(x / r) for x < 2^16, r <= 9: multiply by ceil(2^32 / r)
CZ_HD u32 magic_of(u32 r) { return (u32)(((u64(1) << 32) + r - 1) / r); }
CZ_HD u32 mod_small(u32 x, u32 r, u32 magic) { return x - r * umulhi(x, magic); }

}  // namespace CZ_NS
