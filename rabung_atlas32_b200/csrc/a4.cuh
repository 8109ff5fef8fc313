// a4.cuh -- quadratic A4 counts on the device.
//
// A4(p) = #{x in [1, p-4] : x, x+1, x+2, x+3 share one quadratic character}.
// For p < 1000 it is counted directly (src/census/moment_worker.cpp:11-18).
// Otherwise A4 = (N - 12 - b)/8 with N = #E(F_p), E: y^2 = x(x-1)(x-9) and
// b = 4chi(2) + 2chi(6) + 2chi(3) + 2chi(-1) + 2chi(-2)
// (src/census/theorie/elliptic4_mestre.cpp:64-67).  N is found by the published
// baby-step/giant-step search over the Hasse interval [p+1-R, p+1+R],
// R = isqrt(4p), with an lcm-of-point-orders uniqueness test alternating E and
// its quadratic twist (#E + #E' = 2p+2) (elliptic4_mestre.cpp:42-62).  This
// build also folds in 4 | N (the three 2-torsion points (0,0), (s,0), (9s,0)
// are rational on both curves for p > 3).  N is unique, so the choice of
// points does not change the result.
//
// B200 design: one warp per prime.  Baby steps j*P (j < m) are spread over
// the 32 lanes and hashed by x-coordinate in shared memory; giant steps
// (L + i m) P are taken 32 at a time, one per lane; the point order is
// found lane-parallel per prime factor of the matched multiple; all curve
// arithmetic is affine in Montgomery form (the prime's word width) with
// Fermat inverses.
#pragma once
#include "labels.cuh"

namespace CZ_NS {

constexpr int A4_WARPS = CZ_WIDE ? 2 : 4;   // primes per CTA (shared hash tables: 18 / 10 KB per warp)
constexpr u32 A4_SLOTS = 1024;      // hash slots per warp (m <= 513 below 2^32, <= 610 below 2^33)
constexpr pw_t NO_ROOT = ~(pw_t)0;
constexpr u32 A4_MAX_ATTEMPTS = 64;

struct ECPt { pw_t x, y; bool inf; };

struct Curve {
    Mont M;
    pw_t s10, s9sq, s20, three;  // Montgomery 10s, 9s^2, 20s, 3
};

__device__ __forceinline__ pw_t addm(pw_t a, pw_t b, pw_t p) { u64 c = (u64)a + b; return c >= p ? (pw_t)(c - p) : (pw_t)c; }
__device__ __forceinline__ pw_t subm(pw_t a, pw_t b, pw_t p) { return a >= b ? a - b : (pw_t)((u64)a + p - b); }
__device__ __forceinline__ pw_t invm(pw_t a, const Mont &M) { return mpow(a, M.p - 2u, M); }

__device__ ECPt ec_add(const ECPt &A, const ECPt &B, const Curve &E) {
    if (A.inf) return B;
    if (B.inf) return A;
    const Mont &M = E.M;
    const pw_t p = M.p;
    pw_t lam;
    if (A.x == B.x) {
        if (addm(A.y, B.y, p) == 0u) return ECPt{0, 0, true};
        // tangent: (3x^2 - 20 s x + 9 s^2) / 2y
        const pw_t x2 = mmul(A.x, A.x, M);
        pw_t num = mmul(E.three, x2, M);
        num = subm(num, mmul(E.s20, A.x, M), p);
        num = addm(num, E.s9sq, p);
        lam = mmul(num, invm(addm(A.y, A.y, p), M), M);
    } else {
        lam = mmul(subm(B.y, A.y, p), invm(subm(B.x, A.x, p), M), M);
    }
    pw_t x3 = addm(mmul(lam, lam, M), E.s10, p);
    x3 = subm(subm(x3, A.x, p), B.x, p);
    const pw_t y3 = subm(mmul(lam, subm(A.x, x3, p), M), A.y, p);
    return ECPt{x3, y3, false};
}

__device__ ECPt ec_mul(ECPt A, u64 n, const Curve &E) {
    ECPt z{0, 0, true};
    while (n) {
        if (n & 1ull) z = ec_add(z, A, E);
        n >>= 1;
        if (n) A = ec_add(A, A, E);
    }
    return z;
}

__device__ __forceinline__ u32 isqrt64d(u64 n) {
    u64 x = (u64)sqrt((double)n);
    while (x * x > n) --x;
    while ((x + 1) * (x + 1) <= n) ++x;
    return (u32)x;
}

__device__ __forceinline__ int chi(pw_t a, const Mont &M) {   // a plain, a < p
    if (a == 0u) return 0;
    const pw_t v = mpow(to_mont(a, M), (M.p - 1u) / 2u, M);
    return v == M.one ? 1 : -1;
}

// square root of a Montgomery quadratic residue (Tonelli-Shanks); nr is a
// Montgomery non-residue
__device__ pw_t sqrt_m(pw_t a, pw_t nr, const Mont &M) {
    const pw_t p = M.p;
    if (a == 0u) return 0u;
    if ((p & 3u) == 3u) return mpow(a, (p + 1u) / 4u, M);
    pw_t q = p - 1u;
    u32 S = 0;
    while (!(q & 1u)) { q >>= 1; ++S; }
    pw_t c = mpow(nr, q, M), x = mpow(a, (q + 1u) / 2u, M), t = mpow(a, q, M);
    u32 m = S;
    for (int guard = 0; guard < 40 && t != M.one; ++guard) {
        u32 i = 1;
        pw_t v = mmul(t, t, M);
        while (v != M.one && i < m) { v = mmul(v, v, M); ++i; }
        if (i >= m) return NO_ROOT;
        pw_t b = c;
        for (u32 k = 0; k + i + 1u < m; ++k) b = mmul(b, b, M);
        x = mmul(x, b, M);
        c = mmul(b, b, M);
        t = mmul(t, c, M);
        m = i;
    }
    return x;
}

__device__ __forceinline__ u64 gcd64d(u64 a, u64 b) { while (b) { u64 t = a % b; a = b; b = t; } return a; }

__global__ void __launch_bounds__(A4_WARPS * 32)
a4_kernel(const PrimeDesc *primes, u32 n, u32 *out, u32 *err) {
    __shared__ pw_t hkey[A4_WARPS][A4_SLOTS];
    __shared__ pw_t hy[A4_WARPS][A4_SLOTS];
    __shared__ unsigned short hj[A4_WARPS][A4_SLOTS];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const u32 idx = blockIdx.x * A4_WARPS + warp;
    if (idx >= n) return;
    const pw_t p = primes[idx].p;
    if (p <= 3u) { if (lane == 0) out[idx] = 0u; return; }
    if (primes[idx].status & ST_ROOT) {           // not a prime (setup): no count, the call is refused
        if (lane == 0) { atomicOr(err, 1u); out[idx] = 0u; }
        return;
    }
    const Mont M = make_mont(p);
    if (p < 1000u) {
        // direct count, characters by Euler's criterion
        u32 cnt = 0;
        for (u32 x = 1u + lane; x + 3u < p; x += 32u) {
            const int c0 = chi((pw_t)x, M);
            cnt += (chi((pw_t)x + 1u, M) == c0 && chi((pw_t)x + 2u, M) == c0 && chi((pw_t)x + 3u, M) == c0);
        }
        cnt = __reduce_add_sync(0xFFFFFFFFu, cnt);
        if (lane == 0) out[idx] = cnt;
        return;
    }
    pw_t *keys = hkey[warp];
    pw_t *ys = hy[warp];
    unsigned short *js = hj[warp];
    // least quadratic non-residue (twist parameter and Tonelli-Shanks)
    u32 nr = 0;
    for (u32 base = 2; nr == 0u && base < 100000u; base += 32u) {
        const bool q = chi((pw_t)(base + lane), M) == -1;
        const u32 bal = __ballot_sync(0xFFFFFFFFu, q);
        if (bal) nr = base + (u32)(__ffs(bal) - 1);
    }
    const pw_t nrm = to_mont((pw_t)nr, M);
    const u32 R = isqrt64d(4ull * p);
    const u64 L = (u64)p + 1u - R, H = (u64)p + 1u + R, W = H - L;
    u32 m = isqrt64d(W + 1u);
    if ((u64)m * m < W + 1u) ++m;
    u64 ord[2] = {4, 4};
    u32 nextx[2] = {2, 2};
    u64 N = 0;
    for (u32 attempt = 0; attempt < A4_MAX_ATTEMPTS && N == 0; ++attempt) {
        const u32 cv = attempt & 1u;
        const pw_t s = cv ? nr : 1u;
        Curve E;
        E.M = M;
        const pw_t sm = to_mont(s, M);
        E.s10 = mmul(to_mont((pw_t)10, M), sm, M);
        E.s20 = mmul(to_mont((pw_t)20, M), sm, M);
        E.s9sq = mmul(to_mont((pw_t)9, M), mmul(sm, sm, M), M);
        E.three = to_mont((pw_t)3, M);
        const pw_t s9 = mmul(to_mont((pw_t)9, M), sm, M);
        // a point with y != 0: first lane whose x gives a nonzero square
        ECPt P{0, 0, true};
        for (int g = 0; g < 4096 && P.inf; ++g) {
            const pw_t xp = (pw_t)(nextx[cv] + lane) % p;
            const pw_t xm = to_mont(xp, M);
            const pw_t rhs = mmul(mmul(xm, subm(xm, sm, p), M), subm(xm, s9, p), M);
            const bool ok = rhs != 0u && mpow(rhs, (p - 1u) / 2u, M) == M.one;
            const u32 bal = __ballot_sync(0xFFFFFFFFu, ok);
            if (bal) {
                const int f = __ffs(bal) - 1;
                const pw_t xs = __shfl_sync(0xFFFFFFFFu, xm, f);
                const pw_t rs = __shfl_sync(0xFFFFFFFFu, rhs, f);
                const pw_t y = sqrt_m(rs, nrm, M);
                nextx[cv] += (u32)f + 1u;
                if (y != NO_ROOT) P = ECPt{xs, y, false};
            } else {
                nextx[cv] += 32u;
            }
        }
        if (P.inf) break;
        // baby steps: j P for j in [0, m), hashed by x (key x+1, identity skipped)
        for (u32 i = lane; i < A4_SLOTS; i += 32) keys[i] = 0u;
        __syncwarp();
        const u32 per = (m + 31u) / 32u;
        {
            const u32 j0 = (u32)lane * per;
            ECPt Q = ec_mul(P, j0, E);
            for (u32 j = j0; j < j0 + per && j < m; ++j) {
                if (!Q.inf) {
                    const pw_t key = Q.x + 1u;
                    u32 h = hash_slot(key, 10);
                    for (u32 probe = 0; probe < A4_SLOTS; ++probe) {
                        const pw_t old = cas_key(&keys[h], (pw_t)0, key);
                        if (old == 0u) { ys[h] = Q.y; js[h] = (unsigned short)j; break; }
                        if (old == key) break;
                        h = (h + 1u) & (A4_SLOTS - 1u);
                    }
                }
                Q = ec_add(Q, P, E);
            }
        }
        __syncwarp();
        // giant steps G_i = (L + i m) P; G_i = -jP  =>  n = L + i m + j,
        //                                 G_i = +jP  =>  n = L + i m - j
        const u64 ngiant = W / m + 2u;
        const ECPt step = ec_mul(P, 32ull * m, E);
        ECPt G = ec_mul(P, L + (u64)lane * m, E);
        u64 found = ~0ull;
        for (u64 i = lane; i < ngiant; i += 32u) {
            const u64 base = L + i * m;
            if (G.inf) { if (base <= H) found = min(found, base); }
            else {
                u32 h = hash_slot((pw_t)(G.x + 1u), 10);
                for (u32 probe = 0; probe < A4_SLOTS; ++probe) {
                    const pw_t k = keys[h];
                    if (k == 0u) break;
                    if (k == G.x + 1u) {
                        const u32 j = js[h];
                        if (ys[h] == subm(0u, G.y, p) || (G.y == 0u && ys[h] == 0u)) {
                            const u64 nn = base + j;
                            if (nn >= L && nn <= H) found = min(found, nn);
                        }
                        if (ys[h] == G.y && base >= L + j) {
                            const u64 nn = base - j;
                            if (nn >= L && nn <= H && nn > 0) found = min(found, nn);
                        }
                        break;
                    }
                    h = (h + 1u) & (A4_SLOTS - 1u);
                }
            }
            G = ec_add(G, step, E);
        }
        // warp minimum of the matched multiple
        u32 fhi = (u32)(found >> 32), flo = (u32)found;
        const u32 mhi = __reduce_min_sync(0xFFFFFFFFu, fhi);
        const u32 mlo = __reduce_min_sync(0xFFFFFFFFu, fhi == mhi ? flo : 0xFFFFFFFFu);
        const u64 nmul = ((u64)mhi << 32) | mlo;
        if (nmul == ~0ull) continue;
        // exact order of P: for each prime q | nmul remove q while (nmul/q^k) P = O
        // (lane-parallel trial division over candidate factors)
        u64 rem = nmul;
        // factor by trial division: lanes test odd q in strides
        __shared__ u64 fac[A4_WARPS][24];
        __shared__ u32 nfac[A4_WARPS];
        if (lane == 0) nfac[warp] = 0;
        __syncwarp();
        if (lane == 0) {
            if ((rem & 1ull) == 0ull) { fac[warp][nfac[warp]++] = 2; while ((rem & 1ull) == 0ull) rem >>= 1; }
        }
        {
            const u32 rh = __shfl_sync(0xFFFFFFFFu, (u32)(rem >> 32), 0);
            const u32 rl = __shfl_sync(0xFFFFFFFFu, (u32)rem, 0);
            rem = ((u64)rh << 32) | rl;
        }
        for (u64 qb = 3; qb * qb <= rem; qb += 64u) {
            const u64 q = qb + 2u * (u64)lane;
            const bool div = (q * q <= rem) && (rem % q == 0ull);
            u32 bal = __ballot_sync(0xFFFFFFFFu, div);
            while (bal) {
                const int f = __ffs(bal) - 1;
                bal &= bal - 1u;
                const u64 qq = qb + 2u * (u64)f;
                if (rem % qq != 0ull) continue;         // composite: its prime factors went first
                if (lane == 0 && nfac[warp] < 24u) fac[warp][nfac[warp]++] = qq;
                while (rem % qq == 0ull) rem /= qq;
            }
        }
        __syncwarp();
        if (lane == 0 && rem > 1ull && nfac[warp] < 24u) fac[warp][nfac[warp]++] = rem;
        __syncwarp();
        const u32 nf = nfac[warp];
        u64 keep = 1;   // per lane: q^(v_q(n) - k_q) for its factor
        if ((u32)lane < nf) {
            const u64 q = fac[warp][lane];
            u64 d = nmul;
            u32 v = 0;
            while (d % q == 0ull) { d /= q; ++v; }
            // d = nmul / q^v ; least e with q^e (d P) = O, multiplying by q in place
            ECPt X = ec_mul(P, d, E);
            u32 e = 0;
            while (e < v && !X.inf) { X = ec_mul(X, q, E); ++e; }
            keep = 1;
            for (u32 k = 0; k < e; ++k) keep *= q;
        }
        // order = product of lanes' keep
        u64 o = keep;
        for (int off = 16; off > 0; off >>= 1) {
            const u32 hi2 = __shfl_xor_sync(0xFFFFFFFFu, (u32)(o >> 32), off);
            const u32 lo2 = __shfl_xor_sync(0xFFFFFFFFu, (u32)o, off);
            o *= ((u64)hi2 << 32) | lo2;
        }
        ord[cv] = ord[cv] / gcd64d(ord[cv], o) * o;
        const u64 first = (L + ord[cv] - 1u) / ord[cv] * ord[cv];
        if (first <= H && first + ord[cv] > H) N = cv ? 2ull * p + 2ull - first : first;
    }
    if (lane == 0) {
        if (N == 0) { atomicOr(err, 1u); out[idx] = 0u; return; }
        const int b = 4 * chi((pw_t)2, M) + 2 * chi((pw_t)6 % p, M) + 2 * chi((pw_t)3, M) + 2 * chi(p - 1u, M) +
                      2 * chi(p - 2u, M);
        const long long num = (long long)N - 12 - b;
        if (num < 0 || (num & 7)) { atomicOr(err, 2u); out[idx] = 0u; return; }
        out[idx] = (u32)(num / 8);
    }
}

}  // namespace CZ_NS
