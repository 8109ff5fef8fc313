/*
 * census_oracle.c -- CPU restatement of the reference census arithmetic.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker: it is called by the
 * tests, by __graft_entry__.smoke() and by bench.py's CPU-baseline leg, and
 * never by the product path (rabung_atlas32_b200/), which fails loudly
 * when its CUDA library is missing.
 *
 * Parity is pinned: tests/test_oracle.py checks every function here against
 * the reference's shipped sample blocks (data/sample/scan-00000.vdw,
 * scan-49900.vdw, quadruplets-*.a4), the 4 x 1024 holdout profiles of
 * reproducibility/gpu_method/throughput/holdout-32-mr_selected.json and
 * the outputs of the reference's own CPU programs built into oracle/_ref.
 *
 * Each function cites the reference file:line whose algorithm it restates.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef uint64_t u64;
typedef uint32_t u32;
typedef unsigned __int128 u128;
typedef __int128 i128;

static u64 mulmod(u64 a, u64 b, u64 p) { return (u64)((u128)a * b % p); }

static u64 powmod(u64 a, u64 e, u64 p) {
    u64 v = 1 % p;
    a %= p;
    while (e) {
        if (e & 1) v = mulmod(v, a, p);
        a = mulmod(a, a, p);
        e >>= 1;
    }
    return v;
}

/* Deterministic Miller-Rabin on the first twelve prime bases, exact for
 * every 64-bit n (src/census/theorie/bounded_prime.hpp:6-17). */
int orc_is_prime(u64 n) {
    static const u64 bases[12] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37};
    if (n < 2) return 0;
    for (int i = 0; i < 12; ++i) {
        if (n == bases[i]) return 1;
        if (n % bases[i] == 0) return 0;
    }
    u64 d = n - 1;
    unsigned s = 0;
    while (!(d & 1)) { d >>= 1; ++s; }
    for (int i = 0; i < 12; ++i) {
        u64 x = powmod(bases[i], d, n);
        if (x == 1 || x == n - 1) continue;
        int pass = 0;
        for (unsigned j = 1; j < s; ++j) {
            x = mulmod(x, x, n);
            if (x == n - 1) { pass = 1; break; }
            if (x == 1) return 0;
        }
        if (!pass) return 0;
    }
    return 1;
}

/* Admissibility mask: bit r-2 set when r | p-1, r = 2..9
 * (scripts/atlas_codec.py:6). */
u32 orc_mask(u64 p) {
    u32 m = 0;
    for (u32 r = 2; r <= 9; ++r)
        if ((p - 1) % r == 0) m |= 1u << (r - 2);
    return m;
}

static u64 gcd64(u64 a, u64 b) { while (b) { u64 t = a % b; a = b; b = t; } return a; }

static int factor_distinct(u64 n, u64 *f) {
    int k = 0;
    for (u64 q = 2; q <= n / q; ++q)
        if (n % q == 0) { f[k++] = q; while (n % q == 0) n /= q; }
    if (n > 1) f[k++] = n;
    return k;
}

/* Least primitive root (src/census/small_cpu.cpp:18). */
u64 orc_primitive_root(u64 p) {
    if (p == 2) return 1;
    u64 f[64];
    int k = factor_distinct(p - 1, f);
    for (u64 g = 2;; ++g) {
        int ok = 1;
        for (int i = 0; i < k; ++i)
            if (powmod(g, (p - 1) / f[i], p) == 1) { ok = 0; break; }
        if (ok) return g;
    }
}

/*
 * Dense profiles by a primitive-root walk over the whole of [1, p-1]
 * (src/census/small_cpu.cpp:15-33, without its p <= 2e6 guard; the same
 * walk as reproducibility/bounds_update/independent_profile.cpp:55-88).
 * idx[x] = log_g(x) mod lcm(r); colour_r(x) = idx[x] mod r.  For each set
 * bit r of `mask`: M = longest run, L = initial colour-0 run from x=1,
 * W = least reflected start min(s, p-(s+M-1)) over runs of length M.
 * Arrays are indexed by r (size >= 10).  Returns 0, or -1 on allocation
 * failure.  Memory: 2 bytes per residue.
 */
int orc_profiles_dense(u64 p, u32 mask, u64 *M, u64 *L, u64 *W) {
    if (p < 3 || !mask) return 0;
    u64 m = 1;
    for (u64 r = 2; r <= 9; ++r)
        if (mask & (1u << (r - 2))) m = m / gcd64(m, r) * r;
    uint16_t *idx = (uint16_t *)malloc(sizeof(uint16_t) * p);
    if (!idx) return -1;
    u64 g = orc_primitive_root(p), x = 1;
    u32 label = 0;
    for (u64 e = 0; e < p - 1; ++e) {
        idx[x] = (uint16_t)label;
        if (++label == m) label = 0;
        x = x * g % p;
    }
    for (u32 r = 2; r <= 9; ++r) {
        if (!(mask & (1u << (r - 2)))) continue;
        u64 mx = 0, wi = p, start = 1, len = 0;
        int last = -1;
        for (u64 y = 1; y < p; ++y) {
            int c = idx[y] % r;
            if (c != last) {
                if (len) {
                    u64 w = start < p - (start + len - 1) ? start : p - (start + len - 1);
                    if (len > mx) { mx = len; wi = w; }
                    else if (len == mx && w < wi) wi = w;
                }
                start = y; len = 1; last = c;
            } else ++len;
        }
        if (len) {
            u64 w = start < p - (start + len - 1) ? start : p - (start + len - 1);
            if (len > mx) { mx = len; wi = w; }
            else if (len == mx && w < wi) wi = w;
        }
        u64 pre = 0;
        while (pre + 1 < p && idx[pre + 1] % r == 0) ++pre;
        M[r] = mx; L[r] = pre; W[r] = wi;
    }
    free(idx);
    return 0;
}

/* K (docs/METHODS.md:11-18; scripts/atlas_codec.py:8). */
u64 orc_threshold_k(u64 p, u64 r, u64 M, u64 L) {
    u64 b = (((p - 1) / 2) % r == 0) ? 2 * L + 2 : L + 2;
    return M + 1 > b ? M + 1 : b;
}

/* Initial residue run by direct powering (src/census/worker32.cu:38). */
u64 orc_prefix(u64 p, u64 r) {
    u64 pre = 1;
    while (pre + 1 < p && powmod(pre + 1, (p - 1) / r, p) == 1) ++pre;
    return pre;
}

/* Dense A4 (src/census/moment_worker.cpp:11-18): x in [1, p-4] with
 * x..x+3 all residues or all non-residues. */
u64 orc_a4_dense(u64 p) {
    if (p <= 3) return 0;
    unsigned char *sq = (unsigned char *)calloc(p, 1);
    if (!sq) return (u64)-1;
    for (u64 x = 1; x < p; ++x) sq[mulmod(x, x, p)] = 1;
    u64 n = 0;
    for (u64 x = 1; x + 3 < p; ++x)
        n += (sq[x] == sq[x + 1] && sq[x] == sq[x + 2] && sq[x] == sq[x + 3]);
    free(sq);
    return n;
}

/* ---- elliptic point count of E_s: y^2 = x(x-s)(x-9s) over F_p ----------
 * Restates the published BSGS-in-the-Hasse-interval method with an
 * lcm-of-point-orders uniqueness certificate of
 * src/census/theorie/elliptic4_mestre.cpp:42-62 (curve :22-31), with
 * deterministic point choice.  N is unique, so the point choice does not
 * change the count. */
typedef struct { u64 x, y; int inf; } pt;

static u64 inv_mod(u64 a, u64 p) { return powmod(a, p - 2, p); }

static pt ec_add(pt a, pt b, u64 s, u64 p) {
    if (a.inf) return b;
    if (b.inf) return a;
    u64 lam;
    if (a.x == b.x) {
        if ((a.y + b.y) % p == 0) { pt o = {0, 0, 1}; return o; }
        /* y^2 = x^3 - 10 s x^2 + 9 s^2 x: slope (3x^2 - 20 s x + 9 s^2) / 2y */
        u64 x = a.x;
        u64 num = (mulmod(3, mulmod(x, x, p), p) + p - mulmod(mulmod(20 % p, s, p), x, p)
                   + mulmod(9 % p, mulmod(s, s, p), p)) % p;
        lam = mulmod(num, inv_mod(2 * a.y % p, p), p);
    } else {
        lam = mulmod((b.y + p - a.y) % p, inv_mod((b.x + p - a.x) % p, p), p);
    }
    u64 x3 = (mulmod(lam, lam, p) + mulmod(10 % p, s, p) + 2 * p - a.x - b.x) % p;
    u64 y3 = (mulmod(lam, (a.x + p - x3) % p, p) + p - a.y) % p;
    pt r = {x3, y3, 0};
    return r;
}

static pt ec_mul(pt a, u64 n, u64 s, u64 p) {
    pt z = {0, 0, 1};
    while (n) {
        if (n & 1) z = ec_add(z, a, s, p);
        a = ec_add(a, a, s, p);
        n >>= 1;
    }
    return z;
}

static u64 isqrt64(u64 n) {
    u64 x = 0;
    for (u64 b = (u64)1 << 31; b; b >>= 1)
        if ((x + b) * (x + b) <= n) x += b;
    return x;
}

static u64 rhs(u64 x, u64 s, u64 p) {
    return mulmod(mulmod(x, (x + p - s % p) % p, p), (x + p - mulmod(9, s, p)) % p, p);
}

/* square root mod p (Tonelli-Shanks); returns 0 if a is a non-residue */
static int sqrt_mod(u64 a, u64 p, u64 *out) {
    if (a == 0) { *out = 0; return 1; }
    if (powmod(a, (p - 1) / 2, p) != 1) return 0;
    if (p % 4 == 3) { *out = powmod(a, (p + 1) / 4, p); return 1; }
    u64 q = p - 1, e = 0;
    while (!(q & 1)) { q >>= 1; ++e; }
    u64 z = 2;
    while (powmod(z, (p - 1) / 2, p) != p - 1) ++z;
    u64 c = powmod(z, q, p), x = powmod(a, (q + 1) / 2, p), t = powmod(a, q, p), m = e;
    while (t != 1) {
        u64 i = 1, v = mulmod(t, t, p);
        while (v != 1) { v = mulmod(v, v, p); ++i; }
        u64 b = powmod(c, (u64)1 << (m - i - 1), p);
        x = mulmod(x, b, p); c = mulmod(b, b, p); t = mulmod(t, c, p); m = i;
    }
    *out = x;
    return 1;
}

typedef struct { u64 x, y; u32 j; u32 used; } slot;

/* smallest n in [lo, lo+w] with nP = O (n exists: #E lies in the window) */
static u64 bsgs_window(pt P, u64 lo, u64 w, u64 s, u64 p) {
    u64 m = isqrt64(w + 1);
    if (m * m < w + 1) ++m;
    u64 cap = 1;
    while (cap < 4 * m) cap <<= 1;
    slot *tab = (slot *)calloc(cap, sizeof(slot));
    pt v = {0, 0, 1};
    u64 found = 0;
    for (u64 j = 0; j < m; ++j) {
        u64 h = v.inf ? 0 : (v.x * 0x9E3779B97F4A7C15ull ^ v.y) & (cap - 1);
        while (tab[h].used) h = (h + 1) & (cap - 1);
        tab[h].x = v.inf ? (u64)-1 : v.x; tab[h].y = v.inf ? (u64)-1 : v.y;
        tab[h].j = (u32)j; tab[h].used = 1;
        v = ec_add(v, P, s, p);
    }
    pt step = ec_mul(P, m, s, p);
    if (!step.inf) step.y = (p - step.y) % p;
    pt Q = ec_mul(P, lo, s, p);
    if (!Q.inf) Q.y = (p - Q.y) % p;
    u64 best = 0;
    for (u64 i = 0; i <= w / m + 1 && !found; ++i) {
        u64 kx = Q.inf ? (u64)-1 : Q.x, ky = Q.inf ? (u64)-1 : Q.y;
        u64 h = Q.inf ? 0 : (Q.x * 0x9E3779B97F4A7C15ull ^ Q.y) & (cap - 1);
        while (tab[h].used) {
            if (tab[h].x == kx && tab[h].y == ky) {
                u64 n = lo + i * m + tab[h].j;
                if (n - lo <= w) { best = n; found = 1; }
                break;
            }
            h = (h + 1) & (cap - 1);
        }
        Q = ec_add(Q, step, s, p);
    }
    free(tab);
    return best;
}

static u64 exact_order(pt P, u64 n, u64 s, u64 p) {
    u64 f[64];
    int k = factor_distinct(n, f);
    u64 d = n;
    for (int i = 0; i < k; ++i)
        while (d % f[i] == 0 && ec_mul(P, d / f[i], s, p).inf) d /= f[i];
    return d;
}

/* #E_1(F_p) for p >= 1000, or 0 on failure to certify. */
u64 orc_elliptic_count(u64 p) {
    u64 R = isqrt64(4 * p), L = p + 1 - R, H = p + 1 + R, W = H - L;
    u64 twist = 2;
    while (powmod(twist, (p - 1) / 2, p) != p - 1) ++twist;
    u64 svals[2] = {1, twist}, ord[2] = {1, 1};
    u64 xs[2] = {2, 2};
    for (int attempt = 0; attempt < 400; ++attempt) {
        int c = attempt & 1;
        u64 s = svals[c], y = 0, x;
        for (;;) {
            x = xs[c]++ % p;
            if (sqrt_mod(rhs(x, s, p), p, &y) && y != 0) break;
        }
        pt P = {x, y, 0};
        u64 n = bsgs_window(P, L, W, s, p);
        if (!n) return 0;
        u64 d = exact_order(P, n, s, p);
        ord[c] = ord[c] / gcd64(ord[c], d) * d;
        u64 first = (L + ord[c] - 1) / ord[c] * ord[c];
        if (first <= H && first + ord[c] > H)
            return c ? 2 * p + 2 - first : first;
    }
    return 0;
}

static int legendre(u64 x, u64 p) {
    x %= p;
    if (!x) return 0;
    return powmod(x, (p - 1) / 2, p) == 1 ? 1 : -1;
}

/* A4 from the point count (src/census/theorie/elliptic4_mestre.cpp:64-67):
 * A4 = (N - 12 - b)/8, b = 4chi(2)+2chi(6)+2chi(3)+2chi(-1)+2chi(-2). */
u64 orc_a4_from_count(u64 p, u64 N) {
    i128 b = 4 * legendre(2, p) + 2 * legendre(6, p) + 2 * legendre(3, p)
             + 2 * legendre(p - 1, p) + 2 * legendre(p - 2, p);
    i128 num = (i128)N - 12 - b;
    if (num < 0 || num % 8) return (u64)-1;
    return (u64)(num / 8);
}

/* A4 exactly as the reference worker routes it: dense for p < 1000,
 * elliptic count otherwise (src/census/moment_worker.cpp:37-38). */
u64 orc_a4(u64 p) {
    if (p < 1000) return orc_a4_dense(p);
    u64 N = orc_elliptic_count(p);
    if (!N) return (u64)-1;
    return orc_a4_from_count(p, N);
}

/* Primes in [lo, hi), hi - lo <= 2^26; returns count written (<= cap)
 * (src/census/prime_sieve.cpp:8-22). */
u64 orc_sieve(u64 lo, u64 hi, u64 *out, u64 cap) {
    if (hi <= lo) return 0;
    u64 top = isqrt64(hi);
    unsigned char *base = (unsigned char *)calloc(top + 1, 1);
    unsigned char *mark = (unsigned char *)malloc(hi - lo);
    memset(mark, 1, hi - lo);
    u64 k = 0;
    for (u64 q = 2; q <= top; ++q) {
        if (base[q]) continue;
        for (u64 j = q * q; j <= top; j += q) base[j] = 1;
        u64 first = q * q > ((lo + q - 1) / q) * q ? q * q : ((lo + q - 1) / q) * q;
        for (u64 j = first; j < hi; j += q) mark[j - lo] = 0;
    }
    for (u64 v = lo; v < hi; ++v)
        if (v >= 2 && mark[v - lo] && k < cap) out[k++] = v;
    free(base);
    free(mark);
    return k;
}
