// sparse.cuh -- certified rational-anchor filter with exact completion.
//
// Mathematics (the reference's GPU method, paper/GPU_METHOD_EN.tex:256-560):
//  * Cover (Thm "integer coverage certificate"; P/src/clipped_cover.hpp:7-21):
//    with H = Q-1, B < p, D < p, H*D <= 2B and 4BD - H D^2 > 4p, every window
//    x..x+H of [1, p-1] has numerators a+jd (a = dx mod p, 1 <= d <= D,
//    gcd(a, d) = 1) all in [-B, B]; colour(x+j) = colour(a+jd) - colour(d), so
//    colour constancy of the window is read off the signed table.
//  * A run of length >= q (q <= Q) contains a q-window; it holds s = q-t+1
//    anchors of length t along its row.  Writing an anchor by its top
//    numerator b (numerators b, b-d, ..., b-(t-1)d) and v = b - ceil((t-1)d/2),
//    this build selects b iff v mod (d*s) < d: every s consecutive anchors of a
//    row contain exactly one selected b, and the rule is symmetric under the
//    reflection b -> (t-1)d - b (colours shift by colour(-1), positions x ->
//    p-x, canonical witness unchanged), so only v >= 0 is enumerated (the role
//    of the reference's folded bands and phase rule, P/src/periodic_bands.hpp:28-78;
//    this rule keeps whole bands of d consecutive b, so 32-bit words are full).
//    The anchors of a primitive row share gcd(b, d) = 1, so for even d only odd
//    b are enumerated, on the odd-numerator view of the table (the reference's
//    G = 2 wheel, PBV/src/wheel_filter.hpp:14-46).
//  * Filter (PBV/src/wheel_filter.hpp:52-91): a candidate anchor survives while
//    every offset b - jd (j < t) agrees with b on every colour plane; here 64
//    anchors per lane-word, their stages in batches whose loads issue together.
//  * Bilateral screen (B1/src/two_cuts.hpp:27-74): reject only when known
//    mismatches on both sides bound the run below the verified maximum;
//    numerators outside [-B, B] are unknown and never reject.
//  * Exact completion (PBV/src/completion.hpp:17-57, E32/src/completion_core.hpp:17-48):
//    x = b/d mod p, extend both ways with table colours, falling back to a
//    direct power outside the table; reduce by (length, least witness) with a
//    packed 64-bit atomicMax.
//  * Exactness (Thm "exactness on successful termination"): every row d is
//    processed with a fixed q <= (a verified run length) <= M, so every maximum
//    run (or its reflection) is completed.
//
// B200 design: one persistent kernel over all profiles of a call, handed out
// longest first; a group of CTAs (2 for large calls, up to 64 when a call has
// few profiles) shares one (p, r) profile, its warps pull rows d in increasing
// order from the profile's counter in global memory and re-read the verified
// maximum at every row, so the threshold rises while the profile runs; each
// stored plane count has its own row loop (its own registers); lanes take
// consecutive 64-anchor words of a row, a window is cut from three plane words
// by funnel shifts, fetched through the load/store pipe for 1 and 2 planes and
// through the texture pipe (linear textures over the plane pool) for 4 planes,
// so the two L1 pipes share the load; words that survive are queued per warp
// (across rows) and screened 32 at a time, one per lane, and the screened
// candidates are completed 32 at a time, one per lane.
#pragma once
#include "labels.cuh"

namespace cz {

#ifndef CZ_SB1                       // anchor stages whose loads issue together, by stored planes
#define CZ_SB1 5                     // r = 2 runs t - 1 = 10 stages: two batches of 5
#endif
#ifndef CZ_SB2
#define CZ_SB2 2
#endif
#ifndef CZ_SB4
#define CZ_SB4 1
#endif
#ifndef CZ_SPARSE_MINB                // resident filter CTAs per SM (register budget)
#define CZ_SPARSE_MINB 2
#endif

#ifndef CZ_TEX_MASK                   // stored plane counts (bit NPP) whose windows go through textures
#define CZ_TEX_MASK 4
#endif
constexpr u32 TEX_CHUNK_WORDS_LOG2 = 27;   // texture chunks of the plane pool: 2^27 words (512 MiB)

#ifndef CZ_SPARSE_WARPS               // warps per filter CTA
#define CZ_SPARSE_WARPS 16
#endif
constexpr int SPARSE_WARPS = CZ_SPARSE_WARPS;
constexpr int CAND_CAP = 64;          // per-warp buffers
constexpr u32 RUN_CAP = 4096;         // longest run a completion may walk

struct Tuning {
    u32 screen;        // 1: bilateral screen on
};

struct SparseArgs {
    const PrimeDesc *primes;
    const ProfDesc *profs;
    ProfState *state;
    const u32 *planes;
    const u32 *prof_list;     // global profile indices (sparse-routed)
    u32 nlist;
    u32 *next;                // work counter: CTA slots handed out
    u32 group;                // CTAs that share one profile (its rows)
    Tuning tune;
    const unsigned long long *texs;   // linear textures over the plane pool: [uint, uint2, uint4][chunk]
    u32 tex_chunks;
};

struct Cand { u32 b, d; };

// preferred anchor length: least t with r^(t-1) >= 2^(5+bits), i.e. a word of
// 32 random anchors keeps on average <= 2^-bits survivors
CZ_HD u32 anchor_pref(u32 r, u32 bits) {
    const u64 goal = u64(1) << (5u + bits);
    u64 pw = 1;
    u32 k = 0;
    while (pw < goal) { pw *= r; ++k; }
    return k + 1u;
}

// windows of all NPP interleaved planes at bit index u
template <int NPP> struct Planes;
template <> struct Planes<1> {
    static __device__ __forceinline__ void win(const u32 *__restrict__ P, u32 u, u32 *o) {
        const u32 *q = P + (u >> 5);
        o[0] = __funnelshift_r(__ldg(q), __ldg(q + 1), u & 31u);
    }
    // 64-bit window: lo = bits [u, u+32), hi = bits [u+32, u+64)
    static __device__ __forceinline__ void win64(const u32 *__restrict__ P, u32 u, u32 *lo, u32 *hi) {
        const u32 *q = P + (u >> 5);
        const u32 a = __ldg(q), b = __ldg(q + 1), c = __ldg(q + 2), sh = u & 31u;
        lo[0] = __funnelshift_r(a, b, sh);
        hi[0] = __funnelshift_r(b, c, sh);
    }
};
template <> struct Planes<2> {
    static __device__ __forceinline__ void win(const u32 *__restrict__ P, u32 u, u32 *o) {
        const uint2 *q = reinterpret_cast<const uint2 *>(P) + (u >> 5);
        const uint2 a = __ldg(q), b = __ldg(q + 1);
        o[0] = __funnelshift_r(a.x, b.x, u & 31u);
        o[1] = __funnelshift_r(a.y, b.y, u & 31u);
    }
    static __device__ __forceinline__ void win64(const u32 *__restrict__ P, u32 u, u32 *lo, u32 *hi) {
        const uint2 *q = reinterpret_cast<const uint2 *>(P) + (u >> 5);
        const uint2 a = __ldg(q), b = __ldg(q + 1), c = __ldg(q + 2);
        const u32 sh = u & 31u;
        lo[0] = __funnelshift_r(a.x, b.x, sh); hi[0] = __funnelshift_r(b.x, c.x, sh);
        lo[1] = __funnelshift_r(a.y, b.y, sh); hi[1] = __funnelshift_r(b.y, c.y, sh);
    }
};
template <> struct Planes<4> {
    static __device__ __forceinline__ void win(const u32 *__restrict__ P, u32 u, u32 *o) {
        const uint4 *q = reinterpret_cast<const uint4 *>(P) + (u >> 5);
        const uint4 a = __ldg(q), b = __ldg(q + 1);
        const u32 sh = u & 31u;
        o[0] = __funnelshift_r(a.x, b.x, sh);
        o[1] = __funnelshift_r(a.y, b.y, sh);
        o[2] = __funnelshift_r(a.z, b.z, sh);
        o[3] = __funnelshift_r(a.w, b.w, sh);
    }
};

// mismatch mask of a window against the base windows
template <int NPP>
__device__ __forceinline__ u32 mismatch(const u32 *__restrict__ P, u32 u, const u32 *base) {
    u32 w[NPP];
    Planes<NPP>::win(P, u, w);
    u32 m = w[0] ^ base[0];
#pragma unroll
    for (int k = 1; k < NPP; ++k) m |= w[k] ^ base[k];
    return m;
}


// one view of the signed table: index i <-> numerator c + G i, i in [ilo, ihi]
struct View {
    const u32 *P;     // interleaved planes
    u32 OFF;          // bit index of i = 0
    i32 ilo, ihi;
    u32 G, c;
};

struct ProfCtx {
    u32 p, r, np, npp, Q, D, B, NW, OFF, ex;
    Mont M;
    const u32 *P;          // base view planes
    View base, odd;
    u32 om[9];
    u32 seed, qspec;       // certified stretch from the table, speculative threshold
    u32 tpref;             // preferred anchor stages for this order
    unsigned long long btex, otex;   // textures of the chunks holding the base / odd view
    u32 btoff, otoff;                // uint4 element of each view's word 0 in its chunk
};

// colour of numerator n (|n| <= B) as an integer, from the base view
__device__ __forceinline__ u32 colour_at(const ProfCtx &c, u32 u) {
    const u32 *q = c.P + (size_t)(u >> 5) * c.npp;
    u32 col = 0;
    for (u32 k = 0; k < c.np; ++k) col |= ((__ldg(q + k) >> (u & 31u)) & 1u) << k;
    return col;
}

// absolute colour of x in [1, p-1] by a direct power: x^((p-1)/r) = omega^j
__device__ __forceinline__ u32 colour_direct(u32 x, const ProfCtx &c) {
    const u32 y = mpow(to_mont(x, c.M), c.ex, c.M);
    for (u32 j = 0; j < c.r; ++j)
        if (c.om[j] == y) return j;
    return 0xFFFFFFFFu;
}

// exact completion of one candidate; returns packed key (0 on reject) and
// sets *err on an arithmetic failure
__device__ __noinline__ u64 complete_one(const ProfCtx &c, u32 b, u32 d, u32 *err) {
    const u32 p = c.p;
    // Montgomery d^-1 (= R d^-1), so mmul(b, dinv) = b d^-1 mod p
    const u32 dinv = mpow(to_mont(d, c.M), c.p - 2u, c.M);
    const u32 xr = mmul(b, dinv, c.M);
    if (xr == 0u) return 0;
    const u32 cb = colour_at(c, b + c.OFF);
    const u32 cd = colour_at(c, d + c.OFF);
    const u32 A = cb >= cd ? cb - cd : cb + c.r - cd;  // absolute colour of x_R
    u32 right = 0, left = 0;
    for (u32 k = 1;; ++k) {                            // x = xr + k, numerator b + k d
        if (k > RUN_CAP) { *err = 1; return 0; }
        const u64 x = (u64)xr + k;
        if (x >= p) break;
        const u64 n = (u64)b + (u64)k * d;
        const bool same = n <= c.B ? colour_at(c, (u32)n + c.OFF) == cb : colour_direct((u32)x, c) == A;
        if (!same) break;
        right = k;
    }
    for (u32 k = 1;; ++k) {                            // x = xr - k, numerator b - k d
        if (k > RUN_CAP) { *err = 1; return 0; }
        if (k >= xr) break;
        const u32 x = xr - k;
        const i64 n = (i64)b - (i64)k * d;
        const bool same = n >= -(i64)c.B ? colour_at(c, (u32)(n + (i64)c.OFF)) == cb : colour_direct(x, c) == A;
        if (!same) break;
        left = k;
    }
    const u32 s = xr - left, e = xr + right;
    const u32 w = s < p - e ? s : p - e;
    return pack_key(e - s + 1u, w);
}

// bilateral screen of one word at view index i0 (row step dd = d / G): keep
// bits whose run can still reach t + h (right matches + left matches >= h);
// indices outside [ilo, ihi] are unknown and match
template <int NPP>
__device__ __noinline__ u32 screen_word(const View &v, u32 i0, u32 alive, u32 dd, u32 t, u32 h) {
    if (h >= 64u) return alive;
    const u32 u0 = i0 + v.OFF;
    u32 base[NPP];
    Planes<NPP>::win(v.P, u0, base);
    u32 R[64];
    u32 cur = alive;
    bool unk = false;
    R[0] = cur;
    for (u32 k = 1; k <= h; ++k) {
        if (cur && !unk) {
            const i64 lim = (i64)v.ihi - (i64)(i32)i0 - (i64)k * dd;     // bits <= lim known
            if (lim < 0) unk = true;
            else {
                const u32 m = mismatch<NPP>(v.P, u0 + k * dd, base);
                const u32 known = lim >= 31 ? 0xFFFFFFFFu : ((2u << (u32)lim) - 1u);
                cur &= ~(m & known);
            }
        }
        R[k] = cur;
    }
    u32 lcur = alive, kept = R[h] & alive;
    bool lunk = false;
    for (u32 k = 1; k <= h && (lcur & ~kept); ++k) {
        if (!lunk) {
            const i64 low = (i64)v.ilo - (i64)(i32)i0 + (i64)(t - 1u + k) * dd;   // bits >= low known
            if (low >= 32) lunk = true;
            else {
                const u32 m = mismatch<NPP>(v.P, u0 - (t - 1u + k) * dd, base);
                const u32 known = low <= 0 ? 0xFFFFFFFFu : ~((1u << (u32)low) - 1u);
                lcur &= ~(m & known);
            }
        }
        kept |= R[h - k] & lcur;
    }
    return kept;
}

// warp state carried across rows of one profile
struct WarpQ {
    u32 ncand, nscr;
    u64 best;
    u32 words, comps, tests, err;
};

// complete `count` (<= 32) buffered candidates, one per lane
__device__ __forceinline__ void flush_cands(const ProfCtx &c, Cand *cb, WarpQ &q, u32 count, ProfState *st, int lane) {
    u64 key = 0;
    if ((u32)lane < count) {
        const Cand cd = cb[lane];
        u32 e = 0;
        key = complete_one(c, cd.b, cd.d, &e);
        q.err |= e;
    }
    q.comps += count;
    const u32 hi = (u32)(key >> 32);
    const u32 mhi = __reduce_max_sync(0xFFFFFFFFu, hi);
    const u32 lo = __reduce_max_sync(0xFFFFFFFFu, hi == mhi ? (u32)key : 0u);
    const u64 k2 = ((u64)mhi << 32) | lo;
    if (k2 > q.best) q.best = k2;
    __syncwarp();
    if (q.ncand > count && (u32)lane < q.ncand - count) cb[lane] = cb[count + lane];
    __syncwarp();
    q.ncand -= count;
    if (lane == 0 && q.best) atomicMax(&st->best, (unsigned long long)q.best);
}

// current threshold of the profile: the verified maximum (<= M), raised to the
// speculative threshold when one is set
__device__ __forceinline__ u32 threshold(const ProfCtx &c, ProfState *st) {
    const u64 bk = *(volatile unsigned long long *)&st->best;
    const u32 blen = key_len(bk) > c.seed ? key_len(bk) : c.seed;
    return c.qspec > blen ? c.qspec : blen;
}

// screen `count` (<= 32) queued words -- one per lane, each remembering its row
// (d, t) -- and queue the surviving candidates for completion; the queue is
// carried across rows, so batches stay full
template <int NPP>
__device__ __forceinline__ void screen_batch(const ProfCtx &c, uint4 *sb, Cand *cb, WarpQ &q, u32 count,
                                             bool screen, ProfState *st, int lane) {
    u32 keep = 0, i0 = 0, d = 0, vc = 0, vg = 1;
    const u32 thr = threshold(c, st);
    if ((u32)lane < count) {
        const uint4 e = sb[lane];
        i0 = e.x;
        keep = e.y;
        d = e.z;
        const u32 t = e.w;
        const View &v = (d & 1u) ? c.base : c.odd;
        vc = v.c;
        vg = v.G;
        const u32 h = thr > t ? thr - t : 0u;     // reject runs certified < threshold
        if (screen && h > 0u) keep = screen_word<NPP>(v, i0, keep, d / v.G, t, h);
    }
    __syncwarp();
    if (q.nscr > count && (u32)lane < q.nscr - count) sb[lane] = sb[count + lane];
    __syncwarp();
    q.nscr -= count;
    while (__any_sync(0xFFFFFFFFu, keep != 0u)) {
        const bool has = keep != 0u;
        const u32 bal = __ballot_sync(0xFFFFFFFFu, has);
        const u32 pos = __popc(bal & ((1u << lane) - 1u));
        if (has) {
            const u32 bit = __ffs(keep) - 1u;
            keep &= keep - 1u;
            cb[q.ncand + pos] = Cand{vc + vg * (i0 + bit), d};
        }
        q.ncand += __popc(bal);
        __syncwarp();
        if (q.ncand >= 32u) flush_cands(c, cb, q, 32u, st, lane);
    }
}

// queue one 32-bit half-word per lane for the batched screen (the batch runs
// as soon as 32 are waiting)
template <int NPP>
__device__ __forceinline__ void queue_words(const ProfCtx &c, uint4 *sb, Cand *cb, WarpQ &q, u32 i0, u32 alive,
                                            u32 d, u32 t, bool screen, ProfState *st, int lane) {
    const bool has = alive != 0u;
    const u32 bal = __ballot_sync(0xFFFFFFFFu, has);
    if (!bal) return;
    const u32 pos = __popc(bal & ((1u << lane) - 1u));
    if (has) sb[q.nscr + pos] = make_uint4(i0, alive, d, t);
    q.nscr += __popc(bal);
    __syncwarp();
    if (q.nscr >= 32u) screen_batch<NPP>(c, sb, cb, q, 32u, screen, st, lane);
}

// the NPP words of texel e of a linear texture whose texels hold NPP words
template <int NPP> struct Texel;
template <> struct Texel<1> {
    static __device__ __forceinline__ void get(unsigned long long t, int e, u32 *w) {
        w[0] = tex1Dfetch<unsigned int>(t, e);
    }
};
template <> struct Texel<2> {
    static __device__ __forceinline__ void get(unsigned long long t, int e, u32 *w) {
        const uint2 x = tex1Dfetch<uint2>(t, e);
        w[0] = x.x; w[1] = x.y;
    }
};
template <> struct Texel<4> {
    static __device__ __forceinline__ void get(unsigned long long t, int e, u32 *w) {
        const uint4 x = tex1Dfetch<uint4>(t, e);
        w[0] = x.x; w[1] = x.y; w[2] = x.z; w[3] = x.w;
    }
};

// 64-bit window lo = bits [u, u+32), hi = bits [u+32, u+64) of a view.
// Windows of the plane counts in CZ_TEX_MASK are fetched through the texture
// pipe of the L1 unit (three texels from a linear texture over the plane
// pool; u then counts from the texture chunk's element 0), the others through
// the load/store pipe: the filter is bound by load/store wavefronts, and the
// texture pipe next to it would otherwise stay idle, so profiles of different
// plane counts stop competing for one pipe.
template <int NPP>
__device__ __forceinline__ void win64(const View &v, unsigned long long tex, u32 u, u32 *lo, u32 *hi) {
    if constexpr ((CZ_TEX_MASK & NPP) != 0) {
        const int e = (int)(u >> 5);
        u32 a[NPP], b[NPP], c[NPP];
        Texel<NPP>::get(tex, e, a);
        Texel<NPP>::get(tex, e + 1, b);
        Texel<NPP>::get(tex, e + 2, c);
        const u32 sh = u & 31u;
#pragma unroll
        for (int k = 0; k < NPP; ++k) {
            lo[k] = __funnelshift_r(a[k], b[k], sh);
            hi[k] = __funnelshift_r(b[k], c[k], sh);
        }
    } else {
        Planes<NPP>::win64(v.P, u, lo, hi);
    }
}

// 64-bit mismatch mask (hi:lo) of a window against the base windows
template <int NPP>
__device__ __forceinline__ u64 mismatch64(const View &v, unsigned long long tex, u32 u, const u32 *blo,
                                          const u32 *bhi) {
    u32 lo[NPP], hi[NPP];
    win64<NPP>(v, tex, u, lo, hi);
    u32 ml = 0, mh = 0;
#pragma unroll
    for (int k = 0; k < NPP; ++k) { ml |= lo[k] ^ blo[k]; mh |= hi[k] ^ bhi[k]; }
    return ((u64)mh << 32) | ml;
}

// all selected words of row d on view v, 64 anchors per lane-word: per stage
// three plane words, two funnel shifts and two logic ops per plane test 64
// anchors, so ALU work and L1 requests per anchor-stage drop against 32-bit
// words for a few more stages per word
template <int NPP>
__device__ __forceinline__ void filter_row64(const ProfCtx &c, const View &vref, u32 d, u32 t, u32 s,
                                             const Tuning &tune, uint4 *sb, Cand *cb, WarpQ &q, ProfState *st,
                                             int lane, unsigned long long tex = 0ull, u32 tbits = 0u) {
    const View v = vref;
    const u32 G = v.G, dd = d / G;
    const u32 beta = ((t - 1u) * d + 1u) >> 1;
    const i32 istart = (i32)((beta >= v.c ? beta - v.c + G - 1u : 0u) / G);
    if (istart > v.ihi) return;
    const u32 step = dd * s;
    const u32 K = (u32)(v.ihi - istart) / step + 1u;
    const u32 nw = (dd + 63u) >> 6;
    const u32 W = K * nw;
    const float rnw = 1.0f / (float)nw;
    const bool screen = tune.screen != 0u;
    for (u32 base = 0; base < W; base += 32u) {
        const u32 rank = base + (u32)lane;
        u64 alive = 0;
        u32 i0 = 0;
        if (rank < W) {
            u32 k = (u32)((float)rank * rnw);
            if (k * nw > rank) --k;
            else if ((k + 1u) * nw <= rank) ++k;
            const u32 w = rank - k * nw;
            i0 = (u32)istart + k * step + 64u * w;
            u32 len = dd - 64u * w;
            if (len > 64u) len = 64u;
            if ((i32)i0 > v.ihi) len = 0;
            else if ((u32)(v.ihi - (i32)i0) + 1u < len) len = (u32)(v.ihi - (i32)i0) + 1u;
            alive = len >= 64u ? ~0ull : ((1ull << len) - 1ull);
        }
        if (alive) {
            ++q.words;
            const u32 u = i0 + v.OFF + tbits;        // tbits: texture chunk offset (4 planes), else 0
            u32 blo[NPP], bhi[NPP];
            win64<NPP>(v, tex, u, blo, bhi);
            constexpr int SB = NPP == 4 ? CZ_SB4 : (NPP == 2 ? CZ_SB2 : CZ_SB1);
            u32 j = 1;
            while (j < t && alive) {
                u64 m[SB];
#pragma unroll
                for (int k = 0; k < SB; ++k)
                    m[k] = (j + (u32)k < t) ? mismatch64<NPP>(v, tex, u - (j + (u32)k) * dd, blo, bhi) : 0ull;
#pragma unroll
                for (int k = 0; k < SB; ++k) alive &= ~m[k];
                j += SB;
            }
            q.tests += 2u * min(j, t) * (u32)NPP;
        }
        queue_words<NPP>(c, sb, cb, q, i0, (u32)alive, d, t, screen, st, lane);
        queue_words<NPP>(c, sb, cb, q, i0 + 32u, (u32)(alive >> 32), d, t, screen, st, lane);
    }
}

// the rows of one profile, handed out one per warp in increasing d
template <int NPP>
__device__ __forceinline__ void filter_rows(const ProfCtx &c, const SparseArgs &a, u32 tpref, uint4 *sb, Cand *cb,
                                            WarpQ &q, ProfState *st, int lane) {
    for (;;) {
        u32 d = 0;
        if (lane == 0) d = atomicAdd(&st->rows_next, 1u) + 1u;     // rows in increasing d
        d = __shfl_sync(0xFFFFFFFFu, d, 0);
        if (d > c.D) break;
        // row parameters from the verified maximum so far (<= M); with a
        // speculative threshold every run >= it is still completed, and a
        // profile whose best stays below it is re-run without it
        const u32 blen = threshold(c, st);
        const u32 q_ = blen < c.Q ? blen : c.Q;
        if (q_ < 3u) { q.err |= 2u; break; }
        const u32 t = tpref < q_ ? (tpref < 2u ? 2u : tpref) : q_;
        const u32 s = q_ - t + 1u;
        const View &v = (d & 1u) ? c.base : c.odd;
        if constexpr ((CZ_TEX_MASK & NPP) != 0)
            filter_row64<NPP>(c, v, d, t, s, a.tune, sb, cb, q, st, lane, (d & 1u) ? c.btex : c.otex,
                              32u * ((d & 1u) ? c.btoff : c.otoff));
        else
            filter_row64<NPP>(c, v, d, t, s, a.tune, sb, cb, q, st, lane);
    }
}

__global__ void __launch_bounds__(SPARSE_WARPS * 32, CZ_SPARSE_MINB)
sparse_kernel(SparseArgs a) {
    __shared__ u32 s_item, s_err;
    __shared__ Cand cbuf[SPARSE_WARPS][CAND_CAP];      // candidates awaiting completion
    __shared__ uint4 sbuf[SPARSE_WARPS][CAND_CAP];     // (index, alive, d, t) words awaiting the screen
    __shared__ ProfCtx s_ctx;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (;;) {
        if (threadIdx.x == 0) {
            // a.group consecutive CTA slots share one profile
            s_item = atomicAdd(a.next, 1u) / a.group;
            s_err = 0u;
            if (s_item < a.nlist) {
                const u32 gprof = a.prof_list[s_item];
                const ProfDesc PD = a.profs[gprof];
                const PrimeDesc PR = a.primes[PD.prime];
                ProfCtx c;
                c.p = PR.p; c.r = PD.r; c.np = PD.np; c.npp = PD.npp; c.Q = PD.Q; c.D = PD.D; c.B = PR.B;
                c.NW = PR.nwords; c.OFF = 32u * PR.K0 + 31u; c.ex = (PR.p - 1u) / PD.r;
                c.M = Mont{PR.p, PR.ninv, PR.one, PR.r2};
                c.P = a.planes + PD.plane_off;
                c.base = View{c.P, c.OFF, -(i32)PR.B, (i32)PR.B, 1u, 0u};
                // odd view: n = 2i + 1 in [-B, B]  <=>  i in [ceil((-B-1)/2), floor((B-1)/2)]
                c.odd = View{c.P + (size_t)PR.nwords * PD.npp, 32u * PR.K2, -(i32)((PR.B + 1u) / 2u),
                             (i32)((PR.B - 1u) / 2u), 2u, 1u};
                {
                    const u64 bb = (u64)PD.plane_off * 4ull;
                    const u64 ob = bb + (u64)PR.nwords * PD.npp * 4ull;
                    const u32 f = PD.npp == 1u ? 0u : (PD.npp == 2u ? 1u : 2u), sh = TEX_CHUNK_WORDS_LOG2 + 2u;
                    const u64 msk = (1ull << sh) - 1ull, tb = 4ull * PD.npp;   // bytes per texel
                    c.btex = __ldg(a.texs + f * a.tex_chunks + (bb >> sh));
                    c.btoff = (u32)((bb & msk) / tb);
                    c.otex = __ldg(a.texs + f * a.tex_chunks + (ob >> sh));
                    c.otoff = (u32)((ob & msk) / tb);
                }
                for (int j = 0; j < 9; ++j) c.om[j] = PD.omega[j];
                c.seed = *(volatile u32 *)&a.state[gprof].seed;
                c.qspec = PD.qspec;
                c.tpref = PD.tpref;
                s_ctx = c;
            }
        }
        __syncthreads();
        const u32 item = s_item;
        if (item >= a.nlist) return;
        const ProfCtx &c = s_ctx;
        ProfState *st = a.state + a.prof_list[item];
        const u32 tpref = c.tpref;
        WarpQ q{0, 0, 0, 0, 0, 0, 0};
        uint4 *sb = sbuf[warp];
        Cand *cb = cbuf[warp];
        // one row loop per stored plane count, so each keeps its own registers
        if (c.npp == 1u) filter_rows<1>(c, a, tpref, sb, cb, q, st, lane);
        else if (c.npp == 2u) filter_rows<2>(c, a, tpref, sb, cb, q, st, lane);
        else filter_rows<4>(c, a, tpref, sb, cb, q, st, lane);
        // the screen queue carries across rows: drain it, then the candidates
        if (q.nscr) {
            if (c.npp == 1u) screen_batch<1>(c, sb, cb, q, q.nscr, a.tune.screen != 0u, st, lane);
            else if (c.npp == 2u) screen_batch<2>(c, sb, cb, q, q.nscr, a.tune.screen != 0u, st, lane);
            else screen_batch<4>(c, sb, cb, q, q.nscr, a.tune.screen != 0u, st, lane);
        }
        if (q.ncand) flush_cands(c, cb, q, q.ncand, st, lane);
        if (q.err) atomicOr(&s_err, q.err);
        const u32 words = __reduce_add_sync(0xFFFFFFFFu, q.words);
        const u32 tests = __reduce_add_sync(0xFFFFFFFFu, q.tests);
        if (lane == 0) {
            atomicAdd(&st->words, (unsigned long long)words);
            atomicAdd(&st->completions, (unsigned long long)q.comps);
            atomicAdd(&st->tests, (unsigned long long)tests);
        }
        __syncthreads();
        if (threadIdx.x == 0 && s_err) atomicOr(&st->status, (s_err & 2u) ? ST_SEED : ST_QUEUE);
    }
}

}  // namespace cz
