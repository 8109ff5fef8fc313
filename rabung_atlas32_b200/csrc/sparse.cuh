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
//    every offset b - jd (j < t) agrees with b on every colour plane; here 96
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
// longest first; a group of CTAs (cta_per_profile, 1 by default, for large
// calls; up to 64 when a call has few profiles) shares one (p, r) profile.  A profile's rows d are cut into
// epochs of consecutive d, each run with one threshold q -- the verified
// maximum (or the speculative threshold) when the epoch's first work item is
// claimed -- so the threshold rises between epochs and every row keeps one q.
// A work item is (epoch, view, tile): the rows of the epoch whose parity reads
// that view, restricted to the anchor bands that start in one tile of the
// view's index range.  The tile's plane words, with the halo the t stages read
// to its left and the band width to its right, are staged into shared memory
// by one bulk asynchronous copy (cp.async.bulk, completed on an mbarrier), so
// every anchor-stage window is a shared-memory load instead of an L1/L2 one.
// Warps claim the item's rows from a shared counter; lanes take consecutive
// 96-anchor lane-words of a row (three 32-bit words, so a warp's loads are
// three words apart and conflict-free); a stage's three windows are cut from
// four plane words by funnel shifts; words that survive are queued per warp
// (across rows and items of a profile) and screened 32 at a time, one per
// lane, against the planes in global memory, and the screened candidates are
// completed 32 at a time.
#pragma once
#include "labels.cuh"
#include "finalize.cuh"

namespace CZ_NS {

#ifndef CZ_SB1                       // anchor stages whose loads issue together, by stored planes
#define CZ_SB1 5                     // (measured on 96-anchor words: r = 2 runs 10 stages as 5 + 5;
#endif                               // 2 planes 3 + 3, 3 + 2; 4 planes 2 + 2)
#ifndef CZ_TS1                       // anchor stage counts whose stage loops are compiled for a
#define CZ_TS1 11                    // fixed t, by stored planes (the measured anchor_t per order:
#endif                               // r = 2: 11; r = 3, 4: 7, 6; r = 5..9: 5; 4 the earlier r = 6..9)
#ifndef CZ_TS2A
#define CZ_TS2A 7
#endif
#ifndef CZ_TS2B
#define CZ_TS2B 6
#endif
#ifndef CZ_TS4A
#define CZ_TS4A 5
#endif
#ifndef CZ_TS4B
#define CZ_TS4B 4
#endif
#ifndef CZ_SB2
#define CZ_SB2 3
#endif
#ifndef CZ_SB4
#define CZ_SB4 2
#endif
#ifndef CZ_SPARSE_MINB                // resident filter CTAs per SM (register budget)
#define CZ_SPARSE_MINB 2
#endif

#ifndef CZ_TILE_WORDS                 // shared-memory tile of one work item, 32-bit words (all planes)
#define CZ_TILE_WORDS 20480           // 80 KiB: two filter CTAs per SM
#endif
constexpr u32 TILE_WORDS = CZ_TILE_WORDS;
constexpr u32 EPOCH_ROWS_DEFAULT = 1024;    // rows d per threshold epoch (measured: 256 -> 1024 is 3 % faster)
constexpr u32 MBAR_SPIN_LIMIT = 1u << 22;   // bounded wait on a tile copy

#ifndef CZ_SPARSE_WARPS               // warps per filter CTA
#define CZ_SPARSE_WARPS 16
#endif
constexpr int SPARSE_WARPS = CZ_SPARSE_WARPS;
constexpr int CAND_CAP = 64;          // per-warp buffer of candidates awaiting completion
constexpr int SCR_CAP = 128;          // per-warp buffer of words awaiting the screen (< 32 + three words of 32)
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
    u32 epoch_rows;           // rows d per threshold epoch
    // serving runtime only (out == nullptr otherwise): profiles span launches;
    // the last CTA to leave a profile whose items are all done writes its
    // record and counts its request down
    const volatile u32 *yield;    // mapped host flag: set -> stop claiming, leave, return
    OutRecord *out;               // records, by ProfDesc.out_slot
    u32 verify;                   // certify each record (CZ_VERIFY)
    u32 *req_pending;             // per request slot: sparse profiles not yet final
    volatile u32 *req_done;       // mapped host memory, per request slot: 1 when all are final
};

struct Cand { u32 b, d; };

// a word awaiting the screen: view index of its bit 0, its surviving anchors,
// and its row d and stages t packed as d << 8 | t (d <= D <= 2^20 by the
// cover, t <= Q <= 255 by the configuration)
struct QEnt { u32 i0, alive, dt; };

// preferred anchor length: least t with r^(t-1) >= 2^(5+bits), i.e. a word of
// 32 random anchors keeps on average <= 2^-bits survivors
CZ_HD u32 anchor_pref(u32 r, u32 bits) {
    const u64 goal = u64(1) << (5u + bits);
    u64 pw = 1;
    u32 k = 0;
    while (pw < goal) { pw *= r; ++k; }
    return k + 1u;
}

// 32-bit windows of all NPP interleaved planes at bit index u (global memory; the screen)
template <int NPP> struct Planes;
template <> struct Planes<1> {
    static __device__ __forceinline__ void win(const u32 *__restrict__ P, u32 u, u32 *o) {
        const u32 *q = P + (u >> 5);
        o[0] = __funnelshift_r(__ldg(q), __ldg(q + 1), u & 31u);
    }
};
template <> struct Planes<2> {
    static __device__ __forceinline__ void win(const u32 *__restrict__ P, u32 u, u32 *o) {
        const uint2 *q = reinterpret_cast<const uint2 *>(P) + (u >> 5);
        const uint2 a = __ldg(q), b = __ldg(q + 1);
        o[0] = __funnelshift_r(a.x, b.x, u & 31u);
        o[1] = __funnelshift_r(a.y, b.y, u & 31u);
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
    u32 gs;           // log2 G: the view's divisions by G are shifts
};

// x / y from one float reciprocal ry = 1 / y (round to nearest): the
// truncated product is within one of the quotient for x < 2^21 + 2 y (a
// float32 emulation over the filter's ranges, y <= 2^28, confirms it), and the
// remainder corrects it.  Every quotient of the row set-up is in that range:
// numerators are at most 2^20 + step, ranks below 2^20.
__device__ __forceinline__ u32 div_rcp(u32 x, u32 y, float ry) {
    u32 q = __float2uint_rz(__uint2float_rn(x) * ry);
    const i32 r = (i32)(x - q * y);
    if (r < 0) --q;
    else if ((u32)r >= y) ++q;
    return q;
}

struct ProfCtx {
    pw_t p, ex;            // prime, (p - 1) / r
    u32 r, np, npp, Q, D, B, NW, OFF;
    Mont M;
    const u32 *P;          // base view planes
    View base, odd;
    pw_t om[9];
    u32 seed, qspec;       // certified stretch from the table, speculative threshold
    u32 tpref;             // preferred anchor stages for this order
    u32 NW2;               // odd view words per plane
    u32 tmax;              // most anchor stages a row of this profile runs
    u32 ts[2];             // tile span (anchor indices) of the base / odd view
    u32 nt[2];             // tiles per epoch of each view
    u32 nepoch, nitems;    // epochs, work items
};

// colour of numerator n (|n| <= B) as an integer, from the base view
__device__ __forceinline__ u32 colour_at(const ProfCtx &c, u32 u) {
    const u32 *q = c.P + (size_t)(u >> 5) * c.npp;
    u32 col = 0;
    for (u32 k = 0; k < c.np; ++k) col |= ((__ldg(q + k) >> (u & 31u)) & 1u) << k;
    return col;
}

// absolute colour of x in [1, p-1] by a direct power: x^((p-1)/r) = omega^j
__device__ __forceinline__ u32 colour_direct(pw_t x, const ProfCtx &c) {
    const pw_t y = mpow(to_mont(x, c.M), c.ex, c.M);
    for (u32 j = 0; j < c.r; ++j)
        if (c.om[j] == y) return j;
    return 0xFFFFFFFFu;
}

// exact completion of one candidate; returns packed key (0 on reject) and
// sets *err on an arithmetic failure
__device__ __noinline__ u64 complete_one(const ProfCtx &c, u32 b, u32 d, u32 *err) {
    const pw_t p = c.p;
    // Montgomery d^-1 (= R d^-1), so mmul(b, dinv) = b d^-1 mod p
    const pw_t dinv = mpow(to_mont((pw_t)d, c.M), c.p - 2u, c.M);
    const pw_t xr = mmul((pw_t)b, dinv, c.M);
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
        const bool same = n <= c.B ? colour_at(c, (u32)n + c.OFF) == cb : colour_direct((pw_t)x, c) == A;
        if (!same) break;
        right = k;
    }
    for (u32 k = 1;; ++k) {                            // x = xr - k, numerator b - k d
        if (k > RUN_CAP) { *err = 1; return 0; }
        if (k >= xr) break;
        const pw_t x = xr - k;
        const i64 n = (i64)b - (i64)k * d;
        const bool same = n >= -(i64)c.B ? colour_at(c, (u32)(n + (i64)c.OFF)) == cb : colour_direct(x, c) == A;
        if (!same) break;
        left = k;
    }
    const pw_t s = xr - left, e = xr + right;
    const pw_t w = s < p - e ? s : p - e;             // canonical witness: at most (p - 1) / 2 < 2^32
    return pack_key((u32)(e - s + 1u), (u32)w);
}

// bilateral screen of one word at view index i0 (row step dd = d / G): keep
// bits whose run can still reach t + h, i.e. bits whose right matches rl and
// left matches ll (each counted up to h) satisfy rl + ll >= h; indices outside
// [ilo, ihi] are unknown and match.  The right pass stops once no bit is left
// and records each bit's rl as death events (rl, bits) in registers (a word
// reaching the screen holds few live bits); bits alive after h steps, or at the
// table edge, have rl = h and are kept.  The left pass keeps an event's bits
// that are still alive after h - rl left steps.  Past EV events the newest is
// merged into the last slot with the larger rl, which only keeps more bits.
template <int NPP>
__device__ __noinline__ u32 screen_word(const View &v, u32 i0, u32 alive, u32 dd, u32 t, u32 h) {
    if (h >= 64u) return alive;
    constexpr int EV = 4;
    const u32 u0 = i0 + v.OFF;
    u32 base[NPP];
    Planes<NPP>::win(v.P, u0, base);
    u32 erl[EV], em[EV];
#pragma unroll
    for (int e = 0; e < EV; ++e) { erl[e] = 0xFFFFFFFFu; em[e] = 0u; }
    int ne = 0;
    u32 cur = alive;
    for (u32 k = 1; k <= h && cur; ++k) {
        const i64 lim = (i64)v.ihi - (i64)(i32)i0 - (i64)k * dd;     // bits <= lim known
        if (lim < 0) break;                                          // the rest match: rl = h
        const u32 m = mismatch<NPP>(v.P, u0 + k * dd, base);
        const u32 known = lim >= 31 ? 0xFFFFFFFFu : ((2u << (u32)lim) - 1u);
        const u32 died = cur & m & known;
        if (died) {
            cur &= ~died;
            if (ne < EV) {
#pragma unroll
                for (int e = 0; e < EV; ++e)
                    if (e == ne) { erl[e] = k - 1u; em[e] = died; }
                ++ne;
            } else {
                erl[EV - 1] = k - 1u;
                em[EV - 1] |= died;
            }
        }
    }
    u32 kept = cur;                       // rl = h
    u32 pend = alive & ~kept;             // bits still needing left matches
    u32 lcur = alive;
    for (u32 k = 1; k <= h && (lcur & pend); ++k) {
        const i64 low = (i64)v.ilo - (i64)(i32)i0 + (i64)(t - 1u + k) * dd;   // bits >= low known
        if (low >= 32) { kept |= lcur & pend; break; }               // the rest match
        const u32 m = mismatch<NPP>(v.P, u0 - (t - 1u + k) * dd, base);
        const u32 known = low <= 0 ? 0xFFFFFFFFu : ~((1u << (u32)low) - 1u);
        lcur &= ~(m & known);
#pragma unroll
        for (int e = 0; e < EV; ++e)
            if (erl[e] + k == h) kept |= em[e] & lcur;
        pend &= ~kept;
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
__device__ __forceinline__ void screen_batch(const ProfCtx &c, QEnt *sb, Cand *cb, WarpQ &q, u32 count,
                                             bool screen, ProfState *st, int lane) {
    u32 keep = 0, i0 = 0, d = 0, vc = 0, vg = 1;
    const u32 thr = threshold(c, st);
    if ((u32)lane < count) {
        const QEnt e = sb[lane];
        i0 = e.i0;
        keep = e.alive;
        d = e.dt >> 8;
        const u32 t = e.dt & 0xFFu;
        const View &v = (d & 1u) ? c.base : c.odd;
        vc = v.c;
        vg = v.G;
        const u32 h = thr > t ? thr - t : 0u;     // reject runs certified < threshold
        if (screen && h > 0u) keep = screen_word<NPP>(v, i0, keep, d >> v.gs, t, h);
    }
    __syncwarp();
    // shift the rest down (up to SCR_CAP - 32 entries; each lane moves its own
    // entries in order, so no lane overwrites one another lane still reads)
    for (u32 i = (u32)lane; i + count < q.nscr; i += 32u) sb[i] = sb[count + i];
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


// queue one 32-bit word per lane for the batched screen; the caller runs
// the screen once 32 are waiting (the buffer holds SCR_CAP)
__device__ __forceinline__ void queue_append(QEnt *sb, WarpQ &q, u32 i0, u32 alive, u32 d, u32 t, int lane) {
    const bool has = alive != 0u;
    const u32 bal = __ballot_sync(0xFFFFFFFFu, has);
    if (!bal) return;
    const u32 pos = __popc(bal & ((1u << lane) - 1u));
    if (has) sb[q.nscr + pos] = QEnt{i0, alive, (d << 8) | t};
    q.nscr += __popc(bal);
    __syncwarp();
}

// ---- shared-memory tile: addresses, loads, bulk copy, mbarrier -------------

__device__ __forceinline__ u32 smem_addr(const void *p) { return (u32)__cvta_generic_to_shared(p); }

// plain shared-memory loads at a shared-window byte address
__device__ __forceinline__ u32 lds32(u32 a) {
    u32 v;
    asm volatile("ld.shared.u32 %0, [%1];" : "=r"(v) : "r"(a));
    return v;
}
__device__ __forceinline__ uint2 lds64(u32 a) {
    uint2 v;
    asm volatile("ld.shared.v2.u32 {%0, %1}, [%2];" : "=r"(v.x), "=r"(v.y) : "r"(a));
    return v;
}
__device__ __forceinline__ uint4 lds128(u32 a) {
    uint4 v;
    asm volatile("ld.shared.v4.u32 {%0, %1, %2, %3}, [%4];" : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w) : "r"(a));
    return v;
}

__device__ __forceinline__ void mbar_init(u32 mbar, u32 count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(mbar), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
// one arrival that also announces `bytes` of transaction to come
__device__ __forceinline__ void mbar_expect_tx(u32 mbar, u32 bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" :: "r"(mbar), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(u32 mbar, u32 parity) {
    u32 ok;
    asm volatile("{\n\t.reg .pred P;\n\tmbarrier.try_wait.parity.shared::cta.b64 P, [%1], %2;\n\tselp.u32 %0, 1, 0, P;\n}"
                 : "=r"(ok) : "r"(mbar), "r"(parity) : "memory");
    return ok != 0u;
}
// bounded wait for phase `parity` of the tile barrier; false when the limit ran out
__device__ __forceinline__ bool mbar_wait_bounded(u32 mbar, u32 parity) {
    for (u32 i = 0; i < MBAR_SPIN_LIMIT; ++i)
        if (mbar_try_wait(mbar, parity)) return true;
    return false;
}
// bulk asynchronous copy global -> this CTA's shared memory (no multicast);
// dst, src 16-byte aligned, bytes a multiple of 16
__device__ __forceinline__ void bulk_load(u32 dst, const void *src, u32 bytes, u32 mbar) {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 :: "r"(dst), "l"(src), "r"(bytes), "r"(mbar) : "memory");
}

// three consecutive 32-bit windows of the NPP interleaved planes of a tile at
// shared byte address S (word w of plane k at S + 4 (w NPP + k)): o[c] = bits
// [u + 32 c, u + 32 c + 32), from the four words that hold bits [u, u + 96).
// Lanes holding consecutive lane-words of a band read words three apart: every
// load of a warp is conflict-free at each width (3 l mod 32, mod 16 and mod 8
// are distinct over the lanes that share a wavefront), and the four loads of
// a window give 96 anchors.
template <int NPP> struct Tile;
template <> struct Tile<1> {
    static __device__ __forceinline__ void win3(u32 S, u32 u, u32 (*o)[1]) {
        const u32 a = S + 4u * (u >> 5);
        const u32 p0 = lds32(a), p1 = lds32(a + 4u), p2 = lds32(a + 8u), p3 = lds32(a + 12u);
        o[0][0] = __funnelshift_r(p0, p1, u);
        o[1][0] = __funnelshift_r(p1, p2, u);
        o[2][0] = __funnelshift_r(p2, p3, u);
    }
};
template <> struct Tile<2> {
    static __device__ __forceinline__ void win3(u32 S, u32 u, u32 (*o)[2]) {
        const u32 a = S + 8u * (u >> 5);
        const uint2 p0 = lds64(a), p1 = lds64(a + 8u), p2 = lds64(a + 16u), p3 = lds64(a + 24u);
        o[0][0] = __funnelshift_r(p0.x, p1.x, u); o[0][1] = __funnelshift_r(p0.y, p1.y, u);
        o[1][0] = __funnelshift_r(p1.x, p2.x, u); o[1][1] = __funnelshift_r(p1.y, p2.y, u);
        o[2][0] = __funnelshift_r(p2.x, p3.x, u); o[2][1] = __funnelshift_r(p2.y, p3.y, u);
    }
};
template <> struct Tile<4> {
    static __device__ __forceinline__ void win3(u32 S, u32 u, u32 (*o)[4]) {
        const u32 a = S + 16u * (u >> 5);
        const uint4 p0 = lds128(a), p1 = lds128(a + 16u), p2 = lds128(a + 32u), p3 = lds128(a + 48u);
        o[0][0] = __funnelshift_r(p0.x, p1.x, u); o[0][1] = __funnelshift_r(p0.y, p1.y, u);
        o[0][2] = __funnelshift_r(p0.z, p1.z, u); o[0][3] = __funnelshift_r(p0.w, p1.w, u);
        o[1][0] = __funnelshift_r(p1.x, p2.x, u); o[1][1] = __funnelshift_r(p1.y, p2.y, u);
        o[1][2] = __funnelshift_r(p1.z, p2.z, u); o[1][3] = __funnelshift_r(p1.w, p2.w, u);
        o[2][0] = __funnelshift_r(p2.x, p3.x, u); o[2][1] = __funnelshift_r(p2.y, p3.y, u);
        o[2][2] = __funnelshift_r(p2.z, p3.z, u); o[2][3] = __funnelshift_r(p2.w, p3.w, u);
    }
};

// kill the anchors of the three words whose stage window at u differs from
// their base windows in any plane
template <int NPP>
__device__ __forceinline__ void mismatch3(u32 S, u32 u, const u32 (*b)[NPP], u32 *alive) {
    u32 w[3][NPP];
    Tile<NPP>::win3(S, u, w);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        u32 m = 0;
#pragma unroll
        for (int k = 0; k < NPP; ++k) m |= w[c][k] ^ b[c][k];
        alive[c] &= ~m;
    }
}

// one work item as staged in shared memory
struct Item {
    u32 S;             // shared byte address of the tile's first word
    u32 ubase;         // view bit held by the tile's first word (32 x first view word)
    u32 T0, T1;        // band starts in [T0, T1) (view indices) belong to this item
    u32 view;          // 0 base (odd d), 1 odd view (even d)
    u32 d0, nrows;     // rows d0, d0 + 2, ... (nrows of them)
    u32 t, s;          // anchor stages, anchor spacing of the epoch
};

// the stage windows of one lane-word: its 96 anchors at tile bits [u, u + 96)
// compared with the windows at u - j dd, j = 1 .. t - 1, in batches of SB
// issued together.  T > 0 fixes t at compile time: every stage runs (no
// per-window guard, addresses stepped by dd, no early exit -- some lane of a
// warp keeps a live anchor to the last stage almost always, so a per-lane exit
// saves no issue slot).  T = 0 takes t from the item and stops once the word
// is dead.  Returns the stages a word needs, base window included: those of
// the batches begun while it was alive, the same count in both forms.
template <int NPP, int T>
__device__ __forceinline__ u32 run_stages(u32 S, u32 u, u32 dd, u32 t, u32 *alive) {
    constexpr int SB = NPP == 4 ? CZ_SB4 : (NPP == 2 ? CZ_SB2 : CZ_SB1);
    u32 b[3][NPP];
    Tile<NPP>::win3(S, u, b);
    if constexpr (T > 0) {
        u32 uj = u, nst = 1;
#pragma unroll
        for (int j0 = 1; j0 < T; j0 += SB) {
            if (alive[0] | alive[1] | alive[2]) nst = (u32)(j0 + SB < T ? j0 + SB : T);
#pragma unroll
            for (int k = 0; k < SB; ++k) {
                if (j0 + k < T) {
                    uj -= dd;
                    mismatch3<NPP>(S, uj, b, alive);
                }
            }
        }
        return nst;
    } else {
        u32 j = 1;
        while (j < t && (alive[0] | alive[1] | alive[2])) {
#pragma unroll
            for (int k = 0; k < SB; ++k)
                if (j + (u32)k < t) mismatch3<NPP>(S, u - (j + (u32)k) * dd, b, alive);
            j += SB;
        }
        return min(j, t);
    }
}

// the words of row d whose bands start in the item's tile, every stage window
// read from shared memory.  A band of dd anchors is nw = ceil(dd / 96)
// lane-words of 96 consecutive anchors (three 32-bit words); lanes with
// consecutive ranks hold consecutive lane-words.  A lane's rank (k, w)
// advances by 32 per pass, stepped incrementally from one division per row.
// Survivors are only queued here; when 32 words wait for the screen the
// loop stops at rank `base` and returns false, so the caller screens them with
// none of this loop's state live and then resumes the row (true: the row is
// done)
template <int NPP, int T>
__device__ __forceinline__ bool filter_row_tile(const View &v, const Item &it, u32 d, u32 &base, QEnt *sb,
                                                WarpQ &q, int lane, u32 np) {
    const u32 G = v.G, dd = d >> v.gs, t = T > 0 ? (u32)T : it.t;
    const u32 beta = ((t - 1u) * d + 1u) >> 1;
    const u32 istart = (beta >= v.c ? beta - v.c + G - 1u : 0u) >> v.gs;
    if ((i32)istart > v.ihi || istart >= it.T1) return true;
    const u32 step = dd * it.s;
    const float rstep = __frcp_rn(__uint2float_rn(step));
    const u32 K = div_rcp((u32)v.ihi - istart, step, rstep) + 1u;
    const u32 klo = it.T0 > istart ? div_rcp(it.T0 - istart + step - 1u, step, rstep) : 0u;
    const u32 khi = min(K, div_rcp(it.T1 - istart + step - 1u, step, rstep));
    if (klo >= khi) return true;
    const u32 nw = div_rcp(dd + 95u, 96u, 1.0f / 96.0f);   // lane-words per band
    const u32 W = (khi - klo) * nw;
    if (base >= W) return true;
    // rank = base + lane -> (k, i) = (rank / nw, rank % nw); a pass adds
    // 32 = q32 nw + r32 ranks
    const u32 r0 = base + (u32)lane;
    const float rnw = __frcp_rn(__uint2float_rn(nw));
    u32 k = div_rcp(r0, nw, rnw), i = r0 - k * nw;
    const u32 q32 = div_rcp(32u, nw, rnw), r32 = 32u - q32 * nw;
    u32 i0 = istart + (klo + k) * step + 96u * i;          // view index of the lane-word's first anchor
    const u32 dA = q32 * step + 96u * r32, dB = step - 96u * nw;
    const u32 ubias = v.OFF - it.ubase;
    const u32 S = it.S;
    const i32 ihi = v.ihi;
    auto mask32 = [](i32 len) { return len >= 32 ? 0xFFFFFFFFu : (len <= 0 ? 0u : ((1u << len) - 1u)); };
    while (base < W) {
        const u32 rank = base + (u32)lane;
        base += 32u;
        u32 alive[3] = {0u, 0u, 0u};
        const u32 ia = i0;
        if (rank < W) {
            // anchors of the word: the band's remaining length, and the view's end
            const i32 len = min((i32)(dd - 96u * i), ihi - (i32)ia + 1);
            alive[0] = mask32(len);
            alive[1] = mask32(len - 32);
            alive[2] = mask32(len - 64);
        }
        i += r32;
        const bool wrap = i >= nw;
        if (wrap) i -= nw;
        i0 += wrap ? dA + dB : dA;
        if (alive[0]) {
            // algorithmic tests: stage x plane comparisons of the 32-bit words
            // that hold anchors of the band (one to three per lane-word), over
            // the order's np planes (r = 5..8 also compare a fourth stored
            // plane, all zero, which is not counted)
            const u32 live = 1u + (alive[1] != 0u) + (alive[2] != 0u);
            ++q.words;
            q.tests += live * np * run_stages<NPP, T>(S, ia + ubias, dd, t, alive);
        }
        queue_append(sb, q, ia, alive[0], d, t, lane);
        queue_append(sb, q, ia + 32u, alive[1], d, t, lane);
        queue_append(sb, q, ia + 64u, alive[2], d, t, lane);
        if (q.nscr >= 32u) return base >= W;
    }
    return true;
}

// the rows of the staged item, claimed one per warp from a shared counter
template <int NPP>
__device__ __forceinline__ void filter_item(const ProfCtx &c, const Item &it, const SparseArgs &a, u32 *row_ctr,
                                            QEnt *sb, Cand *cb, WarpQ &q, ProfState *st, int lane) {
    const bool screen = a.tune.screen != 0u;
    for (;;) {
        u32 r = 0;
        if (lane == 0) r = atomicAdd(row_ctr, 1u);
        r = __shfl_sync(0xFFFFFFFFu, r, 0);
        if (r >= it.nrows) break;
        const u32 d = it.d0 + 2u * r;
        const View &v = it.view ? c.odd : c.base;
        u32 base = 0;
        for (;;) {
            // the anchor stage counts CZ_TS* (the default tuning's) run with t fixed at compile time
            bool done;
            if constexpr (NPP == 1) {
                done = it.t == CZ_TS1 ? filter_row_tile<1, CZ_TS1>(v, it, d, base, sb, q, lane, c.np)
                                      : filter_row_tile<1, 0>(v, it, d, base, sb, q, lane, c.np);
            } else if constexpr (NPP == 2) {
                done = it.t == CZ_TS2A ? filter_row_tile<2, CZ_TS2A>(v, it, d, base, sb, q, lane, c.np)
                     : it.t == CZ_TS2B ? filter_row_tile<2, CZ_TS2B>(v, it, d, base, sb, q, lane, c.np)
                                       : filter_row_tile<2, 0>(v, it, d, base, sb, q, lane, c.np);
            } else {
                done = it.t == CZ_TS4A ? filter_row_tile<4, CZ_TS4A>(v, it, d, base, sb, q, lane, c.np)
                     : it.t == CZ_TS4B ? filter_row_tile<4, CZ_TS4B>(v, it, d, base, sb, q, lane, c.np)
                                       : filter_row_tile<4, 0>(v, it, d, base, sb, q, lane, c.np);
            }
            while (q.nscr >= 32u) screen_batch<NPP>(c, sb, cb, q, 32u, screen, st, lane);
            if (done) break;
            asm volatile("" ::: "memory");            // row state is recomputed, not kept across the screen
        }
    }
}

// tiling of a profile: per view, the span of anchor indices one tile holds
// (its words plus the left halo of tmax - 1 row steps, the right halo of one
// band and the window's two extra words fit TILE_WORDS / NPP words), tiles per
// epoch, epochs and items; false if a view cannot be tiled
__device__ inline bool plan_tiles(ProfCtx &c, u32 epoch_rows) {
    const u32 cap_bits = 32u * (TILE_WORDS / c.npp - 16u);
    for (u32 v = 0; v < 2; ++v) {
        const u32 G = v ? 2u : 1u;
        const u32 ddmax = (c.D + G - 1u) / G;
        const u64 halo = (u64)c.tmax * ddmax + 320u;
        if (halo + 1024u > cap_bits) return false;
        const u32 span = ((cap_bits - (u32)halo) / 64u) * 64u;
        const i32 ihi = v ? c.odd.ihi : c.base.ihi;
        const u32 extent = ihi >= 0 ? (u32)ihi + 1u : 0u;       // anchor band starts lie in [0, ihi]
        c.nt[v] = (extent + span - 1u) / span;
        c.ts[v] = c.nt[v] ? ((extent + c.nt[v] - 1u) / c.nt[v] + 63u) / 64u * 64u : span;
    }
    c.nepoch = (c.D + epoch_rows - 1u) / epoch_rows;
    c.nitems = c.nepoch * (c.nt[0] + c.nt[1]);
    return true;
}

// claim the next work item of profile st (thread 0): a 64-bit state holds the
// next item (low 32 bits), and the epoch (bits 32..47, + 1) and threshold
// (bits 48..55) fixed by the first claim of the current epoch
__device__ inline bool claim_item(const ProfCtx &c, ProfState *st, u32 &item, u32 &qe) {
    unsigned long long old = *(volatile unsigned long long *)&st->claim;
    const u32 ipe = c.nt[0] + c.nt[1];
    for (int guard = 0; guard < 1 << 20; ++guard) {
        item = (u32)old;
        if (item >= c.nitems) return false;
        const u32 e = item / ipe;
        unsigned long long nw;
        if ((u32)((old >> 32) & 0xFFFFu) == e + 1u) {
            qe = (u32)((old >> 48) & 0xFFu);
            nw = old + 1ull;
        } else {
            const u32 thr = threshold(c, st);
            qe = thr < c.Q ? thr : c.Q;
            nw = ((unsigned long long)qe << 48) | ((unsigned long long)(e + 1u) << 32) | (item + 1u);
        }
        const unsigned long long prev = atomicCAS(&st->claim, old, nw);
        if (prev == old) return true;
        old = prev;
    }
    return false;
}

// hand out no further item of the profile (after an error: its record is
// refused, and the serving runtime must still see the profile finish)
__device__ inline void exhaust_claims(const ProfCtx &c, ProfState *st) {
    unsigned long long old = *(volatile unsigned long long *)&st->claim;
    for (int guard = 0; guard < 1 << 20 && (u32)old < c.nitems; ++guard) {
        const unsigned long long prev = atomicCAS(&st->claim, old, (old & ~0xFFFFFFFFull) | c.nitems);
        if (prev == old) break;
        old = prev;
    }
}

// serving: a CTA leaves profile g; the last one to leave a profile whose items
// are all handed out writes its record (once) and counts its request down
__device__ __noinline__ void leave_profile(const SparseArgs &a, const ProfCtx &c, u32 g) {
    ProfState *st = a.state + g;
    __threadfence();
    const u32 left = atomicSub(&st->active, 1u) - 1u;
    const u32 claimed = (u32)*(volatile unsigned long long *)&st->claim;
    if (left != 0u || claimed < c.nitems || atomicCAS(&st->done, 0u, 1u) != 0u) return;
    finalize_one(a.primes, a.profs, a.state, nullptr, g, a.verify, a.out);
    __threadfence();
    const u32 req = a.profs[g].req;
    if (atomicSub(&a.req_pending[req], 1u) == 1u) {
        __threadfence_system();
        a.req_done[req] = 1u;
    }
}

// thread 0: claim the profile's next work item, describe it in *out and start
// the bulk copy of its tile into shared memory; false when the profile has no
// item left (or on an error, reported in *err: 2 threshold below 3, 4 tile)
__device__ __noinline__ bool next_item(const ProfCtx &c, ProfState *st, u32 erows, u32 tile, u32 mbar, Item *out,
                                       u32 *err, const volatile u32 *yield) {
    u32 item = 0, qe = 0;
    if (yield && *yield) { *err |= 8u; return false; }
    if (!claim_item(c, st, item, qe)) return false;
    if (qe < 3u) { *err |= 2u; exhaust_claims(c, st); return false; }
    Item it;
    const u32 ipe = c.nt[0] + c.nt[1], e = item / ipe, j = item - e * ipe;
    it.view = j < c.nt[0] ? 0u : 1u;
    const u32 k = it.view ? j - c.nt[0] : j;
    const View &v = it.view ? c.odd : c.base;
    const u32 G = v.G;
    it.T0 = k * c.ts[it.view];
    it.T1 = min(it.T0 + c.ts[it.view], (u32)v.ihi + 1u);
    it.t = c.tpref < qe ? c.tmax : qe;
    it.s = qe - it.t + 1u;
    // rows of the epoch with the view's parity: d odd (base), d even (odd view)
    const u32 dlo = e * erows + 1u, dhi = min(c.D, (e + 1u) * erows);
    it.d0 = (dlo & 1u) == (it.view ? 0u : 1u) ? dlo : dlo + 1u;
    it.nrows = it.d0 <= dhi ? (dhi - it.d0) / 2u + 1u : 0u;
    const u32 ddmax = dhi / G;
    // view words the item reads: left halo (t - 1) row steps, right halo one band + window
    const i64 lob = (i64)it.T0 + v.OFF - (i64)(it.t - 1u) * ddmax - 32;
    const u64 hib = (u64)it.T1 + v.OFF + ddmax + 128u;
    const u32 nwv = it.view ? c.NW2 : c.NW;
    const u32 w0 = lob > 0 ? (u32)(lob >> 5) & ~3u : 0u;
    const u64 w1r = ((hib >> 5) + 4u) & ~3ull;
    u32 w1 = w1r < (u64)nwv ? (u32)w1r : nwv;
    if (w1 < w0 + 4u) w1 = min(nwv, w0 + 4u);
    const u32 bytes = (w1 - w0) * c.npp * 4u;
    if (bytes > TILE_WORDS * 4u || w1 <= w0) { *err |= 4u; exhaust_claims(c, st); return false; }
    it.S = tile;
    it.ubase = 32u * w0;
    *out = it;
    atomicAdd(&st->staged16, bytes >> 4);
    mbar_expect_tx(mbar, bytes);
    bulk_load(tile, v.P + (size_t)w0 * c.npp, bytes, mbar);
    return true;
}

// thread 0: the per-profile constants of global profile gprof, and its tiling
__device__ __noinline__ void load_profile(const SparseArgs &a, u32 gprof, ProfCtx *out, u32 *err) {
    const ProfDesc PD = a.profs[gprof];
    const PrimeDesc PR = a.primes[PD.prime];
    ProfCtx c;
    c.p = PR.p; c.r = PD.r; c.np = PD.np; c.npp = PD.npp; c.Q = PD.Q; c.D = PD.D; c.B = PR.B;
    c.NW = PR.nwords; c.NW2 = PR.nwords2; c.OFF = 32u * PR.K0 + 31u; c.ex = (PR.p - 1u) / PD.r;
    c.M = Mont{PR.p, PR.ninv, PR.one, PR.r2};
    c.P = a.planes + PD.plane_off;
    c.base = View{c.P, c.OFF, -(i32)PR.B, (i32)PR.B, 1u, 0u, 0u};
    // odd view: n = 2i + 1 in [-B, B]  <=>  i in [ceil((-B-1)/2), floor((B-1)/2)]
    c.odd = View{c.P + (size_t)PR.nwords * PD.npp, 32u * PR.K2, -(i32)((PR.B + 1u) / 2u), (i32)((PR.B - 1u) / 2u),
                 2u, 1u, 1u};
    for (int j = 0; j < 9; ++j) c.om[j] = PD.omega[j];
    c.seed = *(volatile u32 *)&a.state[gprof].seed;
    c.qspec = PD.qspec;
    c.tpref = PD.tpref;
    c.tmax = c.tpref < 2u ? 2u : c.tpref;
    if (!plan_tiles(c, a.epoch_rows ? a.epoch_rows : EPOCH_ROWS_DEFAULT)) { c.nitems = 0; *err |= 4u; }
    if (PR.status & ST_ROOT) c.nitems = 0;     // setup found no root (a non-prime): no work, its record is refused
    *out = c;
}

__global__ void __launch_bounds__(SPARSE_WARPS * 32, CZ_SPARSE_MINB)
sparse_kernel(SparseArgs a) {
    extern __shared__ __align__(128) uint4 s_tile[];   // TILE_WORDS words
    __shared__ unsigned long long s_mbar;
    __shared__ u32 s_item, s_err, s_row, s_has, s_phase;
    __shared__ Cand cbuf[SPARSE_WARPS][CAND_CAP];      // candidates awaiting completion
    __shared__ QEnt sbuf[SPARSE_WARPS][SCR_CAP];       // words awaiting the screen
    __shared__ ProfCtx s_ctx;
    __shared__ Item s_it;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        mbar_init(smem_addr(&s_mbar), 1u);
        s_phase = 0u;                                  // tile copies completed so far
    }
    __syncthreads();
    for (;;) {
        if (threadIdx.x == 0) {
            // a.group consecutive CTA slots share one profile
            s_item = (a.yield && *a.yield) ? a.nlist : atomicAdd(a.next, 1u) / a.group;
            s_err = 0u;
            if (s_item < a.nlist) {
                load_profile(a, a.prof_list[s_item], &s_ctx, &s_err);
                if (a.out) atomicAdd(&a.state[a.prof_list[s_item]].active, 1u);
                if (s_err & 4u) exhaust_claims(s_ctx, a.state + a.prof_list[s_item]);
            }
        }
        __syncthreads();
        const u32 pitem = s_item;
        if (pitem >= a.nlist) return;
        const ProfCtx &c = s_ctx;
        ProfState *st = a.state + a.prof_list[pitem];
        WarpQ q{0, 0, 0, 0, 0, 0, 0};
        QEnt *sb = sbuf[warp];
        Cand *cb = cbuf[warp];
        for (;;) {
            if (threadIdx.x == 0) {
                u32 err = 0;
                s_has = next_item(c, st, a.epoch_rows ? a.epoch_rows : EPOCH_ROWS_DEFAULT, smem_addr(s_tile),
                                  smem_addr(&s_mbar), &s_it, &err, a.yield) ? 1u : 0u;
                s_err |= err;
                s_row = 0u;
            }
            __syncthreads();
            if (!s_has) break;
            // wait for the tile copy (bounded); the verdict is made CTA-uniform
            const u32 par = s_phase & 1u;
            const bool ok = __syncthreads_and(mbar_wait_bounded(smem_addr(&s_mbar), par) ? 1 : 0) != 0;
            if (!ok) {
                if (threadIdx.x == 0) atomicOr(&st->status, ST_QUEUE);
                mbar_wait_bounded(smem_addr(&s_mbar), par);    // let the copy land before leaving
                return;
            }
            const Item &it = s_it;
            if (c.npp == 1u) filter_item<1>(c, it, a, &s_row, sb, cb, q, st, lane);
            else if (c.npp == 2u) filter_item<2>(c, it, a, &s_row, sb, cb, q, st, lane);
            else filter_item<4>(c, it, a, &s_row, sb, cb, q, st, lane);
            if (threadIdx.x == 0) s_phase += 1u;
            __syncthreads();                               // the tile is free for the next copy
        }
        // the screen queue carries across rows and items: drain it, then the candidates
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
        const u32 errs = s_err & 7u, yielded = s_err & 8u;
        if (threadIdx.x == 0) {
            if (errs) atomicOr(&st->status, (errs & 2u) ? ST_SEED : ((errs & 4u) ? ST_COVER : ST_QUEUE));
            if (a.out) leave_profile(a, c, a.prof_list[pitem]);
        }
        if (yielded) return;
    }
}

}  // namespace CZ_NS
