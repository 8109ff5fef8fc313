// sparse.cuh -- certified rational-anchor filter with exact completion.
//
// Mathematics (the reference's GPU method, paper/GPU_METHOD_EN.tex:256-560):
//  * Cover (Thm "integer coverage certificate"; P/src/clipped_cover.hpp:7-21):
//    with H = Q-1, B < p, D < p, H*D <= 2B and 4BD - H D^2 > 4p, every window
//    x..x+H of [1, p-1] has numerators a+jd (a = dx mod p, 1 <= d <= D) all in
//    [-B, B]; colour(x+j) = colour(a+jd) - colour(d), so colour constancy of
//    the window is read off the signed table.
//  * A run of length >= q (q <= Q) contains a q-window; it holds s = q-t+1
//    anchors of length t along its row.  Writing an anchor by its top
//    numerator b (numerators b, b-d, ..., b-(t-1)d) and v = b - ceil((t-1)d/2),
//    this build selects b iff v mod (d*s) < d: every s consecutive anchors of a
//    row contain exactly one selected b, and the rule is symmetric under the
//    reflection b -> (t-1)d - b (colours shift by colour(-1), positions x ->
//    p-x, canonical witness unchanged), so only v >= 0 is enumerated
//    (the role of the reference's folded bands and phase rule,
//    P/src/periodic_bands.hpp:28-78; this rule keeps whole bands of d
//    consecutive b, so each 32-bit word is full).
//  * Filter (PBV/src/wheel_filter.hpp:52-91): 32 anchors per word; a candidate
//    survives while every anchor offset agrees with b on every colour plane.
//  * Bilateral screen (B1/src/two_cuts.hpp:27-74): reject only when known
//    mismatches on both sides bound the run below the threshold; numerators
//    outside [-B, B] are unknown and never reject.
//  * Exact completion (PBV/src/completion.hpp:17-57, E32/src/completion_core.hpp:17-48):
//    x = b/d mod p, extend both ways with table colours, falling back to a
//    direct power outside the table; reduce by (length, least witness) with a
//    packed 64-bit atomicMax.
//  * Exactness (Thm "exactness on successful termination"): every row d is
//    processed with a fixed q <= (a verified run length) <= M, so every maximum
//    run (or its reflection) is completed.
//
// B200 design: one persistent kernel; a CTA owns one (p, r) profile at a time
// (its planes stay hot in that SM's L1 and in L2), its warps pull rows d in
// increasing order from a shared-memory counter and re-read the verified
// maximum at every row, so the threshold rises while the profile runs; lanes
// take consecutive words of a row (coalesced plane reads, funnel-shift
// windows); survivors go to a per-warp shared-memory buffer and are completed
// 32 at a time, one per lane.
#pragma once
#include "labels.cuh"

namespace cz {

constexpr int SPARSE_WARPS = 16;
constexpr int CAND_CAP = 64;          // per-warp candidate buffer
constexpr u32 RUN_CAP = 4096;         // longest run a completion may walk (M <= 46 below 2^32 in practice)

struct Tuning {
    u32 anchor_bits;   // t chosen so 32 * r^-(t-1) <= 2^-anchor_bits per word
    u32 screen;        // 1: bilateral screen on
};

struct SparseArgs {
    const PrimeDesc *primes;
    const ProfDesc *profs;
    ProfState *state;
    const u32 *planes;
    const u32 *prof_list;     // global profile indices (sparse-routed)
    u32 nlist;
    u32 *next;                // work counter (profiles handed out)
    Tuning tune;
};

struct Cand { u32 b, d, dinv; };

__device__ __forceinline__ u32 win(const u32 *__restrict__ P, u32 u) {
    const u32 w = u >> 5;
    return __funnelshift_r(__ldg(P + w), __ldg(P + w + 1), u & 31u);
}

// preferred anchor length: least t with r^(t-1) >= 2^(5+bits), i.e. a word of
// 32 random anchors keeps on average <= 2^-bits survivors
__device__ __forceinline__ u32 anchor_pref(u32 r, u32 bits) {
    const u64 goal = u64(1) << (5u + bits);
    u64 pw = 1;
    u32 k = 0;
    while (pw < goal) { pw *= r; ++k; }
    return k + 1u;
}

// colour of numerator n (|n| <= B) as an integer, np planes of NW words
__device__ __forceinline__ u32 colour_at(const u32 *__restrict__ P, u32 NW, u32 np, u32 u) {
    u32 c = 0;
    for (u32 k = 0; k < np; ++k) c |= ((__ldg(P + (size_t)k * NW + (u >> 5)) >> (u & 31u)) & 1u) << k;
    return c;
}

// absolute colour of x in [1, p-1] by a direct power: x^((p-1)/r) = omega^j
__device__ __forceinline__ u32 colour_direct(u32 x, const Mont &M, u32 ex, const u32 *om, u32 r) {
    const u32 y = mpow(to_mont(x, M), ex, M);
    for (u32 j = 0; j < r; ++j)
        if (om[j] == y) return j;
    return 0xFFFFFFFFu;
}

struct ProfCtx {
    u32 p, r, np, Q, D, B, NW, OFF, ex;
    Mont M;
    const u32 *P;          // plane 0
    u32 om[9];
};

// exact completion of one candidate; returns packed key (0 on reject) and
// sets *err on an arithmetic failure
__device__ __noinline__ u64 complete_one(const ProfCtx &c, u32 b, u32 d, u32 dinv, u32 *err) {
    const u32 p = c.p;
    const u32 xr = mmul(b, dinv, c.M);                 // b * d^-1 mod p (dinv in Montgomery form)
    if (xr == 0u) return 0;
    const u32 cb = colour_at(c.P, c.NW, c.np, b + c.OFF);
    const u32 cd = colour_at(c.P, c.NW, c.np, d + c.OFF);
    const u32 A = cb >= cd ? cb - cd : cb + c.r - cd;  // absolute colour of x_R
    u32 right = 0, left = 0;
    // extend right: x = xr + k, numerator b + k d
    for (u32 k = 1;; ++k) {
        if (k > RUN_CAP) { *err = 1; return 0; }
        const u64 x = (u64)xr + k;
        if (x >= p) break;
        const u64 n = (u64)b + (u64)k * d;
        bool same;
        if (n <= c.B) same = colour_at(c.P, c.NW, c.np, (u32)n + c.OFF) == cb;
        else same = colour_direct((u32)x, c.M, c.ex, c.om, c.r) == A;
        if (!same) break;
        right = k;
    }
    // extend left: x = xr - k, numerator b - k d
    for (u32 k = 1;; ++k) {
        if (k > RUN_CAP) { *err = 1; return 0; }
        if (k >= xr) break;                            // x would reach 0
        const u32 x = xr - k;
        const i64 n = (i64)b - (i64)k * d;
        bool same;
        if (n >= -(i64)c.B) same = colour_at(c.P, c.NW, c.np, (u32)(n + (i64)c.OFF)) == cb;
        else same = colour_direct(x, c.M, c.ex, c.om, c.r) == A;
        if (!same) break;
        left = k;
    }
    const u32 s = xr - left, e = xr + right;
    const u32 len = e - s + 1u;
    const u32 w = s < p - e ? s : p - e;
    return pack_key(len, w);
}

// window of plane k at bit index u (planes are NW words apart)
__device__ __forceinline__ u32 winp(const u32 *__restrict__ P, u32 k, u32 NW, u32 u) {
    return win(P + (size_t)k * NW, u);
}

// bilateral screen of one word: keep bits whose run can still reach Ts
// (right matches + left matches >= Ts - t); unknown numerators match
__device__ __noinline__ u32 screen_word(const ProfCtx &c, const u32 *base_w, u32 b0, u32 alive, u32 d, u32 t, u32 h) {
    if (h >= 64u) return alive;
    const u32 u0 = b0 + c.OFF;
    u32 R[64];
    u32 cur = alive;
    bool unk = false;
    R[0] = cur;
    for (u32 k3 = 1; k3 <= h; ++k3) {
        if (cur && !unk) {
            const i64 lim = (i64)c.B - (i64)b0 - (i64)k3 * d;        // bits i <= lim known
            if (lim < 0) unk = true;
            else {
                const u32 u = u0 + k3 * d;
                u32 eq = 0xFFFFFFFFu;
                for (u32 k2 = 0; k2 < c.np; ++k2) eq &= ~(winp(c.P, k2, c.NW, u) ^ base_w[k2]);
                const u32 known = lim >= 31 ? 0xFFFFFFFFu : ((2u << (u32)lim) - 1u);
                cur &= eq | ~known;
            }
        }
        R[k3] = cur;
    }
    u32 lcur = alive, kept = R[h] & alive;
    bool lunk = false;
    for (u32 k3 = 1; k3 <= h && (lcur & ~kept); ++k3) {
        if (!lunk) {
            const i64 low = (i64)(t - 1u + k3) * d - (i64)c.B - (i64)b0;   // bits i >= low known
            if (low >= 32) lunk = true;
            else {
                const u32 u = u0 - (t - 1u + k3) * d;
                u32 eq = 0xFFFFFFFFu;
                for (u32 k2 = 0; k2 < c.np; ++k2) eq &= ~(winp(c.P, k2, c.NW, u) ^ base_w[k2]);
                const u32 known = low <= 0 ? 0xFFFFFFFFu : ~((1u << (u32)low) - 1u);
                lcur &= eq | ~known;
            }
        }
        kept |= R[h - k3] & lcur;
    }
    return kept;
}

__global__ void __launch_bounds__(SPARSE_WARPS * 32, 2)
sparse_kernel(SparseArgs a) {
    __shared__ u32 s_item, s_row;
    __shared__ Cand cbuf[SPARSE_WARPS][CAND_CAP];      // candidates awaiting completion
    __shared__ uint2 sbuf[SPARSE_WARPS][CAND_CAP];     // (b0, alive) words awaiting the screen
    __shared__ u32 s_err;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (;;) {
        if (threadIdx.x == 0) {
            s_item = atomicAdd(a.next, 1u);
            s_row = 1u;
            s_err = 0u;
        }
        __syncthreads();
        const u32 item = s_item;
        if (item >= a.nlist) return;
        const u32 gprof = a.prof_list[item];
        const ProfDesc PD = a.profs[gprof];
        const PrimeDesc PR = a.primes[PD.prime];
        ProfState *st = a.state + gprof;
        ProfCtx c;
        c.p = PR.p; c.r = PD.r; c.np = PD.np; c.Q = PD.Q; c.D = PD.D; c.B = PR.B;
        c.NW = PR.nwords; c.OFF = 32u * PR.K0 + 31u; c.ex = (PR.p - 1u) / PD.r;
        c.M = Mont{PR.p, PR.ninv, PR.one, PR.r2};
        c.P = a.planes + PD.plane_off;
#pragma unroll
        for (int j = 0; j < 9; ++j) c.om[j] = PD.omega[j];
        const u32 *P0 = c.P, *P1 = c.P + c.NW, *P2 = c.P + 2u * (size_t)c.NW, *P3 = c.P + 3u * (size_t)c.NW;
        const u32 np = c.np;
        const u32 seed = *(volatile u32 *)&st->seed;
        const u32 tpref = anchor_pref(c.r, a.tune.anchor_bits);
        u32 ncand = 0, nscr = 0;             // warp-uniform buffer fills
        u64 warp_best = 0;
        u32 words = 0, comps = 0, err = 0;
        u32 tests = 0;
        // complete `count` (<= 32) buffered candidates, one per lane
        auto flush = [&](u32 count) {
            u64 key = 0;
            if ((u32)lane < count) {
                const Cand cd = cbuf[warp][lane];
                u32 e = 0;
                key = complete_one(c, cd.b, cd.d, cd.dinv, &e);
                err |= e;
            }
            comps += count;
            const u32 hi = (u32)(key >> 32);
            const u32 mhi = __reduce_max_sync(0xFFFFFFFFu, hi);
            const u32 lo = __reduce_max_sync(0xFFFFFFFFu, hi == mhi ? (u32)key : 0u);
            const u64 k2 = ((u64)mhi << 32) | lo;
            if (k2 > warp_best) warp_best = k2;
            __syncwarp();
            if (ncand > count && (u32)lane < ncand - count) cbuf[warp][lane] = cbuf[warp][count + lane];
            __syncwarp();
            ncand -= count;
            if (lane == 0 && warp_best) atomicMax(&st->best, (unsigned long long)warp_best);
        };
        for (;;) {
            u32 d = 0;
            if (lane == 0) d = atomicAdd(&s_row, 1u);
            d = __shfl_sync(0xFFFFFFFFu, d, 0);
            if (d > c.D) break;
            // row parameters from the verified maximum so far (<= M)
            const u64 bk = *(volatile unsigned long long *)&st->best;
            const u32 blen = key_len(bk) > seed ? key_len(bk) : seed;
            const u32 q = blen < c.Q ? blen : c.Q;
            if (q < 3u) { err |= 2u; break; }
            const u32 t = tpref < q ? (tpref < 2u ? 2u : tpref) : q;
            const u32 s = q - t + 1u;
            const u32 h = blen > t ? blen - t : 0u;      // screen: reject runs certified < blen
            const u32 beta = ((t - 1u) * d + 1u) >> 1;
            if (beta > c.B) continue;
            const u32 ds = d * s;
            const u32 K = (c.B - beta) / ds + 1u;
            const u32 nw = (d + 31u) >> 5;
            const u32 W = K * nw;
            const float rnw = 1.0f / (float)nw;
            u32 dinv = 0;
            bool have_inv = false;
            // screen the queued words (count <= 32), push survivors to the completion buffer
            auto screen_batch = [&](u32 count) {
                u32 keep = 0, b0 = 0;
                if ((u32)lane < count) {
                    const uint2 e = sbuf[warp][lane];
                    b0 = e.x;
                    keep = e.y;
                    if (a.tune.screen && h > 0u) {
                        const u32 u0 = b0 + c.OFF;
                        u32 bw[4];
                        bw[0] = win(P0, u0);
                        bw[1] = np > 1u ? win(P1, u0) : 0u;
                        bw[2] = np > 2u ? win(P2, u0) : 0u;
                        bw[3] = np > 3u ? win(P3, u0) : 0u;
                        keep = screen_word(c, bw, b0, keep, d, t, h);
                    }
                }
                __syncwarp();
                if (nscr > count && (u32)lane < nscr - count) sbuf[warp][lane] = sbuf[warp][count + lane];
                __syncwarp();
                nscr -= count;
                while (__any_sync(0xFFFFFFFFu, keep != 0u)) {
                    if (!have_inv) {
                        // Montgomery d^-1 (= R d^-1), so mmul(b, dinv) = b d^-1 mod p
                        dinv = mpow(to_mont(d, c.M), c.p - 2u, c.M);
                        have_inv = true;
                    }
                    const bool has = keep != 0u;
                    const u32 bal = __ballot_sync(0xFFFFFFFFu, has);
                    const u32 pos = __popc(bal & ((1u << lane) - 1u));
                    if (has) {
                        const u32 bit = __ffs(keep) - 1u;
                        keep &= keep - 1u;
                        cbuf[warp][ncand + pos] = Cand{b0 + bit, d, dinv};
                    }
                    ncand += __popc(bal);
                    __syncwarp();
                    if (ncand >= 32u) flush(32u);
                }
            };
            for (u32 base = 0; base < W; base += 32u) {
                const u32 rank = base + (u32)lane;
                u32 alive = 0, b0 = 0;
                if (rank < W) {
                    u32 k = (u32)((float)rank * rnw);
                    if (k * nw > rank) --k;
                    else if ((k + 1u) * nw <= rank) ++k;
                    const u32 w = rank - k * nw;
                    b0 = beta + k * ds + 32u * w;
                    u32 len = d - 32u * w;
                    if (len > 32u) len = 32u;
                    if (b0 > c.B) len = 0;
                    else if (c.B - b0 + 1u < len) len = c.B - b0 + 1u;
                    alive = len >= 32u ? 0xFFFFFFFFu : ((1u << len) - 1u);
                }
                if (alive) {
                    ++words;
                    u32 u = b0 + c.OFF;
                    const u32 w0 = win(P0, u);
                    const u32 w1 = np > 1u ? win(P1, u) : 0u;
                    const u32 w2 = np > 2u ? win(P2, u) : 0u;
                    const u32 w3 = np > 3u ? win(P3, u) : 0u;
                    tests += np;                           // base windows
                    for (u32 j = 1; j < t && alive; ++j) {
                        tests += np;
                        u -= d;
                        u32 m = win(P0, u) ^ w0;
                        if (np > 1u) m |= win(P1, u) ^ w1;
                        if (np > 2u) m |= win(P2, u) ^ w2;
                        if (np > 3u) m |= win(P3, u) ^ w3;
                        alive &= ~m;
                    }
                }
                // queue surviving words for the batched screen
                const bool has = alive != 0u;
                const u32 bal = __ballot_sync(0xFFFFFFFFu, has);
                if (bal) {
                    const u32 pos = __popc(bal & ((1u << lane) - 1u));
                    if (has) sbuf[warp][nscr + pos] = make_uint2(b0, alive);
                    nscr += __popc(bal);
                    __syncwarp();
                    if (nscr >= 32u) screen_batch(32u);
                }
            }
            if (nscr) screen_batch(nscr);
        }
        if (ncand) flush(ncand);
        if (err) atomicOr(&s_err, err);
        words = __reduce_add_sync(0xFFFFFFFFu, words);
        tests = __reduce_add_sync(0xFFFFFFFFu, tests);
        if (lane == 0) {
            atomicAdd(&st->words, (unsigned long long)words);
            atomicAdd(&st->completions, (unsigned long long)comps);
            atomicAdd(&st->tests, (unsigned long long)tests);
        }
        __syncthreads();
        if (threadIdx.x == 0 && s_err) atomicOr(&st->status, (s_err & 2u) ? ST_SEED : ST_QUEUE);
    }
}

}  // namespace cz
