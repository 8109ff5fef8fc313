// table.cuh -- signed colour bit-planes for the certified rational-anchor filter.
//
// For a sparse-routed prime p with table radius B, every admissible order r gets
// bit planes of colour_r (written in binary, np = ceil(log2 r) planes, padded to
// NPP in {1, 2, 4} with zero planes) over two views of the signed numerators
// n in [-B, B], with colour_r(-n) = colour_r(n) + colour_r(-1):
//   base view: index i = n, stored at bit u = i + 32*K0 + 31;
//   odd view:  index i with n = 2i + 1 (odd numerators only), bit u = i + 32*K2;
//              rows with an even denominator d only ever meet odd numerators
//              (a primitive pair (b, d) with d even has b odd), so they read
//              this half-size view (the reference's wheel rows for G = 2,
//              src/census/engine32/vendor/research/baseline/baseline/previous/
//              baseline/vendor/src/wheel_filter.hpp:14-46).
// Planes of one profile are interleaved: word w of plane k sits at
// [w * NPP + k], so one (vector) load fetches every plane of a word.
// This replaces the reference's small_table / fine_labels / pack_pair kernels
// (src/census/engine32/src/small_table.cuh:7-52).
//
// B200 design:
//  * labels are computed only for primes q in the table (one Montgomery power
//    each, kept in shared memory); every other n takes its label additively
//    through a prime-power chain n -> n / q^e, q = spf(n) (the colour is a
//    character: label(n) = sum of e label(q)), so a table of ~10^6 entries
//    costs ~6e4 powers, not 10^6, and a walk takes one step per distinct
//    prime factor;
//  * each warp stages 32 consecutive labels per step in shared memory, then
//    emits plane words profile by profile with one ballot per plane bit: the
//    negative half of the base view is one __brev'd ballot (aligned by the
//    +31 centring), the positive half is the previous step's ballot shifted
//    by one with this step's first bit on top; two steps make one odd-view
//    word per sign;
//  * the same pass records the longest monochromatic stretch inside [1, B] of
//    each profile planned without a speculative threshold: a real run length,
//    hence a certified lower bound on M (the role of the reference's
//    seed_runs/finish_seed, small_table.cuh:64-136); a speculated profile is
//    certified by its best run reaching the speculative threshold instead;
//  * the planes of one numerator step are stored with one instruction per
//    word kind, lane b holding plane b.
#pragma once
#include "labels.cuh"

namespace CZ_NS {

constexpr int TABLE_THREADS = 1024;
constexpr int TABLE_WARPS = TABLE_THREADS / 32;
constexpr u32 TABLE_SUB = 8;       // steps staged per warp (even)

struct TableArgs {
    const PrimeDesc *primes;
    const ProfDesc *profs;
    ProfState *state;
    u32 *planes;                 // pool
    const u32 *sparse_primes;    // indices of sparse-routed primes
    u32 nsparse;
    const u32 *small_primes;     // all primes below chain_limit, ascending
    u32 n_small;
    const uint2 *chain;          // chain[n] = (index of q = spf(n) in small_primes | e << 24, n / q^e)
    u32 chain_limit;
};

struct TabProf {            // per-profile constants of the CTA's prime
    u32 r, magic, npp, sig;
    u32 seed;               // 1: track the seed stretch (no speculative threshold)
    u32 *base, *odd;
};

struct TabWarp {            // per-warp, per-profile carried state
    u32 prevw[8][4];        // last base ballot per plane (positive carry)
    u32 stp[8][4], stn[8][4];   // odd-view half words of the even step of a pair
    u32 cc[8], clen[8], best[8];    // seed stretch: last colour, open length, best
};

__global__ void __launch_bounds__(TABLE_THREADS, 1)
table_kernel(TableArgs a) {
    extern __shared__ __align__(16) u32 tsm[];
    __shared__ TabProf tp[8];
    __shared__ unsigned short lab[TABLE_WARPS][TABLE_SUB + 1][32];
    __shared__ TabWarp tw[TABLE_WARPS];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (u32 it = blockIdx.x; it < a.nsparse; it += gridDim.x) {
        const u32 pi = a.sparse_primes[it];
        const PrimeDesc P = a.primes[pi];
        if (P.status & ST_ROOT) continue;   // not a prime, or no root of order m: the filter skips it
        const Mont M{P.p, P.ninv, P.one, P.r2};
        const u32 slots = hash_slots(P.m);
        // shared layout: root hash keys (slots words), their labels (slots u16),
        // 4 u16 of padding, labels of the primes below the table end
        pw_t *keys = reinterpret_cast<pw_t *>(tsm);
        unsigned short *hl = reinterpret_cast<unsigned short *>(keys + slots);
        unsigned short *plab = hl + slots + 4u;
        build_root_hash(keys, hl, slots, M, P.z, P.m);
        const u32 KS = (P.B + 1u + 31u) / 32u + 1u;            // steps: n in [0, 32*KS)
        const u32 nmax = 32u * KS;
        u32 lo = 0, hi = a.n_small;                              // primes below nmax
        while (lo < hi) {
            u32 mid = (lo + hi) >> 1;
            if (a.small_primes[mid] < nmax) lo = mid + 1; else hi = mid;
        }
        const u32 nq = lo;
        u32 bad = (nmax > a.chain_limit) ? 1u : 0u;
        for (u32 i = threadIdx.x; i < nq; i += blockDim.x) {
            const pw_t y = mpow(to_mont((pw_t)a.small_primes[i], M), P.e, M);
            u32 l = lookup_label(keys, hl, slots, y);
            if (l == 0xFFFFu) { bad = 1; l = 0; }
            plab[i] = (unsigned short)l;
        }
        const u32 nprof = P.nprof;
        if (threadIdx.x < nprof) {
            const ProfDesc D = a.profs[P.first_prof + threadIdx.x];
            TabProf t;
            t.r = D.r;
            t.magic = magic_of(D.r);
            t.npp = D.npp;
            t.sig = mod_small(P.sigma, D.r, t.magic);
            // a profile with a speculative threshold is certified by its best
            // run reaching q_spec (else it is re-run unspeculated, seed and
            // all), so its records never depend on the seed; the seed would
            // only raise its starting threshold when a stretch inside [1, B]
            // beat q_spec, which the margins make rare
            t.seed = D.qspec == 0u ? 1u : 0u;
            t.base = a.planes + D.plane_off;
            t.odd = a.planes + D.plane_off + (u64)P.nwords * D.npp;
            tp[threadIdx.x] = t;
        }
        {   // per-warp carried state
            u32 *w = reinterpret_cast<u32 *>(&tw[warp]);
            for (u32 i = lane; i < sizeof(TabWarp) / 4; i += 32) w[i] = 0u;
        }
        __syncthreads();
        if (lane < 8) tw[warp].cc[lane] = 0xFFFFFFFFu;
        const u32 K0 = P.K0, NW = P.nwords, K2 = P.K2, NW2 = P.nwords2;
        // guard words of both views (everything outside the written ranges)
        for (u32 s = 0; s < nprof; ++s) {
            const TabProf t = tp[s];
            for (u32 w = threadIdx.x; w < NW; w += blockDim.x)
                if (w + KS <= K0 || w >= K0 + KS)
                    for (u32 k = 0; k < t.npp; ++k) t.base[(size_t)w * t.npp + k] = 0u;
            const u32 half = (KS + 1u) / 2u;                     // step pairs
            for (u32 w = threadIdx.x; w < NW2; w += blockDim.x)
                if (w + half + 1u <= K2 || w >= K2 + half)
                    for (u32 k = 0; k < t.npp; ++k) t.odd[(size_t)w * t.npp + k] = 0u;
        }
        // warp chunk of steps [k0, k1), k0 even
        u32 per = (KS + TABLE_WARPS - 1) / TABLE_WARPS;
        per = (per + 1u) & ~1u;
        const u32 k0 = min(KS, (u32)warp * per), k1 = min(KS, k0 + per);
        const u32 B = P.B;
        __syncwarp();
        for (u32 ks = k0; ks < k1; ks += TABLE_SUB) {
            const u32 ke = min(k1, ks + TABLE_SUB);
            const bool need_pre = (ks == k0 && k0 > 0);
            // stage labels of steps [ks - need_pre, ke): the TABLE_SUB + 1 chains of
            // a lane are walked in lockstep, so their dependent loads overlap
            {
                const u32 kfirst = ks - (need_pre ? 1u : 0u);
                u32 v[TABLE_SUB + 1], l[TABLE_SUB + 1];
#pragma unroll
                for (u32 i = 0; i <= TABLE_SUB; ++i) {
                    const u32 k = kfirst + i;
                    const u32 n = 32u * k + (u32)lane;
                    v[i] = (k < ke && n >= 2u && n < a.chain_limit) ? n : 1u;
                    l[i] = 0u;
                }
                for (int g = 0; g < 24; ++g) {
                    bool any = false;
#pragma unroll
                    for (u32 i = 0; i <= TABLE_SUB; ++i) {
                        if (v[i] > 1u) {
                            const uint2 c = a.chain[v[i]];
                            l[i] += (c.x >> 24) * plab[c.x & 0xFFFFFFu];   // e label(q): the sum stays <= 20 (m - 1)
                            v[i] = c.y;
                            any = true;
                        }
                    }
                    if (!any) break;
                }
                const u32 mgm = magic_of(P.m);
#pragma unroll
                for (u32 i = 0; i <= TABLE_SUB; ++i) {
                    const u32 k = kfirst + i;
                    if (k >= ke) break;
                    if (v[i] > 1u) bad = 1;
                    lab[warp][k + 1u - ks][lane] = (unsigned short)mod_small(l[i], P.m, mgm);   // slot 0 = pre-step
                }
            }
            __syncwarp();
            for (u32 s = 0; s < nprof; ++s) {
                const TabProf t = tp[s];
                TabWarp &W = tw[warp];
                u32 prevw[4], stp[4], stn[4];
#pragma unroll
                for (int b = 0; b < 4; ++b) { prevw[b] = W.prevw[s][b]; stp[b] = W.stp[s][b]; stn[b] = W.stn[s][b]; }
                u32 cc = W.cc[s], clen = W.clen[s], best = W.best[s];
                if (need_pre) {
                    const u32 c = mod_small(lab[warp][0][lane], t.r, t.magic);
#pragma unroll
                    for (int b = 0; b < 4; ++b)
                        if (b < (int)t.npp) prevw[b] = __ballot_sync(0xFFFFFFFFu, (c >> b) & 1u);
                }
                for (u32 k = ks; k < ke; ++k) {
                    const u32 n = 32u * k + (u32)lane;
                    u32 c = mod_small(lab[warp][k + 1u - ks][lane], t.r, t.magic);
                    u32 cn = c + t.sig;
                    if (cn >= t.r) cn -= t.r;
                    if (n == 0u) { c = 0u; cn = 0u; }
                    // odd numerators of the step (odd lanes): lanes 0..15 take the
                    // colour of lane 2l + 1, lanes 16..31 its reflection, from one
                    // shuffle of the packed pair (colours < 16), so one ballot per
                    // plane gives both odd-view half words
                    const u32 pk = __shfl_sync(0xFFFFFFFFu, c | (cn << 4), 2 * (lane & 15) + 1);
                    const u32 ch = lane < 16 ? (pk & 15u) : (pk >> 4);
                    const bool odd_step = (k & 1u) != 0u;
                    // lane b collects plane b's words; one store per word kind
                    // then writes the interleaved planes of a word together
                    u32 vneg = 0u, vpos = 0u, vop = 0u, von = 0u;
#pragma unroll
                    for (int b = 0; b < 4; ++b) {
                        if (b >= (int)t.npp) break;
                        const u32 wp = __ballot_sync(0xFFFFFFFFu, (c >> b) & 1u);
                        const u32 wn = __ballot_sync(0xFFFFFFFFu, (cn >> b) & 1u);
                        const u32 hb = __ballot_sync(0xFFFFFFFFu, (ch >> b) & 1u);
                        const u32 hp = hb & 0xFFFFu, hn = hb >> 16;
                        if (lane == b) {
                            vneg = __brev(wn);
                            vpos = (prevw[b] >> 1) | ((wp & 1u) << 31);
                            vop = stp[b] | (hp << 16);
                            von = __brev(stn[b] | (hn << 16));
                        }
                        prevw[b] = wp;
                        if (!odd_step) { stp[b] = hp; stn[b] = hn; }
                    }
                    if ((u32)lane < t.npp) {
                        t.base[(size_t)(K0 - k) * t.npp + lane] = vneg;
                        if (k >= 1u) t.base[(size_t)(K0 + k) * t.npp + lane] = vpos;
                        if (odd_step) {
                            const u32 kap = k >> 1;
                            t.odd[(size_t)(K2 + kap) * t.npp + lane] = vop;
                            t.odd[(size_t)(K2 - kap - 1u) * t.npp + lane] = von;
                        }
                    }
                    // odd-view word of a final unpaired even step
                    if (!odd_step && k + 1u == KS) {
#pragma unroll
                        for (int b = 0; b < 4; ++b) {
                            if (b >= (int)t.npp) break;
                            if (lane == b) {
                                const u32 kap = k >> 1;
                                t.odd[(size_t)(K2 + kap) * t.npp + b] = stp[b];
                                t.odd[(size_t)(K2 - kap - 1u) * t.npp + b] = __brev(stn[b]);
                            }
                        }
                    }
                    // longest monochromatic stretch inside [1, B] (n = 1 starts a run)
                    const bool sv = n >= 1u && n <= B;
                    const u32 V = t.seed ? __ballot_sync(0xFFFFFFFFu, sv) : 0u;
                    if (V) {
                        const u32 fv = (u32)(__ffs(V) - 1), top = 31u - __clz(V);
                        u32 pc = __shfl_up_sync(0xFFFFFFFFu, c, 1);
                        if (lane == 0) pc = cc;
                        const bool chg = sv && (c != pc || n == 1u);
                        const u32 C = __ballot_sync(0xFFFFFFFFu, chg);
                        u32 cl = 0;
                        if (chg) {
                            const u32 below = C & ((1u << lane) - 1u);
                            cl = below ? (u32)lane - (31u - __clz(below)) : clen + (u32)lane - fv;
                        }
                        const u32 mx = __reduce_max_sync(0xFFFFFFFFu, cl);
                        if (mx > best) best = mx;
                        if (C) clen = top - (31u - __clz(C)) + 1u;
                        else clen += top - fv + 1u;
                        cc = __shfl_sync(0xFFFFFFFFu, c, top);
                    }
                }
                __syncwarp();
                if (lane == 0) {
#pragma unroll
                    for (int b = 0; b < 4; ++b) { W.prevw[s][b] = prevw[b]; W.stp[s][b] = stp[b]; W.stn[s][b] = stn[b]; }
                    W.cc[s] = cc; W.clen[s] = clen; W.best[s] = best;
                }
                __syncwarp();
            }
        }
        if (lane == 0) {
            for (u32 s = 0; s < nprof; ++s) {
                const u32 v = max(tw[warp].best[s], tw[warp].clen[s]);
                atomicMax(&a.state[P.first_prof + s].seed, v);
            }
        }
        bad = __syncthreads_or(bad);
        if (bad && threadIdx.x == 0) atomicOr(&a.state[P.first_prof].status, ST_LABEL);
        __syncthreads();
    }
}

}  // namespace CZ_NS
