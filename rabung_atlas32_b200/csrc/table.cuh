// table.cuh -- signed colour bit-planes for the certified rational-anchor filter.
//
// For a sparse-routed prime p with table radius B, every admissible order r gets
// np = ceil(log2 r) bit planes over the signed numerators n in [-B, B]:
// the bit at index u = n + 32*K0 + 31 of plane k is bit k of colour_r(n) written
// in binary, with colour_r(-n) = colour_r(n) + colour_r(-1).  This replaces the
// reference's small_table / fine_labels / pack_pair kernels
// (src/census/engine32/src/small_table.cuh:7-52) and its folded mirror rows.
//
// B200 design:
//  * labels are computed only for primes q in the table (one Montgomery power
//    each, kept in shared memory); every other n takes its label additively
//    through a smallest-prime-factor chain n -> n / spf(n) (the colour is a
//    character), so a table of ~10^6 entries costs ~8e4 powers, not 10^6;
//  * each warp produces 32 consecutive labels per step and emits plane words
//    with one ballot per plane bit: the negative half is one __brev'd ballot
//    (aligned thanks to the +31 centring), the positive half is the previous
//    step's ballot shifted by one with this step's first bit on top;
//  * the same pass records the longest monochromatic stretch inside [1, B] per
//    profile: a real run length, hence a certified lower bound on M (the role
//    of the reference's seed_runs/finish_seed, small_table.cuh:64-136).
#pragma once
#include "labels.cuh"

namespace cz {

constexpr int TABLE_THREADS = 1024;

struct TableArgs {
    const PrimeDesc *primes;
    const ProfDesc *profs;
    ProfState *state;
    u32 *planes;                 // pool
    const u32 *sparse_primes;    // indices of sparse-routed primes
    u32 nsparse;
    const u32 *small_primes;     // all primes below chain_limit, ascending
    u32 n_small;
    const uint2 *chain;          // chain[n] = (index of spf(n) in small_primes, n / spf(n))
    u32 chain_limit;
};

__device__ __forceinline__ u32 table_smem_bytes(u32 slots, u32 nq) {
    return slots * 4u + slots * 2u + 8u + nq * 2u;
}

__global__ void __launch_bounds__(TABLE_THREADS, 1)
table_kernel(TableArgs a) {
    extern __shared__ u32 tsm[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nwarps = blockDim.x >> 5;
    for (u32 it = blockIdx.x; it < a.nsparse; it += gridDim.x) {
        const u32 pi = a.sparse_primes[it];
        const PrimeDesc P = a.primes[pi];
        const Mont M{P.p, P.ninv, P.one, P.r2};
        const u32 slots = hash_slots(P.m);
        u32 *keys = tsm;
        unsigned short *hl = reinterpret_cast<unsigned short *>(keys + slots);
        unsigned short *plab = reinterpret_cast<unsigned short *>(keys + slots + slots / 2u + 2u);
        build_root_hash(keys, hl, slots, M, P.z, P.m);
        const u32 KS = (P.B + 1u + 31u) / 32u + 1u;            // steps: n in [0, 32*KS)
        const u32 nmax = 32u * KS;                               // exclusive
        u32 lo = 0, hi = a.n_small;                              // primes below nmax
        while (lo < hi) {
            u32 mid = (lo + hi) >> 1;
            if (a.small_primes[mid] < nmax) lo = mid + 1; else hi = mid;
        }
        const u32 nq = lo;
        u32 bad = (nmax > a.chain_limit) ? 1u : 0u;
        for (u32 i = threadIdx.x; i < nq; i += blockDim.x) {
            u32 y = mpow(to_mont(a.small_primes[i], M), P.e, M);
            u32 l = lookup_label(keys, hl, slots, y);
            if (l == 0xFFFFu) { bad = 1; l = 0; }
            plab[i] = (unsigned short)l;
        }
        __syncthreads();
        const u32 nprof = P.nprof;
        const u32 mgm = magic_of(P.m);
        u32 rr[8], mg[8], np[8], sg[8];
        u32 *pl[8];
#pragma unroll
        for (int s = 0; s < 8; ++s) {
            if (s < (int)nprof) {
                const ProfDesc D = a.profs[P.first_prof + s];
                rr[s] = D.r; np[s] = D.np; pl[s] = a.planes + D.plane_off;
            } else {
                rr[s] = 2; np[s] = 0; pl[s] = a.planes;
            }
            mg[s] = magic_of(rr[s]);
            sg[s] = mod_small(P.sigma, rr[s], mg[s]);
        }
        const u32 K0 = P.K0, NW = P.nwords;
        for (u32 w = threadIdx.x; w < NW; w += blockDim.x) {      // guard words
            if (w + KS <= K0 || w >= K0 + KS) {
#pragma unroll
                for (int s = 0; s < 8; ++s) {
                    if (s >= (int)nprof) break;
                    for (u32 k = 0; k < np[s]; ++k) pl[s][(size_t)k * NW + w] = 0u;
                }
            }
        }
        const u32 per = (KS + nwarps - 1) / nwarps;
        const u32 k0 = min(KS, warp * per), k1 = min(KS, k0 + per);
        u32 prevw[8][4];
        u32 carry_c[8], carry_len[8], seedbest[8];
#pragma unroll
        for (int s = 0; s < 8; ++s) {
            carry_c[s] = 0xFFFFFFFFu; carry_len[s] = 0; seedbest[s] = 0;
#pragma unroll
            for (int k = 0; k < 4; ++k) prevw[s][k] = 0u;
        }
        const u32 B = P.B;
        for (u32 k = (k0 > 0 ? k0 - 1u : 0u); k < k1; ++k) {
            const u32 n = 32u * k + (u32)lane;
            u32 lab = 0;                       // label of n, additively along the spf chain
            if (n >= 2 && n < a.chain_limit) {
                u32 v = n;
                for (int g = 0; g < 24 && v > 1u; ++g) {
                    const uint2 c = a.chain[v];
                    lab += plab[c.x];
                    v = c.y;
                }
                if (v > 1u) bad = 1;
                lab = mod_small(lab, P.m, mgm);
            }
            const bool pre_step = (k0 > 0 && k == k0 - 1u);
            const bool seedv = !pre_step && n >= 1u && n <= B;
            const u32 V = __ballot_sync(0xFFFFFFFFu, seedv);
            const u32 fv = V ? (u32)(__ffs(V) - 1) : 0u;
            const u32 top = V ? 31u - __clz(V) : 0u;
#pragma unroll
            for (int s = 0; s < 8; ++s) {
                if (s >= (int)nprof) break;
                u32 c = mod_small(lab, rr[s], mg[s]);
                u32 cn = c + sg[s];
                if (cn >= rr[s]) cn -= rr[s];
                if (n == 0) { c = 0; cn = 0; }
#pragma unroll
                for (int bit = 0; bit < 4; ++bit) {
                    if (bit >= (int)np[s]) break;
                    const u32 wp = __ballot_sync(0xFFFFFFFFu, (c >> bit) & 1u);
                    const u32 wn = __ballot_sync(0xFFFFFFFFu, (cn >> bit) & 1u);
                    if (!pre_step && lane == bit) {
                        u32 *P0 = pl[s] + (size_t)bit * NW;
                        P0[K0 - k] = __brev(wn);
                        if (k >= 1) P0[K0 + k] = (prevw[s][bit] >> 1) | ((wp & 1u) << 31);
                    }
                    prevw[s][bit] = wp;
                }
                if (!pre_step && V) {
                    // longest monochromatic stretch inside [1, B] (n = 1 starts a run)
                    u32 pc = __shfl_up_sync(0xFFFFFFFFu, c, 1);
                    if (lane == 0) pc = carry_c[s];
                    const bool chg = seedv && (c != pc || n == 1u);
                    const u32 C = __ballot_sync(0xFFFFFFFFu, chg);
                    u32 clen = 0;
                    if (chg) {
                        const u32 below = C & ((1u << lane) - 1u);
                        clen = below ? (u32)lane - (31u - __clz(below)) : carry_len[s] + (u32)lane - fv;
                    }
                    const u32 mx = __reduce_max_sync(0xFFFFFFFFu, clen);
                    if (mx > seedbest[s]) seedbest[s] = mx;
                    if (C) carry_len[s] = top - (31u - __clz(C)) + 1u;
                    else carry_len[s] += top - fv + 1u;
                    carry_c[s] = __shfl_sync(0xFFFFFFFFu, c, top);
                }
            }
        }
        if (lane == 0) {
#pragma unroll
            for (int s = 0; s < 8; ++s) {
                if (s >= (int)nprof) break;
                u32 v = seedbest[s] > carry_len[s] ? seedbest[s] : carry_len[s];
                atomicMax(&a.state[P.first_prof + s].seed, v);
            }
        }
        bad = __syncthreads_or(bad);
        if (bad && threadIdx.x == 0) atomicOr(&a.state[P.first_prof].status, ST_LABEL);
    }
}

}  // namespace cz
