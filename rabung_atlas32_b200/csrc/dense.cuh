// dense.cuh -- exhaustive half-interval census scan (the dense oracle).
//
// Behaviour follows the reference's dense oracle (src/census/dense_oracle.cu:12-66)
// and historical dense engine (src/census/engine32/build/original_scan_gpu.cu:311-389):
// colour every x in [1, (p-1)/2] by x^((p-1)/m) mod p (one power per x, shared
// by all admissible r of p), keep per-segment run summaries, merge them in
// order, and recover the full profile by reflection with an explicit centre
// join.  The B200 design is its own: integer Montgomery powers (no FP64),
// root labels from a shared-memory hash, run boundaries from warp ballots and
// per-lane __clz on the change mask, segment summaries reduced per CTA in
// shared memory and merged per profile on the device.
//
// Within [1, (p-1)/2] the canonical witness min(s, p-(s+len-1)) of a run
// equals its start s, and the centre run (when r | (p-1)/2) has witness equal
// to its start as well, so summaries carry starts.
#pragma once
#include "labels.cuh"

namespace CZ_NS {

constexpr int DENSE_WARPS = 8;           // warps per CTA = segments per chunk
constexpr int DENSE_STEPS = 256;         // 32-wide steps per segment
constexpr u32 DENSE_SEG = 32u * DENSE_STEPS;

// ordered run summary of a contiguous interval [start, start+len)
struct Summ {
    u32 start, len;
    u32 pre, suf;        // length of the run touching the left / right end
    u32 best, bstart;    // longest run touching neither end, least start
    u32 cf, cl;          // first / last colour
};

__device__ __forceinline__ void take_best(u32 &bl, u32 &bs, u32 l, u32 s) {
    if (l > bl || (l == bl && l != 0 && s < bs)) { bl = l; bs = s; }
}

// a (left) then b (right)
__device__ __forceinline__ Summ merge_summ(const Summ &a, const Summ &b) {
    Summ o;
    o.start = a.start;
    o.len = a.len + b.len;
    o.cf = a.cf;
    o.cl = b.cl;
    bool join = a.cl == b.cf;
    o.pre = (join && a.pre == a.len) ? a.len + b.pre : a.pre;
    o.suf = (join && b.suf == b.len) ? b.len + a.suf : b.suf;
    o.best = a.best; o.bstart = a.bstart;
    take_best(o.best, o.bstart, b.best, b.bstart);
    bool a_closed_left = a.suf < a.len;   // a's suffix run does not touch a's left end
    bool b_closed_right = b.pre < b.len;
    if (join) {
        if (a_closed_left && b_closed_right)
            take_best(o.best, o.bstart, a.suf + b.pre, a.start + a.len - a.suf);
    } else {
        if (a_closed_left) take_best(o.best, o.bstart, a.suf, a.start + a.len - a.suf);
        if (b_closed_right) take_best(o.best, o.bstart, b.pre, b.start);
    }
    return o;
}

// warp-uniform run state of one profile within a warp's segment
struct DRun {
    u32 r, mg;                   // order, its division magic
    u32 carry_c, carry_start, carry_len;   // colour, start and length of the run open at the last x
    u32 pre, bl, bs, cf, inpre;  // prefix run, best closed run (length, start), first colour, prefix open
    u32 pad[2];
};

struct DenseArgs {
    const PrimeDesc *primes;       // all primes of the call
    const u32 *dense_idx;          // dense-local index -> prime index
    const ProfDesc *profs;
    const u32 *chunk_prefix;       // [nprimes+1] CTA chunks per prime (prefix)
    const u32 *summ_prefix;        // [nprimes] first chunk-summary slot of the prime
    u32 nprimes;
    u32 nchunks;                   // total chunks
    Summ *summ;                    // per prime: nprof x nchunks chunk summaries, profile-major
    ProfState *state;
    u32 seg;                       // x per segment (a multiple of 32; DENSE_SEG by default)
};

// One CTA per (prime, chunk of DENSE_WARPS segments); one warp per segment.
__global__ void __launch_bounds__(DENSE_WARPS * 32)
dense_scan_kernel(DenseArgs a) {
    extern __shared__ __align__(16) u32 dsm[];
    __shared__ Summ wsum[DENSE_WARPS][8];
    __shared__ __align__(16) DRun drun[DENSE_WARPS][8];
    __shared__ u32 cur_prime;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    u32 prev_prime = 0xFFFFFFFFu;
    pw_t *keys = reinterpret_cast<pw_t *>(dsm);
    unsigned short *labs = nullptr;
    u32 slots = 0;
    for (u32 chunk = blockIdx.x; chunk < a.nchunks; chunk += gridDim.x) {
        if (threadIdx.x == 0) {
            u32 lo = 0, hi = a.nprimes;           // last i with prefix[i] <= chunk
            while (hi - lo > 1) {
                u32 mid = (lo + hi) >> 1;
                if (a.chunk_prefix[mid] <= chunk) lo = mid; else hi = mid;
            }
            cur_prime = lo;
        }
        __syncthreads();
        const u32 pi = cur_prime;
        const PrimeDesc P = a.primes[a.dense_idx[pi]];
        const Mont M{P.p, P.ninv, P.one, P.r2};
        if (pi != prev_prime) {
            slots = hash_slots(P.m);
            labs = reinterpret_cast<unsigned short *>(keys + slots);
            build_root_hash(keys, labs, slots, M, P.z, P.m);
            prev_prime = pi;
        }
        const u32 local_chunk = chunk - a.chunk_prefix[pi];
        const u32 nh = (u32)((P.p - 1u) >> 1);             // p < 2^33: fits 32 bits
        const u32 seg = local_chunk * DENSE_WARPS + warp;
        // x of the segment's first element; in 64 bits, since (p-1)/2 reaches
        // 2^32 - 1 in 64-bit words and the chunk's last segments lie past it
        const u64 seg_start64 = 1ull + (u64)seg * a.seg;
        const u32 seg_start = (u32)seg_start64;
        const u32 nprof = P.nprof;
        // per-profile run state: warp-uniform, so it lives in this warp's shared
        // records (one read and one write per profile per 32 x) instead of
        // registers, which keeps the kernel's occupancy up
        if ((u32)lane < nprof) {
            const u32 r = a.profs[P.first_prof + lane].r;
            drun[warp][lane] = DRun{r, magic_of(r), 0xFFFFFFFFu, seg_start, 0u, 0u, 0u, 0u, 0u, 1u, 0u, 0u};
        }
        __syncwarp();
        const bool active = seg_start64 <= (u64)nh;
        const u32 seg_end = active ? (u32)min((u64)nh, seg_start64 + a.seg - 1u) : 0u;   // inclusive
        // x is compared through its offset in the segment: seg_start + offset
        // may pass 2^32 - 1 beyond seg_end, the offset never wraps
        const u32 seg_last = seg_end - seg_start;
        u32 bad = 0;
        if (active) {
            const u32 nsteps = (seg_end - seg_start) / 32u + 1u;
            // the run bookkeeping of one 32-wide step for every profile
            auto step_runs = [&](u32 st, u32 label) {
                const u32 base = seg_start + st * 32u;
                const bool valid = st * 32u + (u32)lane <= seg_last;
                const u32 nvalid = min(32u, seg_last - st * 32u + 1u);
                for (u32 s = 0; s < nprof; ++s) {
                    DRun R = drun[warp][s];
                    const u32 c = mod_small(label, R.r, R.mg);
                    u32 pc = __shfl_up_sync(0xFFFFFFFFu, c, 1);
                    if (lane == 0) pc = R.carry_c;
                    const bool chg = valid && (c != pc);
                    const u32 C = __ballot_sync(0xFFFFFFFFu, chg);
                    if (st == 0) R.cf = __shfl_sync(0xFFFFFFFFu, c, 0);
                    // run closing at lane-1 for each lane that starts a new run
                    u32 clen = 0, cst = 0;
                    if (chg) {
                        const u32 below = C & ((1u << lane) - 1u);
                        if (below) {
                            const u32 h = 31u - __clz(below);
                            clen = lane - h; cst = base + h;
                        } else {
                            clen = R.carry_len + lane; cst = R.carry_start;
                        }
                    }
                    // the first closed run of the segment is its prefix run
                    if (R.inpre && C) {
                        const u32 first = __ffs(C) - 1u;   // lowest change lane
                        const u32 plen = __shfl_sync(0xFFFFFFFFu, clen, first);
                        if (plen > 0) {
                            R.pre = plen;
                            R.inpre = 0u;
                            if (lane == (int)first) clen = 0;
                        } else {
                            // change at the segment's first element: the empty carry run
                            const u32 rest = C & ~(1u << first);
                            if (rest) {
                                const u32 f2 = __ffs(rest) - 1u;
                                const u32 pl2 = __shfl_sync(0xFFFFFFFFu, clen, f2);
                                R.pre = pl2;
                                R.inpre = 0u;
                                if (lane == (int)f2) clen = 0;
                            }
                        }
                    }
                    const u32 mlen = __reduce_max_sync(0xFFFFFFFFu, clen);
                    if (mlen > 0 && mlen >= R.bl) {
                        const u32 mst = __reduce_min_sync(0xFFFFFFFFu, clen == mlen ? cst : 0xFFFFFFFFu);
                        take_best(R.bl, R.bs, mlen, mst);
                    }
                    if (C) {
                        const u32 h = 31u - __clz(C);
                        R.carry_start = base + h;
                        R.carry_len = nvalid - h;
                    } else {
                        R.carry_len += nvalid;
                    }
                    R.carry_c = __shfl_sync(0xFFFFFFFFu, c, nvalid - 1u);
                    __syncwarp();
                    drun[warp][s] = R;                     // every lane writes the same record
                    __syncwarp();
                }
            };
            // labels two steps at a time: each lane's two powers are independent chains
            auto label_of = [&](pw_t y, bool valid) {
                if (!valid) return 0u;
                u32 l = lookup_label(keys, labs, slots, y);
                if (l == 0xFFFFu) { bad = 1; l = 0; }
                return l;
            };
            for (u32 st = 0; st < nsteps; st += 2u) {
                const u32 o0 = st * 32u + (u32)lane, o1 = o0 + 32u;
                const bool v0 = o0 <= seg_last, v1 = st + 1u < nsteps && o1 <= seg_last;
                const u32 x0 = seg_start + o0, x1 = seg_start + o1;
                pw_t y0, y1;
                mpow2(to_mont((pw_t)(v0 ? x0 : 1u), M), to_mont((pw_t)(v1 ? x1 : 1u), M), P.e, M, y0, y1);
                const u32 l0 = label_of(y0, v0), l1 = label_of(y1, v1);
                step_runs(st, l0);
                if (st + 1u < nsteps) step_runs(st + 1u, l1);
            }
        }
        bad = __reduce_or_sync(0xFFFFFFFFu, bad);
        if (lane == 0) {
            if (bad) atomicOr(&a.state[P.first_prof].status, ST_LABEL);
            for (u32 s = 0; s < nprof; ++s) {
                const DRun &R = drun[warp][s];
                Summ o;
                if (active) {
                    o.start = seg_start; o.len = seg_end - seg_start + 1u;
                    o.suf = R.carry_len;
                    o.pre = R.inpre ? o.len : R.pre;
                    o.best = R.bl; o.bstart = R.bs;
                    o.cf = R.cf; o.cl = R.carry_c;
                } else {
                    o.start = 0; o.len = 0; o.pre = o.suf = o.best = o.bstart = 0; o.cf = o.cl = 0;
                }
                wsum[warp][s] = o;
            }
        }
        __syncthreads();
        // thread s merges the CTA's segments for profile s, in order
        if (threadIdx.x < nprof) {
            const int s = threadIdx.x;
            Summ acc = wsum[0][s];
            for (int w = 1; w < DENSE_WARPS; ++w)
                if (wsum[w][s].len) acc = merge_summ(acc, wsum[w][s]);
            const u32 nch = a.chunk_prefix[pi + 1] - a.chunk_prefix[pi];
            a.summ[a.summ_prefix[pi] + (u32)s * nch + local_chunk] = acc;
        }
        __syncthreads();
    }
}

struct DenseMergeArgs {
    const PrimeDesc *primes;
    const ProfDesc *profs;
    const u32 *chunk_prefix;
    const u32 *summ_prefix;
    u32 nprimes;
    const Summ *summ;
    ProfState *state;        // indexed by global profile index
    u32 *prefix_out;         // L per global profile index
};

// one warp per dense profile: lanes merge contiguous runs of chunk summaries,
// lane 0 merges the 32 partial summaries, applies the reflection centre join.
__global__ void dense_merge_kernel(DenseMergeArgs a, const u32 *dense_prof_list, u32 ndprof) {
    const u32 gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (gw >= ndprof) return;
    const u32 gprof = dense_prof_list[gw];
    const ProfDesc D = a.profs[gprof];
    const u32 pi = D.local;                  // dense-local prime index
    const PrimeDesc P = a.primes[D.prime];
    const u32 s = gprof - P.first_prof;
    const u32 nch = a.chunk_prefix[pi + 1] - a.chunk_prefix[pi];
    const Summ *base = a.summ + a.summ_prefix[pi] + s * nch;
    const u32 per = (nch + 31u) / 32u;
    const u32 lo = min(nch, lane * per), hi = min(nch, lo + per);
    Summ acc{};
    bool have = false;
    for (u32 i = lo; i < hi; ++i) {
        Summ v = base[i];
        if (!v.len) continue;
        acc = have ? merge_summ(acc, v) : v;
        have = true;
    }
    __shared__ Summ part[32 * 8];
    Summ *mine = part + (threadIdx.x >> 5) * 32;
    mine[lane] = have ? acc : Summ{};
    __syncwarp();
    if (lane != 0) return;
    Summ tot{};
    bool h2 = false;
    for (int l = 0; l < 32; ++l) {
        if (!mine[l].len) continue;
        tot = h2 ? merge_summ(tot, mine[l]) : mine[l];
        h2 = true;
    }
    const pw_t p = P.p;
    const u32 nh = (u32)((p - 1u) >> 1), r = D.r;
    const bool sym = (nh % r) == 0u;     // r | (p-1)/2: colour(p-x) = colour(x)
    u32 bl = tot.best, bs = tot.bstart;
    u32 L;
    if (tot.pre == nh) {
        // the whole half interval is one run
        if (sym) { bl = (u32)(p - 1u); bs = 1u; L = (u32)(p - 1u); }
        else { bl = nh; bs = 1u; L = nh; }
    } else {
        take_best(bl, bs, tot.pre, 1u);                       // run from x = 1
        if (sym) take_best(bl, bs, 2u * tot.suf, nh - tot.suf + 1u);   // centre join
        else take_best(bl, bs, tot.suf, nh - tot.suf + 1u);
        L = tot.pre;                                          // colour(1) = 0
    }
    a.state[gprof].best = pack_key(bl, bs);
    a.prefix_out[gprof] = L;
}

}  // namespace CZ_NS
