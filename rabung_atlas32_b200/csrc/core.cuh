#pragma once
// core.cuh -- host planning and one census call of librabung_census.so, for
// one prime word width.  Included once by census.cu (p < 2^32, 32-bit words,
// handle cz_handle, records cz_profile) and once by census_wide.cu (CZ_WIDE:
// p < 2^33, 64-bit words, handle cz_handle64, records cz_profile64), so the
// two domains share every line of planning, routing, waves, re-runs and
// kernel launches.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "common.cuh"
#include "labels.cuh"
#include "dense.cuh"
#include "table.cuh"
#include "sparse.cuh"
#include "finalize.cuh"
#include "a4.cuh"
#include "../../include/rabung_census.h"

#if CZ_WIDE
#define CZ_HANDLE cz_handle64
#define CZ_RECORD cz_profile64
#else
#define CZ_HANDLE cz_handle
#define CZ_RECORD cz_profile
#endif

using namespace CZ_NS;

namespace {

constexpr u32 CHAIN_LIMIT = (1u << 20) + 8192u;   // table labels cover n < CHAIN_LIMIT
constexpr u32 B_MAX = (1u << 20);
constexpr u64 PW_LIMIT = CZ_WIDE ? (1ull << 33) : (1ull << 32);   // primes of this build lie below
constexpr u32 TABLE_DYN_SMEM = 190u * 1024u;        // dynamic part; static part ~34 KB

struct Buf {
    void *p = nullptr;
    size_t cap = 0;
};

bool cover_cert(u64 B, u64 D, u64 H, u64 p) {
    if (H * D > 2 * B) return false;
    const unsigned __int128 lhs = (unsigned __int128)4 * B * D - (unsigned __int128)H * D * D;
    return lhs > (unsigned __int128)4 * p;
}

// table radius for a prime: D = floor(2 sqrt(p/H) / n), B = floor((4p + H D^2)/(4D)) + 1
// (the reference's lower-branch choice, paper/GPU_METHOD_EN.tex "Choosing parameters";
// P/src/clipped_cover.hpp:14-21), certified in integers.
bool cover_B(u64 p, u32 Q, u32 ndiv, u32 &Bout) {
    const u64 H = Q - 1u;
    const double D0 = 2.0 * std::sqrt((double)p / (double)H);
    u64 D = (u64)(D0 / (double)ndiv);
    if (D < 1) D = 1;
    const u64 B = (4ull * p + H * D * D) / (4ull * D) + 1ull;
    if (B >= p || D >= p || B > B_MAX) return false;
    if (!cover_cert(B, D, H, p)) return false;
    Bout = (u32)B;
    return true;
}

// least D with the certificate for (p, B, Q)
bool cover_D(u64 p, u32 B, u32 Q, u32 &Dout) {
    const u64 H = Q - 1u;
    const long double disc = (long double)B * B - (long double)H * p;
    if (disc <= 0) return false;
    long double est = (2.0L * B - 2.0L * std::sqrt(disc)) / (long double)H;
    u64 D = est < 1 ? 1 : (u64)est;
    while (D > 1 && cover_cert(B, D - 1, H, p)) --D;
    while (!cover_cert(B, D, H, p)) {
        ++D;
        if (H * D > 2ull * B || D >= p || D > B_MAX) return false;
    }
    Dout = (u32)D;
    return true;
}

u32 popc(u32 x) { return (u32)__builtin_popcount(x); }

// one launch with its own error code: a launch failure is reported through the
// return value, and an error the caller left pending is neither read nor cleared
template <class... A>
bool launch(void (*k)(A...), dim3 grid, dim3 block, size_t smem, cudaStream_t st, A... args) {
    void *argv[] = {static_cast<void *>(&args)...};
    return cudaLaunchKernel(reinterpret_cast<const void *>(k), grid, block, argv, smem, st) == cudaSuccess;
}

}  // namespace

struct CZ_HANDLE {
    cz_config cfg{};
    int dev = 0;
    int sms = 148;
    cudaStream_t st = nullptr;
    std::string err;
    u32 *d_small = nullptr;
    uint2 *d_chain = nullptr;
    u32 n_small = 0;
    // device buffers
    Buf b_in, b_primes, b_profs, b_state, b_planes, b_summ, b_chunk, b_summp, b_didx, b_sidx,
        b_slist, b_dlist, b_dpre, b_out, b_a4, b_counter, b_sreq, b_sout;
    // host copies of the current plan
    std::vector<PrimeDesc> hp;
    std::vector<ProfDesc> hprof;
    std::vector<u32> h_chunk, h_summp, h_didx, h_sidx, h_slist, h_dlist;
    u32 n = 0, nprof = 0, ndense = 0, nsparse = 0, nchunks = 0, nsl = 0, ndl = 0;
    u32 table_smem = 0, dense_smem = 0;
    u32 flags = 0;
    bool have_plan = false;
    cudaEvent_t ev[10]{};
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t gexec = nullptr;
    cz_stats last{};
    std::vector<OutRecord> hout;
    void *pin = nullptr;
    size_t pin_cap = 0;
};

namespace {

bool ck(CZ_HANDLE *h, cudaError_t e, const char *what) {
    if (e == cudaSuccess) return true;
    h->err = std::string(what) + ": " + cudaGetErrorString(e);
    return false;
}

bool ensure(CZ_HANDLE *h, Buf &b, size_t bytes) {
    if (bytes == 0) bytes = 16;
    if (b.cap >= bytes) return true;
    if (b.p) cudaFree(b.p);
    b.p = nullptr;
    b.cap = 0;
    size_t want = bytes + bytes / 4;
    if (!ck(h, cudaMalloc(&b.p, want), "cudaMalloc")) return false;
    b.cap = want;
    return true;
}

template <class T> T *P(Buf &b) { return reinterpret_cast<T *>(b.p); }

bool build_static_tables(CZ_HANDLE *h) {
    // primes below CHAIN_LIMIT and the prime-power chain: chain[n] =
    // (index of q = spf(n) | e << 24, n / q^e) with q^e the full power of q in
    // n, so a walk takes one step per distinct prime factor (at most 7 below
    // 2^20), not one per factor
    std::vector<u32> spf(CHAIN_LIMIT, 0);
    std::vector<u32> primes;
    for (u32 i = 2; i < CHAIN_LIMIT; ++i) {
        if (!spf[i]) {
            spf[i] = i;
            primes.push_back(i);
            if ((u64)i * i < CHAIN_LIMIT)
                for (u32 j = i * i; j < CHAIN_LIMIT; j += i)
                    if (!spf[j]) spf[j] = i;
        }
    }
    std::vector<u32> index(CHAIN_LIMIT, 0);
    for (u32 k = 0; k < primes.size(); ++k) index[primes[k]] = k;
    std::vector<uint2> chain(CHAIN_LIMIT);
    chain[0] = make_uint2(0, 0);
    chain[1] = make_uint2(0, 1);
    for (u32 n = 2; n < CHAIN_LIMIT; ++n) {
        const u32 q = spf[n];
        u32 m = n, e = 0;
        while (m % q == 0) { m /= q; ++e; }
        chain[n] = make_uint2(index[q] | (e << 24), m);     // index < 2^17, e <= 20
    }
    h->n_small = (u32)primes.size();
    if (!ck(h, cudaMalloc(&h->d_small, primes.size() * 4), "cudaMalloc small")) return false;
    if (!ck(h, cudaMalloc(&h->d_chain, chain.size() * sizeof(uint2)), "cudaMalloc chain")) return false;
    if (!ck(h, cudaMemcpy(h->d_small, primes.data(), primes.size() * 4, cudaMemcpyHostToDevice), "copy small")) return false;
    if (!ck(h, cudaMemcpy(h->d_chain, chain.data(), chain.size() * sizeof(uint2), cudaMemcpyHostToDevice), "copy chain")) return false;
    return true;
}

u32 q_for(const cz_config &c, u32 r) { return c.q_cap[r] ? c.q_cap[r] : 16u; }

// dense segment length in x (32 x steps), default DENSE_SEG
u32 dense_seg(const cz_config &c) {
    const u32 steps = c.dense_steps ? std::min(4096u, std::max(8u, c.dense_steps)) : (u32)DENSE_STEPS;
    return 32u * steps;
}

// speculative threshold: floor(log_r p - margin_r), a low quantile of M for
// random-looking colourings (M ~ log_r p); 0 disables
u32 qspec_for(const cz_config &c, pw_t p, u32 r, bool allow) {
    if (!allow || !c.speculate) return 0u;
    const double lg = std::log((double)p) / std::log((double)r);
    const double m = c.spec_margin10[r] / 10.0;
    const double v = std::floor(lg - m);
    return v < 3.0 ? 0u : (u32)v;
}

// host plan of one call
constexpr u32 CZ_NOSPEC = 1u << 16;      // internal: plan without speculative thresholds

int plan(CZ_HANDLE *h, const pw_t *primes, u32 n, u32 flags) {
    const cz_config &c = h->cfg;
    h->hp.assign(n, PrimeDesc{});
    h->hprof.clear();
    h->h_didx.clear(); h->h_sidx.clear(); h->h_slist.clear(); h->h_dlist.clear();
    h->h_chunk.assign(1, 0u); h->h_summp.clear();
    u64 plane_words = 0;
    u32 max_slots_t = 8, max_slots_d = 8, max_nq = 0;
    u64 summ_slots = 0;
    const u32 mode = flags & CZ_AUTO;
    for (u32 i = 0; i < n; ++i) {
        const pw_t p = primes[i];
        if (p < 2u || (u64)p >= PW_LIMIT) { h->err = "prime out of domain: " + std::to_string(p); return CZ_EINVAL; }
        PrimeDesc &P = h->hp[i];
        P.p = p;
        P.mask = p > 2u ? mask_of(p) : 0u;
        P.m = lcm_of_mask(P.mask);
        P.e = P.mask ? (p - 1u) / P.m : 0u;
        P.first_prof = (u32)h->hprof.size();
        P.nprof = popc(P.mask);
        P.route = 0;
        if (!P.nprof) continue;
        bool sparse = false;
        if (mode == CZ_SPARSE) sparse = true;
        else if (mode == CZ_AUTO) sparse = p >= c.sparse_min_p;
        u32 B = 0, Qmax = 0;
        std::vector<u32> Ds;
        if (sparse) {
            for (u32 r = 2; r <= 9; ++r)
                if (P.mask & (1u << (r - 2))) Qmax = std::max(Qmax, q_for(c, r));
            if (p < 4096u || Qmax + 1u >= p || !cover_B(p, Qmax, c.cover_n, B)) sparse = false;
            if (sparse) {
                for (u32 r = 2; r <= 9 && sparse; ++r) {
                    if (!(P.mask & (1u << (r - 2)))) continue;
                    u32 D = 0;
                    if (!cover_D(p, B, q_for(c, r), D)) sparse = false;
                    Ds.push_back(D);
                }
            }
            if (!sparse && mode == CZ_SPARSE) {
                h->err = "sparse path unsupported for p = " + std::to_string(p);
                return CZ_EINVAL;
            }
        }
        P.route = sparse ? 2u : 1u;
        if (sparse) {
            P.B = B;
            // view widths in words, multiples of 4: every view and every tile
            // copy of the filter starts on a 16-byte boundary
            P.K0 = (B + 31u) / 32u + 4u;
            P.nwords = (2u * P.K0 + 8u + 3u) & ~3u;
            P.K2 = (B + 63u) / 64u + 4u;
            P.nwords2 = (2u * P.K2 + 8u + 3u) & ~3u;
            h->h_sidx.push_back(i);
            max_slots_t = std::max(max_slots_t, hash_slots(P.m));
        } else {
            const u32 nh = (u32)((p - 1u) / 2u);           // < 2^32 for p < 2^33
            const u32 seg = dense_seg(c);
            const u32 nseg = (u32)(((u64)nh + seg - 1u) / seg);   // nh + seg wraps 32 bits near 2^33
            const u32 nch = (nseg + DENSE_WARPS - 1u) / DENSE_WARPS;
            if ((u64)h->h_chunk.back() + nch > 0xFFFFFFFFull || summ_slots + (u64)nch * P.nprof > 0xFFFFFFFFull) {
                h->err = "dense scan too large for one call (chunk index beyond 32 bits)";
                return CZ_ELIMIT;
            }
            h->h_didx.push_back(i);
            h->h_summp.push_back((u32)summ_slots);
            summ_slots += (u64)nch * P.nprof;
            h->h_chunk.push_back(h->h_chunk.back() + nch);
            max_slots_d = std::max(max_slots_d, hash_slots(P.m));
        }
        u32 k = 0;
        for (u32 r = 2; r <= 9; ++r) {
            if (!(P.mask & (1u << (r - 2)))) continue;
            ProfDesc D{};
            D.prime = i;
            D.r = r;
            D.np = planes_for(r);
            D.npp = planes_stored(r);
            D.out_slot = (u32)h->hprof.size();
            if (sparse) {
                D.Q = q_for(c, r);
                D.D = Ds[k];
                D.qspec = qspec_for(c, p, r, !(flags & CZ_NOSPEC));
                D.tpref = c.anchor_t[r] ? c.anchor_t[r] : anchor_pref(r, c.anchor_bits);
                const u64 pw = ((u64)D.npp * (P.nwords + P.nwords2) + 7ull) & ~7ull;
                D.plane_off = plane_words;              // multiple of 8 words: vector loads and tile copies align
                plane_words += pw;
                D.local = (u32)h->h_sidx.size() - 1u;
                h->h_slist.push_back((u32)h->hprof.size());
            } else {
                D.local = (u32)h->h_didx.size() - 1u;
                h->h_dlist.push_back((u32)h->hprof.size());
            }
            h->hprof.push_back(D);
            ++k;
        }
    }
    h->n = n;
    h->nprof = (u32)h->hprof.size();
    h->ndense = (u32)h->h_didx.size();
    h->nsparse = (u32)h->h_sidx.size();
    h->nchunks = h->h_chunk.back();
    // longest first: the persistent filter hands out profiles in list order,
    // so the costly ones (more stored planes, larger p) start first and the
    // launch ends on short profiles
    std::stable_sort(h->h_slist.begin(), h->h_slist.end(), [h](u32 x, u32 y) {
        const ProfDesc &a = h->hprof[x], &b = h->hprof[y];
        if (a.npp != b.npp) return a.npp > b.npp;
        return h->hp[a.prime].p > h->hp[b.prime].p;
    });
    h->nsl = (u32)h->h_slist.size();
    h->ndl = (u32)h->h_dlist.size();
    // primes below the largest table end, for the table kernel's shared memory
    u32 maxB = 0;
    for (u32 i : h->h_sidx) maxB = std::max(maxB, h->hp[i].B);
    if (h->nsparse) {
        const u32 nmax = 32u * ((maxB + 1u + 31u) / 32u + 1u);
        // count primes below nmax on the host (static table is sorted)
        static std::vector<u32> hs;
        static std::once_flag once;
        std::call_once(once, [] {
            std::vector<char> comp(CHAIN_LIMIT, 0);
            for (u32 i = 2; i < CHAIN_LIMIT; ++i)
                if (!comp[i]) {
                    hs.push_back(i);
                    if ((u64)i * i < CHAIN_LIMIT)
                        for (u32 j = i * i; j < CHAIN_LIMIT; j += i) comp[j] = 1;
                }
        });
        max_nq = (u32)(std::lower_bound(hs.begin(), hs.end(), nmax) - hs.begin());
    }
    h->table_smem = max_slots_t * (u32)(sizeof(pw_t) + 2u) + 8u + max_nq * 2u + 16u;
    if (h->table_smem > TABLE_DYN_SMEM) {
        h->err = "table shared memory above the per-block limit";
        return CZ_EINVAL;
    }
    h->dense_smem = max_slots_d * (u32)(sizeof(pw_t) + 2u) + 16u;
    // device buffers
    if (!ensure(h, h->b_primes, sizeof(PrimeDesc) * n) ||
        !ensure(h, h->b_profs, sizeof(ProfDesc) * h->nprof) ||
        !ensure(h, h->b_state, sizeof(ProfState) * h->nprof) ||
        !ensure(h, h->b_planes, plane_words * 4ull) ||
        !ensure(h, h->b_summ, sizeof(Summ) * summ_slots) ||
        !ensure(h, h->b_chunk, 4ull * h->h_chunk.size()) ||
        !ensure(h, h->b_summp, 4ull * h->h_summp.size()) ||
        !ensure(h, h->b_didx, 4ull * h->ndense) ||
        !ensure(h, h->b_sidx, 4ull * h->nsparse) ||
        !ensure(h, h->b_slist, 4ull * h->nsl) ||
        !ensure(h, h->b_dlist, 4ull * h->ndl) ||
        !ensure(h, h->b_dpre, 4ull * h->nprof) ||
        !ensure(h, h->b_out, sizeof(OutRecord) * h->nprof) ||
        !ensure(h, h->b_a4, 4ull * n) ||
        !ensure(h, h->b_counter, 64))
        return CZ_ECUDA;
    h->flags = flags;
    h->have_plan = true;
    return CZ_OK;
}

int upload(CZ_HANDLE *h, cz_stats *s) {
    cudaStream_t st = h->st;
    size_t total = sizeof(PrimeDesc) * h->n + sizeof(ProfDesc) * h->nprof +
                   4ull * (h->h_chunk.size() + h->h_summp.size() + h->ndense + h->nsparse + h->nsl + h->ndl) + 64 * 8;
    if (h->pin_cap < total) {
        if (h->pin) cudaFreeHost(h->pin);
        h->pin = nullptr;
        h->pin_cap = 0;
        if (!ck(h, cudaHostAlloc(&h->pin, total + total / 4, cudaHostAllocDefault), "cudaHostAlloc")) return CZ_ECUDA;
        h->pin_cap = total + total / 4;
    }
    // the host plan is staged in pinned memory and copied asynchronously
    char *stage = static_cast<char *>(h->pin);
    size_t bytes = 0;
    auto put = [&](Buf &b, const void *src, size_t n) {
        if (n == 0) return true;
        std::memcpy(stage + bytes, src, n);
        const bool ok = ck(h, cudaMemcpyAsync(b.p, stage + bytes, n, cudaMemcpyHostToDevice, st), "h2d");
        bytes += (n + 63) & ~size_t(63);
        return ok;
    };
    if (!put(h->b_primes, h->hp.data(), sizeof(PrimeDesc) * h->n) ||
        !put(h->b_profs, h->hprof.data(), sizeof(ProfDesc) * h->nprof) ||
        !put(h->b_chunk, h->h_chunk.data(), 4ull * h->h_chunk.size()) ||
        !put(h->b_summp, h->h_summp.data(), 4ull * h->h_summp.size()) ||
        !put(h->b_didx, h->h_didx.data(), 4ull * h->ndense) ||
        !put(h->b_sidx, h->h_sidx.data(), 4ull * h->nsparse) ||
        !put(h->b_slist, h->h_slist.data(), 4ull * h->nsl) ||
        !put(h->b_dlist, h->h_dlist.data(), 4ull * h->ndl))
        return CZ_ECUDA;
    if (s) s->h2d_bytes = bytes;
    return CZ_OK;
}

// enqueue the device work of the current plan on h->st; returns launches
int enqueue(CZ_HANDLE *h, bool timed, u32 &launches) {
    cudaStream_t st = h->st;
    launches = 0;
    auto rec = [&](int i) { if (timed) cudaEventRecord(h->ev[i], st); };
    rec(0);
    if (h->n) {
        setup_kernel<<<(h->n + 127) / 128, 128, 0, st>>>(P<PrimeDesc>(h->b_primes), P<ProfDesc>(h->b_profs),
                                                         P<ProfState>(h->b_state), h->n);
        ++launches;
    }
    rec(1);
    if (h->nsparse) {
        TableArgs ta;
        ta.primes = P<PrimeDesc>(h->b_primes);
        ta.profs = P<ProfDesc>(h->b_profs);
        ta.state = P<ProfState>(h->b_state);
        ta.planes = P<u32>(h->b_planes);
        ta.sparse_primes = P<u32>(h->b_sidx);
        ta.nsparse = h->nsparse;
        ta.small_primes = h->d_small;
        ta.n_small = h->n_small;
        ta.chain = h->d_chain;
        ta.chain_limit = CHAIN_LIMIT;
        const u32 grid = std::min<u32>(h->nsparse, (u32)h->sms);
        table_kernel<<<grid, TABLE_THREADS, h->table_smem, st>>>(ta);
        ++launches;
    }
    rec(2);
    if (h->nsl) {
        cudaMemsetAsync(h->b_counter.p, 0, 64, st);
        SparseArgs sa{};                       // serving fields stay null: one-call census
        sa.primes = P<PrimeDesc>(h->b_primes);
        sa.profs = P<ProfDesc>(h->b_profs);
        sa.state = P<ProfState>(h->b_state);
        sa.planes = P<u32>(h->b_planes);
        sa.prof_list = P<u32>(h->b_slist);
        sa.nlist = h->nsl;
        sa.next = P<u32>(h->b_counter);
        u32 grid = h->cfg.sparse_blocks ? h->cfg.sparse_blocks : (u32)CZ_SPARSE_MINB * (u32)h->sms;
        // a call with few profiles spreads each profile's rows over more CTAs
        // (up to 64), so small calls fill the GPU; large calls keep the tuned group
        sa.group = std::max(std::max(1u, h->cfg.cta_per_profile), std::min(64u, grid / std::max(1u, h->nsl)));
        sa.tune.screen = h->cfg.screen;
        sa.epoch_rows = h->cfg.epoch_rows;
        grid = std::min(grid, h->nsl * sa.group);
        sparse_kernel<<<grid, SPARSE_WARPS * 32, TILE_WORDS * 4u, st>>>(sa);
        ++launches;
    }
    rec(3);
    if (h->ndense) {
        DenseArgs da;
        da.primes = P<PrimeDesc>(h->b_primes);
        da.dense_idx = P<u32>(h->b_didx);
        da.profs = P<ProfDesc>(h->b_profs);
        da.chunk_prefix = P<u32>(h->b_chunk);
        da.summ_prefix = P<u32>(h->b_summp);
        da.nprimes = h->ndense;
        da.nchunks = h->nchunks;
        da.summ = P<Summ>(h->b_summ);
        da.state = P<ProfState>(h->b_state);
        da.seg = dense_seg(h->cfg);
        const u32 grid = std::min<u32>(h->nchunks, (u32)h->sms * 8u);
        dense_scan_kernel<<<grid, DENSE_WARPS * 32, h->dense_smem, st>>>(da);
        DenseMergeArgs ma;
        ma.primes = P<PrimeDesc>(h->b_primes);
        ma.profs = P<ProfDesc>(h->b_profs);
        ma.chunk_prefix = P<u32>(h->b_chunk);
        ma.summ_prefix = P<u32>(h->b_summp);
        ma.nprimes = h->ndense;
        ma.summ = P<Summ>(h->b_summ);
        ma.state = P<ProfState>(h->b_state);
        ma.prefix_out = P<u32>(h->b_dpre);
        dense_merge_kernel<<<(h->ndl + 7) / 8, 256, 0, st>>>(ma, P<u32>(h->b_dlist), h->ndl);
        launches += 2;
    }
    rec(4);
    if (h->nprof) {
        finalize_kernel<<<(h->nprof + 127) / 128, 128, 0, st>>>(
            P<PrimeDesc>(h->b_primes), P<ProfDesc>(h->b_profs), P<ProfState>(h->b_state), P<u32>(h->b_dpre),
            h->nprof, (h->flags & CZ_VERIFY) ? 1u : 0u, P<OutRecord>(h->b_out));
        ++launches;
    }
    rec(5);
    if ((h->flags & CZ_A4) && h->n) {
        // the A4 error word is cleared by every call that counts points, also
        // when no sparse profile cleared the counter block above
        cudaMemsetAsync(P<u32>(h->b_counter) + 8, 0, 4, st);
        a4_kernel<<<(h->n + A4_WARPS - 1) / A4_WARPS, A4_WARPS * 32, 0, st>>>(P<PrimeDesc>(h->b_primes), h->n,
                                                                           P<u32>(h->b_a4), P<u32>(h->b_counter) + 8);
        ++launches;
    }
    rec(6);
    return ck(h, cudaGetLastError(), "launch") ? CZ_OK : CZ_ECUDA;
}

void read_times(CZ_HANDLE *h, cz_stats *s) {
    float t[6] = {0};
    for (int i = 0; i < 6; ++i) cudaEventElapsedTime(&t[i], h->ev[i], h->ev[i + 1]);
    s->ms_setup = t[0]; s->ms_table = t[1]; s->ms_sparse = t[2]; s->ms_dense = t[3];
    s->ms_finalize = t[4]; s->ms_a4 = t[5];
    cudaEventElapsedTime(&s->ms_device, h->ev[0], h->ev[6]);
}

int check_records(CZ_HANDLE *h, std::vector<u32> *fallback, std::vector<u32> *respec = nullptr) {
    for (u32 g = 0; g < h->nprof; ++g) {
        const OutRecord &o = h->hout[g];
        if (o.status) {
            const PrimeDesc &P = h->hp[h->hprof[g].prime];
            if (respec && P.route == 2u && o.status == ST_SPEC) {
                if (respec->empty() || respec->back() != h->hprof[g].prime)
                    respec->push_back(h->hprof[g].prime);
                continue;
            }
            if (fallback && P.route == 2u && !(o.status & (ST_ROOT | ST_LABEL | ST_VERIFY))) {
                if (fallback->empty() || fallback->back() != h->hprof[g].prime)
                    fallback->push_back(h->hprof[g].prime);
                continue;
            }
            char buf[160];
            snprintf(buf, sizeof buf, "refused: p=%llu r=%u status=0x%x", (unsigned long long)o.p, o.r, o.status);
            h->err = buf;
            return CZ_EREFUSED;
        }
    }
    return CZ_OK;
}

}  // namespace


namespace {

void handle_close(CZ_HANDLE *h) {
    if (!h) return;
    cudaSetDevice(h->dev);
    if (h->gexec) cudaGraphExecDestroy(h->gexec);
    if (h->graph) cudaGraphDestroy(h->graph);
    Buf *bufs[] = {&h->b_in, &h->b_primes, &h->b_profs, &h->b_state, &h->b_planes, &h->b_summ, &h->b_chunk,
                   &h->b_summp, &h->b_didx, &h->b_sidx, &h->b_slist, &h->b_dlist, &h->b_dpre, &h->b_out,
                   &h->b_a4, &h->b_counter, &h->b_sreq, &h->b_sout};
    for (Buf *b : bufs) if (b->p) cudaFree(b->p);
    if (h->pin) cudaFreeHost(h->pin);
    if (h->d_small) cudaFree(h->d_small);
    if (h->d_chain) cudaFree(h->d_chain);
    for (auto &e : h->ev) if (e) cudaEventDestroy(e);
    if (h->st) cudaStreamDestroy(h->st);
    delete h;
}

int handle_open(const cz_config *cfg, CZ_HANDLE **out) {
    if (!out) return CZ_EINVAL;
    *out = nullptr;
    CZ_HANDLE *h = new CZ_HANDLE();
    if (cfg) h->cfg = *cfg; else cz_default_config(&h->cfg);
    if (h->cfg.cover_n < 2 || h->cfg.cover_n > 8) { delete h; return CZ_EINVAL; }
    for (int r = 2; r <= 9; ++r)
        if (h->cfg.q_cap[r] && (h->cfg.q_cap[r] < 3 || h->cfg.q_cap[r] > 255)) { delete h; return CZ_EINVAL; }
    for (int r = 0; r < 10; ++r)
        if (h->cfg.anchor_t[r] && (h->cfg.anchor_t[r] < 2 || h->cfg.anchor_t[r] > 32)) { delete h; return CZ_EINVAL; }
    if (h->cfg.epoch_rows > (1u << 20)) { delete h; return CZ_EINVAL; }
    h->dev = h->cfg.device;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || h->dev < 0 || h->dev >= ndev) { delete h; return CZ_ECUDA; }
    cudaSetDevice(h->dev);
    cudaDeviceProp prop;
    cudaGetDeviceProperties(&prop, h->dev);
    h->sms = prop.multiProcessorCount;
    if (cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking) != cudaSuccess) { delete h; return CZ_ECUDA; }
    for (auto &e : h->ev) cudaEventCreate(&e);
    cudaFuncSetAttribute(table_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, TABLE_DYN_SMEM);
    cudaFuncSetAttribute(dense_scan_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 64 * 1024);
    // the filter stages its tiles in shared memory: the whole unified array
    // goes to shared memory, two CTAs of TILE_WORDS words each per SM
    cudaFuncSetAttribute(sparse_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(TILE_WORDS * 4u));
    cudaFuncSetAttribute(sparse_kernel, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    if (!build_static_tables(h)) { handle_close(h); return CZ_ECUDA; }
    *out = h;
    return CZ_OK;
}

// profiles of n primes: sum over primes of #{r in 2..9 : r | p - 1}
u32 count_profiles(const pw_t *primes, u32 n) {
    u32 c = 0;
    for (u32 i = 0; i < n; ++i)
        if (primes[i] > 2u) c += popc(mask_of(primes[i]));
    return c;
}

// plane-pool bytes one prime would take (0 for the dense route)
u64 plane_bytes(const cz_config &c, pw_t p, u32 flags) {
    if (p < 3u) return 0;
    const u32 mode = flags & CZ_AUTO;
    if (mode == CZ_DENSE || (mode == CZ_AUTO && p < c.sparse_min_p)) return 0;
    const u32 mask = mask_of(p);
    u32 Qmax = 0, units = 0;
    for (u32 r = 2; r <= 9; ++r)
        if (mask & (1u << (r - 2))) { Qmax = std::max(Qmax, q_for(c, r)); units += planes_stored(r); }
    u32 B = 0;
    if (Qmax + 1u >= p || !cover_B(p, Qmax, c.cover_n, B)) return 0;
    const u64 words = (2ull * ((B + 31u) / 32u + 4u) + 8ull) + (2ull * ((B + 63u) / 64u + 4u) + 8ull);
    return 4ull * words * units + 64ull * units;
}

int census_impl(CZ_HANDLE *h, const pw_t *primes, uint32_t n, uint32_t flags, CZ_RECORD *out,
                uint32_t out_cap, uint32_t *a4_out, cz_stats *stats, bool allow_fallback);

// a batch whose plane pool would exceed the budget runs as consecutive waves
int census_waves(CZ_HANDLE *h, const pw_t *primes, uint32_t n, uint32_t flags, CZ_RECORD *out,
                        uint32_t out_cap, uint32_t *a4_out, cz_stats *stats) {
    const u64 budget = (u64)h->cfg.plane_budget_mb << 20;
    u64 acc = 0;
    u32 start = 0, prof_off = 0, waves = 0;
    cz_stats tot{};
    for (u32 i = 0; i <= n; ++i) {
        const u64 b = i < n ? plane_bytes(h->cfg, primes[i], flags) : 0;
        if (i == n || (acc + b > budget && i > start)) {
            const u32 m = i - start;
            const u32 np = count_profiles(primes + start, m);
            cz_stats s{};
            int rc = census_impl(h, primes + start, m, flags, out + prof_off, out_cap - prof_off,
                                 a4_out ? a4_out + start : nullptr, &s, true);
            if (rc) return rc;
            ++waves;
            tot.ms_setup += s.ms_setup; tot.ms_table += s.ms_table; tot.ms_sparse += s.ms_sparse;
            tot.ms_dense += s.ms_dense; tot.ms_a4 += s.ms_a4; tot.ms_finalize += s.ms_finalize;
            tot.ms_device += s.ms_device; tot.ms_h2d += s.ms_h2d; tot.ms_d2h += s.ms_d2h;
            tot.n_dense += s.n_dense; tot.n_sparse += s.n_sparse; tot.n_profiles += s.n_profiles;
            tot.n_fallback += s.n_fallback; tot.n_respec += s.n_respec; tot.ms_respec += s.ms_respec;
            tot.kernels += s.kernels; tot.words += s.words; tot.completions += s.completions;
            tot.tests += s.tests; tot.h2d_bytes += s.h2d_bytes; tot.d2h_bytes += s.d2h_bytes;
            tot.staged_bytes += s.staged_bytes;
            prof_off += np;
            start = i;
            acc = 0;
        }
        acc += b;
    }
    tot.n_primes = n;
    tot.waves = waves;
    h->have_plan = waves == 1 && h->have_plan;
    if (stats) *stats = tot;
    return CZ_OK;
}

int census_impl(CZ_HANDLE *h, const pw_t *primes, uint32_t n, uint32_t flags, CZ_RECORD *out,
                       uint32_t out_cap, uint32_t *a4_out, cz_stats *stats, bool allow_fallback) {
    if (!h) return CZ_EINVAL;
    cudaSetDevice(h->dev);
    h->err.clear();
    cz_stats s{};
    if (n == 0) { if (stats) *stats = s; return CZ_OK; }
    if (!primes || !out || ((flags & CZ_A4) && !a4_out)) { h->err = "null buffer"; return CZ_EINVAL; }
    if ((flags & CZ_AUTO) == 0) flags |= CZ_AUTO;
    const u32 need = count_profiles(primes, n);
    if (out_cap < need) { h->err = "output capacity below profile count"; return CZ_EINVAL; }
    int rc = plan(h, primes, n, flags);
    if (rc) return rc;
    if (h->gexec) { cudaGraphExecDestroy(h->gexec); h->gexec = nullptr; }
    if (h->graph) { cudaGraphDestroy(h->graph); h->graph = nullptr; }
    cudaEvent_t t0, t1;
    cudaEventCreate(&t0); cudaEventCreate(&t1);
    cudaEventRecord(t0, h->st);
    if ((rc = upload(h, &s))) return rc;
    cudaEventRecord(t1, h->st);
    u32 launches = 0;
    if ((rc = enqueue(h, true, launches))) return rc;
    h->hout.resize(h->nprof);
    cudaEvent_t t2;
    cudaEventCreate(&t2);
    if (h->nprof && !ck(h, cudaMemcpyAsync(h->hout.data(), h->b_out.p, sizeof(OutRecord) * h->nprof,
                                           cudaMemcpyDeviceToHost, h->st), "d2h"))
        return CZ_ECUDA;
    if ((flags & CZ_A4) && !ck(h, cudaMemcpyAsync(a4_out, h->b_a4.p, 4ull * n, cudaMemcpyDeviceToHost, h->st), "d2h a4"))
        return CZ_ECUDA;
    cudaEventRecord(t2, h->st);
    if (!ck(h, cudaStreamSynchronize(h->st), "census")) return CZ_ECUDA;
    cudaEventElapsedTime(&s.ms_h2d, t0, t1);
    cudaEventElapsedTime(&s.ms_d2h, h->ev[6], t2);
    cudaEventDestroy(t0); cudaEventDestroy(t1); cudaEventDestroy(t2);
    read_times(h, &s);
    s.d2h_bytes = sizeof(OutRecord) * h->nprof + ((flags & CZ_A4) ? 4ull * n : 0ull);
    s.n_primes = n; s.n_dense = h->ndense; s.n_sparse = h->nsparse; s.n_profiles = h->nprof;
    s.kernels = launches;
    {
        std::vector<ProfState> hs(h->nprof);
        if (h->nprof) cudaMemcpy(hs.data(), h->b_state.p, sizeof(ProfState) * h->nprof, cudaMemcpyDeviceToHost);
        for (auto &x : hs) {
            s.words += x.words; s.completions += x.completions; s.tests += x.tests;
            s.staged_bytes += 16ull * x.staged16;
        }
    }
    // records first: a refusal names the prime and its status
    std::vector<u32> fb, rs;
    rc = check_records(h, allow_fallback ? &fb : nullptr, allow_fallback ? &rs : nullptr);
    if (rc) return rc;
    if (flags & CZ_A4) {
        u32 a4err = 0;
        cudaMemcpy(&a4err, P<u32>(h->b_counter) + 8, 4, cudaMemcpyDeviceToHost);
        if (a4err) { h->err = "refused: A4 point count not certified"; return CZ_EREFUSED; }
    }
    for (u32 g = 0; g < h->nprof; ++g) {
        const OutRecord &o = h->hout[g];
        CZ_RECORD &d = out[g];
        d.p = o.p; d.r = o.r; d.M = o.M; d.L = o.L; d.witness = o.witness; d.status = o.status; d.K = o.K;
    }
    // the re-runs below re-plan the handle: take the primes and record slots first
    std::vector<pw_t> fb_p;
    std::vector<u32> fb_first;
    for (u32 pi : fb) { fb_p.push_back(h->hp[pi].p); fb_first.push_back(h->hp[pi].first_prof); }
    if (!rs.empty()) {
        // profiles whose best run stayed below the speculative threshold: the
        // speculation was not certified, re-run those primes without it
        std::vector<pw_t> sub;
        for (u32 pi : rs) sub.push_back(h->hp[pi].p);
        std::vector<u32> first(rs.size());
        for (size_t k = 0; k < rs.size(); ++k) first[k] = h->hp[rs[k]].first_prof;
        const u32 fflags = (flags & ~CZ_A4) | CZ_NOSPEC;
        std::vector<CZ_RECORD> tmp(count_profiles(sub.data(), (u32)sub.size()));
        cz_stats s2{};
        rc = census_impl(h, sub.data(), (u32)sub.size(), fflags, tmp.data(), (u32)tmp.size(), nullptr, &s2, true);
        if (rc) return rc;
        u32 t = 0;
        for (size_t k = 0; k < rs.size(); ++k) {
            const u32 np = popc(mask_of(sub[k]));
            for (u32 j = 0; j < np; ++j) out[first[k] + j] = tmp[t++];
        }
        s.n_respec = (u32)rs.size();
        s.ms_respec = s2.ms_device;
        h->have_plan = false;
    }
    if (!fb.empty()) {
        // sparse primes whose seed could not certify a threshold: dense re-run
        const std::vector<pw_t> &sub = fb_p;
        const std::vector<u32> &first = fb_first;
        const u32 fflags = (flags & ~CZ_AUTO & ~CZ_A4) | CZ_DENSE;
        std::vector<CZ_RECORD> tmp(count_profiles(sub.data(), (u32)sub.size()));
        cz_stats s2{};
        rc = census_impl(h, sub.data(), (u32)sub.size(), fflags, tmp.data(), (u32)tmp.size(), nullptr, &s2, false);
        if (rc) return rc;
        u32 t = 0;
        for (size_t k = 0; k < fb.size(); ++k) {
            const u32 np = popc(mask_of(sub[k]));
            for (u32 j = 0; j < np; ++j) out[first[k] + j] = tmp[t++];
        }
        s.n_fallback = (u32)fb.size();
        h->have_plan = false;   // the plan now describes the fallback batch
    }
    h->last = s;
    if (stats) *stats = s;
    return CZ_OK;
}

// a census call: waves when the plane pool of the batch exceeds its budget
int census_entry(CZ_HANDLE *h, const pw_t *primes, uint32_t n, uint32_t flags, CZ_RECORD *out,
                 uint32_t out_cap, uint32_t *a4_out, cz_stats *stats) {
    if (!h) return CZ_EINVAL;
    if (n && primes && out && ((flags & CZ_A4) == 0 || a4_out)) {
        if ((flags & CZ_AUTO) == 0) flags |= CZ_AUTO;
        if (out_cap < count_profiles(primes, n)) { h->err = "output capacity below profile count"; return CZ_EINVAL; }
        u64 tot = 0;
        for (u32 i = 0; i < n && tot <= ((u64)h->cfg.plane_budget_mb << 20); ++i) tot += plane_bytes(h->cfg, primes[i], flags);
        if (tot > ((u64)h->cfg.plane_budget_mb << 20)) return census_waves(h, primes, n, flags, out, out_cap, a4_out, stats);
    }
    int rc = census_impl(h, primes, n, flags, out, out_cap, a4_out, stats, true);
    if (!rc && stats) stats->waves = 1;
    return rc;
}

}  // namespace
