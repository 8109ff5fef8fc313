// census.cu -- host orchestration and C ABI of librabung_census.so.
//
// One call (cz_census) takes a batch of primes through:
//   plan (host, O(n)): admissible orders, route (dense / sparse), cover
//     (B, D_r, Q_r) by the integer certificate, plane and summary layout;
//   setup_kernel: primality, Montgomery constants, roots of unity;
//   table_kernel + sparse_kernel: signed planes, persistent anchor filter;
//   dense_scan_kernel + dense_merge_kernel: exhaustive half-interval scan;
//   finalize_kernel: prefix, optional direct certification, K, records;
//   a4_kernel: quadratic A4 counts.
// The device work of the last call can be replayed on resident inputs
// (cz_replay), optionally through a captured CUDA graph.  runtime.cuh,
// included at the end, adds the
// interval census and the serving runtime on top of these entry points.
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
#include "microbench.cuh"
#include "sieve.cuh"
#include "../../include/rabung_census.h"

using namespace cz;

namespace {

constexpr u32 CHAIN_LIMIT = (1u << 20) + 8192u;   // table labels cover n < CHAIN_LIMIT
constexpr u32 B_MAX = (1u << 20);
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
bool cover_B(u32 p, u32 Q, u32 ndiv, u32 &Bout) {
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
bool cover_D(u32 p, u32 B, u32 Q, u32 &Dout) {
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

struct cz_handle {
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

bool ck(cz_handle *h, cudaError_t e, const char *what) {
    if (e == cudaSuccess) return true;
    h->err = std::string(what) + ": " + cudaGetErrorString(e);
    return false;
}

bool ensure(cz_handle *h, Buf &b, size_t bytes) {
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

bool build_static_tables(cz_handle *h) {
    // primes below CHAIN_LIMIT and the smallest-prime-factor chain
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
    for (u32 n = 2; n < CHAIN_LIMIT; ++n) chain[n] = make_uint2(index[spf[n]], n / spf[n]);
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
u32 qspec_for(const cz_config &c, u32 p, u32 r, bool allow) {
    if (!allow || !c.speculate) return 0u;
    const double lg = std::log((double)p) / std::log((double)r);
    const double m = c.spec_margin10[r] / 10.0;
    const double v = std::floor(lg - m);
    return v < 3.0 ? 0u : (u32)v;
}

// host plan of one call
constexpr u32 CZ_NOSPEC = 1u << 16;      // internal: plan without speculative thresholds

int plan(cz_handle *h, const u32 *primes, u32 n, u32 flags) {
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
        const u32 p = primes[i];
        if (p < 2u) { h->err = "prime out of domain: " + std::to_string(p); return CZ_EINVAL; }
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
            const u32 nh = (p - 1u) / 2u;
            const u32 seg = dense_seg(c);
            const u32 nseg = (nh + seg - 1u) / seg;
            const u32 nch = (nseg + DENSE_WARPS - 1u) / DENSE_WARPS;
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
    h->table_smem = max_slots_t * 6u + 8u + max_nq * 2u + 16u;
    if (h->table_smem > TABLE_DYN_SMEM) {
        h->err = "table shared memory above the per-block limit";
        return CZ_EINVAL;
    }
    h->dense_smem = max_slots_d * 6u + 16u;
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

int upload(cz_handle *h, cz_stats *s) {
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
int enqueue(cz_handle *h, bool timed, u32 &launches) {
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
        SparseArgs sa;
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

void read_times(cz_handle *h, cz_stats *s) {
    float t[6] = {0};
    for (int i = 0; i < 6; ++i) cudaEventElapsedTime(&t[i], h->ev[i], h->ev[i + 1]);
    s->ms_setup = t[0]; s->ms_table = t[1]; s->ms_sparse = t[2]; s->ms_dense = t[3];
    s->ms_finalize = t[4]; s->ms_a4 = t[5];
    cudaEventElapsedTime(&s->ms_device, h->ev[0], h->ev[6]);
}

int check_records(cz_handle *h, std::vector<u32> *fallback, std::vector<u32> *respec = nullptr) {
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
            snprintf(buf, sizeof buf, "refused: p=%u r=%u status=0x%x", o.p, o.r, o.status);
            h->err = buf;
            return CZ_EREFUSED;
        }
    }
    return CZ_OK;
}

}  // namespace

extern "C" {

int cz_default_config(cz_config *c) {
    if (!c) return CZ_EINVAL;
    std::memset(c, 0, sizeof *c);
    c->device = 0;
    c->sparse_min_p = 1u << 20;
    c->cover_n = 3;
    const u32 q[10] = {0, 0, 30, 24, 20, 16, 16, 15, 14, 13};
    for (int r = 0; r < 10; ++r) c->q_cap[r] = q[r];
    c->anchor_bits = 4;
    c->screen = 1;
    c->sparse_blocks = 0;
    c->use_graph = 1;
    c->cta_per_profile = 2;
    c->epoch_rows = EPOCH_ROWS_DEFAULT;
    c->speculate = 1;
    c->plane_budget_mb = 24u * 1024u;
    c->dense_steps = DENSE_STEPS;
    const u32 sm[10] = {0, 0, 30, 20, 15, 15, 10, 0, 5, 10};   // measured per order
    for (int r = 0; r < 10; ++r) c->spec_margin10[r] = sm[r];
    const u32 at[10] = {0, 0, 11, 7, 6, 5, 4, 4, 4, 4};   // measured per order on a top block
    for (int r = 0; r < 10; ++r) c->anchor_t[r] = at[r];
    return CZ_OK;
}

int cz_open(const cz_config *cfg, cz_handle **out) {
    if (!out) return CZ_EINVAL;
    *out = nullptr;
    cz_handle *h = new cz_handle();
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
    cudaFuncSetAttribute(sieve_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, SIEVE_MAX_WIDTH / 16 + 64);
    // the filter stages its tiles in shared memory: the whole unified array
    // goes to shared memory, two CTAs of TILE_WORDS words each per SM
    cudaFuncSetAttribute(sparse_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(TILE_WORDS * 4u));
    cudaFuncSetAttribute(sparse_kernel, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    if (!build_static_tables(h)) { cz_close(h); return CZ_ECUDA; }
    *out = h;
    return CZ_OK;
}

void cz_close(cz_handle *h) {
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

const char *cz_last_error(const cz_handle *h) { return h ? h->err.c_str() : "null handle"; }

uint32_t cz_count_profiles(const uint32_t *primes, uint32_t n) {
    u32 c = 0;
    for (u32 i = 0; i < n; ++i)
        if (primes[i] > 2u) c += popc(mask_of(primes[i]));
    return c;
}

// plane-pool bytes one prime would take (0 for the dense route)
static u64 plane_bytes(const cz_config &c, u32 p, u32 flags) {
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

static int census_impl(cz_handle *h, const uint32_t *primes, uint32_t n, uint32_t flags, cz_profile *out,
                       uint32_t out_cap, uint32_t *a4_out, cz_stats *stats, bool allow_fallback);

// a batch whose plane pool would exceed the budget runs as consecutive waves
static int census_waves(cz_handle *h, const uint32_t *primes, uint32_t n, uint32_t flags, cz_profile *out,
                        uint32_t out_cap, uint32_t *a4_out, cz_stats *stats) {
    const u64 budget = (u64)h->cfg.plane_budget_mb << 20;
    u64 acc = 0;
    u32 start = 0, prof_off = 0, waves = 0;
    cz_stats tot{};
    for (u32 i = 0; i <= n; ++i) {
        const u64 b = i < n ? plane_bytes(h->cfg, primes[i], flags) : 0;
        if (i == n || (acc + b > budget && i > start)) {
            const u32 m = i - start;
            const u32 np = cz_count_profiles(primes + start, m);
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

static int census_impl(cz_handle *h, const uint32_t *primes, uint32_t n, uint32_t flags, cz_profile *out,
                       uint32_t out_cap, uint32_t *a4_out, cz_stats *stats, bool allow_fallback) {
    if (!h) return CZ_EINVAL;
    cudaSetDevice(h->dev);
    h->err.clear();
    cz_stats s{};
    if (n == 0) { if (stats) *stats = s; return CZ_OK; }
    if (!primes || !out || ((flags & CZ_A4) && !a4_out)) { h->err = "null buffer"; return CZ_EINVAL; }
    if ((flags & CZ_AUTO) == 0) flags |= CZ_AUTO;
    const u32 need = cz_count_profiles(primes, n);
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
        for (auto &x : hs) { s.words += x.words; s.completions += x.completions; s.tests += x.tests; }
    }
    if (flags & CZ_A4) {
        u32 a4err = 0;
        cudaMemcpy(&a4err, P<u32>(h->b_counter) + 8, 4, cudaMemcpyDeviceToHost);
        if (a4err) { h->err = "refused: A4 point count not certified"; return CZ_EREFUSED; }
    }
    std::vector<u32> fb, rs;
    rc = check_records(h, allow_fallback ? &fb : nullptr, allow_fallback ? &rs : nullptr);
    if (rc) return rc;
    for (u32 g = 0; g < h->nprof; ++g) {
        const OutRecord &o = h->hout[g];
        cz_profile &d = out[g];
        d.p = o.p; d.r = o.r; d.M = o.M; d.L = o.L; d.witness = o.witness; d.status = o.status; d.K = o.K;
    }
    // the re-runs below re-plan the handle: take the primes and record slots first
    std::vector<u32> fb_p, fb_first;
    for (u32 pi : fb) { fb_p.push_back(h->hp[pi].p); fb_first.push_back(h->hp[pi].first_prof); }
    if (!rs.empty()) {
        // profiles whose best run stayed below the speculative threshold: the
        // speculation was not certified, re-run those primes without it
        std::vector<u32> sub;
        for (u32 pi : rs) sub.push_back(h->hp[pi].p);
        std::vector<u32> first(rs.size());
        for (size_t k = 0; k < rs.size(); ++k) first[k] = h->hp[rs[k]].first_prof;
        const u32 fflags = (flags & ~CZ_A4) | CZ_NOSPEC;
        std::vector<cz_profile> tmp(cz_count_profiles(sub.data(), (u32)sub.size()));
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
        const std::vector<u32> &sub = fb_p, &first = fb_first;
        const u32 fflags = (flags & ~CZ_AUTO & ~CZ_A4) | CZ_DENSE;
        std::vector<cz_profile> tmp(cz_count_profiles(sub.data(), (u32)sub.size()));
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

int cz_census(cz_handle *h, const uint32_t *primes, uint32_t n, uint32_t flags, cz_profile *out,
              uint32_t out_cap, uint32_t *a4_out, cz_stats *stats) {
    if (!h) return CZ_EINVAL;
    if (n && primes && out && ((flags & CZ_A4) == 0 || a4_out)) {
        if ((flags & CZ_AUTO) == 0) flags |= CZ_AUTO;
        if (out_cap < cz_count_profiles(primes, n)) { h->err = "output capacity below profile count"; return CZ_EINVAL; }
        u64 tot = 0;
        for (u32 i = 0; i < n && tot <= ((u64)h->cfg.plane_budget_mb << 20); ++i) tot += plane_bytes(h->cfg, primes[i], flags);
        if (tot > ((u64)h->cfg.plane_budget_mb << 20)) return census_waves(h, primes, n, flags, out, out_cap, a4_out, stats);
    }
    int rc = census_impl(h, primes, n, flags, out, out_cap, a4_out, stats, true);
    if (!rc && stats) stats->waves = 1;
    return rc;
}

uint64_t cz_plane_bytes(const cz_handle *h, const uint32_t *primes, uint32_t n, uint32_t flags) {
    if (!h || !primes) return 0;
    if ((flags & CZ_AUTO) == 0) flags |= CZ_AUTO;
    u64 t = 0;
    for (u32 i = 0; i < n; ++i) t += plane_bytes(h->cfg, primes[i], flags);
    return t;
}

int cz_device_info(cz_handle *h, char *name, uint32_t len, uint32_t *sms) {
    if (!h || !name || !len || !sms) return CZ_EINVAL;
    cudaDeviceProp prop;
    if (!ck(h, cudaGetDeviceProperties(&prop, h->dev), "device properties")) return CZ_ECUDA;
    snprintf(name, len, "%s", prop.name);
    *sms = (uint32_t)prop.multiProcessorCount;
    return CZ_OK;
}

int cz_mem_info(cz_handle *h, uint64_t *free_bytes, uint64_t *total_bytes) {
    if (!h || !free_bytes || !total_bytes) return CZ_EINVAL;
    cudaSetDevice(h->dev);
    size_t f = 0, t = 0;
    if (!ck(h, cudaMemGetInfo(&f, &t), "cudaMemGetInfo")) return CZ_ECUDA;
    *free_bytes = f;
    *total_bytes = t;
    return CZ_OK;
}

int cz_replay(cz_handle *h, cz_stats *stats) {
    if (!h || !h->have_plan) { if (h) h->err = "no resident plan to replay"; return CZ_EINVAL; }
    cudaSetDevice(h->dev);
    cz_stats s{};
    u32 launches = 0;
    int rc;
    if (h->cfg.use_graph) {
        if (!h->gexec) {
            if (!ck(h, cudaStreamBeginCapture(h->st, cudaStreamCaptureModeThreadLocal), "capture")) return CZ_ECUDA;
            rc = enqueue(h, false, launches);
            cudaGraph_t g = nullptr;
            cudaError_t e = cudaStreamEndCapture(h->st, &g);
            if (rc || !ck(h, e, "end capture")) return CZ_ECUDA;
            h->graph = g;
            if (!ck(h, cudaGraphInstantiate(&h->gexec, g, 0), "instantiate")) return CZ_ECUDA;
        } else {
            rc = CZ_OK;
        }
        cudaEventRecord(h->ev[0], h->st);
        if (!ck(h, cudaGraphLaunch(h->gexec, h->st), "graph launch")) return CZ_ECUDA;
        cudaEventRecord(h->ev[6], h->st);
        if (!ck(h, cudaStreamSynchronize(h->st), "replay")) return CZ_ECUDA;
        cudaEventElapsedTime(&s.ms_device, h->ev[0], h->ev[6]);
        launches = h->last.kernels;
    } else {
        if ((rc = enqueue(h, true, launches))) return rc;
        if (!ck(h, cudaStreamSynchronize(h->st), "replay")) return CZ_ECUDA;
        read_times(h, &s);
    }
    s.kernels = launches;
    s.n_primes = h->n; s.n_dense = h->ndense; s.n_sparse = h->nsparse; s.n_profiles = h->nprof;
    // results must still pass every status check
    h->hout.resize(h->nprof);
    if (h->nprof) cudaMemcpy(h->hout.data(), h->b_out.p, sizeof(OutRecord) * h->nprof, cudaMemcpyDeviceToHost);
    if ((rc = check_records(h, nullptr))) return rc;
    if (stats) *stats = s;
    return CZ_OK;
}

int cz_sieve(cz_handle *h, const uint32_t *lo, const uint32_t *count, uint32_t n, uint32_t *out,
             uint32_t *found) {
    if (!h || (n && (!lo || !count || !out || !found))) return CZ_EINVAL;
    cudaSetDevice(h->dev);
    h->err.clear();
    if (n == 0) return CZ_OK;
    std::vector<SieveReq> rq(n);
    u64 total = 0;
    for (u32 i = 0; i < n; ++i) {
        rq[i] = SieveReq{};
        rq[i].lo = lo[i];
        rq[i].count = count[i];
        rq[i].out_off = (u32)total;
        total += count[i];
        // prime number theorem with slack; widened below if a window comes up short
        const double ln = std::log(std::max(16.0, (double)lo[i] + 1.0));
        const u64 w = (u64)(count[i] * ln * 1.3) + 4096ull;
        const u64 room = (1ull << 32) - lo[i];
        rq[i].width = (u32)std::min<u64>({w, (u64)SIEVE_MAX_WIDTH, room});
        found[i] = 0;
    }
    if (total > 0xFFFFFFFFull) { h->err = "sieve output too large"; return CZ_EINVAL; }
    if (!ensure(h, h->b_sreq, sizeof(SieveReq) * n) || !ensure(h, h->b_sout, 4ull * std::max<u64>(1, total)))
        return CZ_ECUDA;
    std::vector<u32> todo(n);
    for (u32 i = 0; i < n; ++i) todo[i] = i;
    for (int round = 0; round < 24 && !todo.empty(); ++round) {
        std::vector<SieveReq> sub;
        for (u32 i : todo) sub.push_back(rq[i]);
        cudaMemcpyAsync(h->b_sreq.p, sub.data(), sizeof(SieveReq) * sub.size(), cudaMemcpyHostToDevice, h->st);
        const u32 grid = std::min<u32>((u32)sub.size(), (u32)h->sms);
        sieve_kernel<<<grid, SIEVE_THREADS, SIEVE_MAX_WIDTH / 16 + 64, h->st>>>(P<SieveReq>(h->b_sreq), (u32)sub.size(),
                                                                              h->d_small, h->n_small, P<u32>(h->b_sout));
        cudaMemcpyAsync(sub.data(), h->b_sreq.p, sizeof(SieveReq) * sub.size(), cudaMemcpyDeviceToHost, h->st);
        if (!ck(h, cudaStreamSynchronize(h->st), "sieve")) return CZ_ECUDA;
        std::vector<u32> next;
        for (size_t k = 0; k < todo.size(); ++k) {
            SieveReq &R = rq[todo[k]];
            R.found = sub[k].found;
            const bool at_top = (u64)R.lo + R.width >= (1ull << 32);
            if (R.found < R.count && !at_top) {
                // too few primes in the window: widen it (the output slots are unchanged)
                const u64 room = (1ull << 32) - R.lo;
                const u64 w = std::min<u64>({(u64)R.width * 2ull, (u64)SIEVE_MAX_WIDTH, room});
                if (w == R.width) { h->err = "sieve window limit reached"; return CZ_EINVAL; }
                R.width = (u32)w;
                next.push_back(todo[k]);
            }
        }
        todo.swap(next);
    }
    if (!todo.empty()) { h->err = "sieve did not converge"; return CZ_EREFUSED; }
    if (total && !ck(h, cudaMemcpy(out, h->b_sout.p, 4ull * total, cudaMemcpyDeviceToHost), "sieve d2h")) return CZ_ECUDA;
    for (u32 i = 0; i < n; ++i) found[i] = rq[i].found;
    h->have_plan = false;
    return CZ_OK;
}

int cz_a4(cz_handle *h, const uint32_t *primes, uint32_t n, uint32_t *a4_out) {
    if (!h || !primes || !a4_out) return CZ_EINVAL;
    std::vector<u32> cnt(n);
    // reuse the census path with an all-dense plan restricted to A4
    cudaSetDevice(h->dev);
    h->err.clear();
    std::vector<PrimeDesc> hp(n);
    for (u32 i = 0; i < n; ++i) {
        if (primes[i] < 2u) { h->err = "prime out of domain"; return CZ_EINVAL; }
        hp[i] = PrimeDesc{};
        hp[i].p = primes[i];
    }
    if (!ensure(h, h->b_primes, sizeof(PrimeDesc) * n) || !ensure(h, h->b_a4, 4ull * n) || !ensure(h, h->b_counter, 64))
        return CZ_ECUDA;
    cudaMemcpyAsync(h->b_primes.p, hp.data(), sizeof(PrimeDesc) * n, cudaMemcpyHostToDevice, h->st);
    cudaMemsetAsync(h->b_counter.p, 0, 64, h->st);
    a4_kernel<<<(n + A4_WARPS - 1) / A4_WARPS, A4_WARPS * 32, 0, h->st>>>(P<PrimeDesc>(h->b_primes), n,
                                                                      P<u32>(h->b_a4), P<u32>(h->b_counter) + 8);
    cudaMemcpyAsync(a4_out, h->b_a4.p, 4ull * n, cudaMemcpyDeviceToHost, h->st);
    u32 err = 0;
    cudaMemcpyAsync(&err, P<u32>(h->b_counter) + 8, 4, cudaMemcpyDeviceToHost, h->st);
    if (!ck(h, cudaStreamSynchronize(h->st), "a4")) return CZ_ECUDA;
    if (err) { h->err = "refused: A4 point count not certified"; return CZ_EREFUSED; }
    h->have_plan = false;
    return CZ_OK;
}

int cz_microbench(cz_handle *h, uint32_t kind, double *per_second) {
    if (!h || !per_second || kind > 1) return CZ_EINVAL;
    cudaSetDevice(h->dev);
    if (!ensure(h, h->b_counter, 64)) return CZ_ECUDA;
    const u32 blocks = (u32)h->sms * 8u, threads = 256, iters = kind == 0 ? 4096u : 1024u;
    const u32 p = 4294967291u;
    const Mont M = make_mont(p);
    float best = 1e30f;
    for (int rep = 0; rep < 4; ++rep) {
        cudaEventRecord(h->ev[0], h->st);
        if (kind == 0) mb_alu_kernel<<<blocks, threads, 0, h->st>>>(iters, 0x9E3779B9u + rep, P<u32>(h->b_counter));
        else mb_mont_kernel<<<blocks, threads, 0, h->st>>>(iters, p, M.ninv, P<u32>(h->b_counter));
        cudaEventRecord(h->ev[1], h->st);
        if (!ck(h, cudaStreamSynchronize(h->st), "microbench")) return CZ_ECUDA;
        float ms = 0;
        cudaEventElapsedTime(&ms, h->ev[0], h->ev[1]);
        if (rep > 0 && ms < best) best = ms;
    }
    *per_second = (double)blocks * threads * iters * 8.0 / (best * 1e-3);
    return CZ_OK;
}

// ---- dense census without device allocation ---------------------------------
//
// Some callers cannot call cudaMalloc: plugins inside a host process that owns
// the device's memory budget, and allocator-free services that must not grow
// their device footprint after start-up.  cz_census_dense_noalloc serves them.
// Its only device scratch is the file-scope array below (NOALLOC_BYTES, held by
// every GPU that loads this library until the process exits); descriptors, run
// summaries, per-profile state and output records are carved out of it.  The
// host side uses fixed stack arrays only.  The call is synchronous: it returns
// after its stream has finished.  Calls share the array: two calls that overlap
// on the GPU (different streams, or different host threads) race.

constexpr u32 NOALLOC_BYTES = 2u << 20;          // 2 MiB
constexpr u32 NOALLOC_MAX_PRIMES = 64;
constexpr u32 NOALLOC_MAX_P = 1u << 22;          // p < 4,194,304
constexpr u32 NOALLOC_MAX_PROFILES = NOALLOC_MAX_PRIMES * 8u;
// chunks per profile for p < 2^22: ceil(ceil(2^21 / DENSE_SEG) / DENSE_WARPS)
constexpr u32 NOALLOC_MAX_CHUNKS = ((1u << 21) / DENSE_SEG + DENSE_WARPS - 1u) / DENSE_WARPS;

static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_BYTES];

namespace {

struct NoallocLayout {      // byte offsets inside the scratch array (256-aligned)
    size_t primes, profs, state, chunk, summp, didx, dlist, dpre, out, summ, end;
};

constexpr size_t al256(size_t x) { return (x + 255) & ~size_t(255); }

constexpr NoallocLayout noalloc_layout() {
    NoallocLayout L{};
    size_t o = 0;
    L.primes = o; o = al256(o + sizeof(PrimeDesc) * NOALLOC_MAX_PRIMES);
    L.profs = o;  o = al256(o + sizeof(ProfDesc) * NOALLOC_MAX_PROFILES);
    L.state = o;  o = al256(o + sizeof(ProfState) * NOALLOC_MAX_PROFILES);
    L.chunk = o;  o = al256(o + 4 * (NOALLOC_MAX_PRIMES + 1));
    L.summp = o;  o = al256(o + 4 * NOALLOC_MAX_PRIMES);
    L.didx = o;   o = al256(o + 4 * NOALLOC_MAX_PRIMES);
    L.dlist = o;  o = al256(o + 4 * NOALLOC_MAX_PROFILES);
    L.dpre = o;   o = al256(o + 4 * NOALLOC_MAX_PROFILES);
    L.out = o;    o = al256(o + sizeof(OutRecord) * NOALLOC_MAX_PROFILES);
    L.summ = o;   o = al256(o + sizeof(Summ) * NOALLOC_MAX_PROFILES * NOALLOC_MAX_CHUNKS);
    L.end = o;
    return L;
}
static_assert(noalloc_layout().end <= NOALLOC_BYTES, "static scratch too small for its limits");

// Set-up for the current device: the device address of the scratch array (the
// host-side name of the array is only a stand-in for the symbol, never a device
// address) and the dense kernel's shared-memory limit.  Resolved on every call
// with the caller's device current, so the address stays right after a
// cudaDeviceReset reloads the module; both steps are cheap lookups.
int noalloc_setup(unsigned char **out) {
    void *ptr = nullptr;
    if (cudaGetSymbolAddress(&ptr, g_noalloc_scratch) != cudaSuccess || !ptr) return CZ_ECUDA;
    if (cudaFuncSetAttribute(dense_scan_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 64 * 1024) !=
        cudaSuccess)
        return CZ_ECUDA;
    *out = static_cast<unsigned char *>(ptr);
    return CZ_OK;
}

}  // namespace

extern "C" int cz_census_dense_noalloc(const uint32_t *primes, uint32_t n, cz_profile *out, uint32_t out_cap,
                                       void *stream) {
    if (n == 0) return CZ_OK;
    if (!primes || !out) return CZ_EINVAL;
    if (n > NOALLOC_MAX_PRIMES) return CZ_ELIMIT;
    // host plan on fixed arrays (the dense route of plan())
    PrimeDesc hp[NOALLOC_MAX_PRIMES];
    ProfDesc hprof[NOALLOC_MAX_PROFILES];
    u32 chunk[NOALLOC_MAX_PRIMES + 1], summp[NOALLOC_MAX_PRIMES], didx[NOALLOC_MAX_PRIMES];
    u32 dlist[NOALLOC_MAX_PROFILES];
    u32 nprof = 0, nd = 0, summ_slots = 0;
    chunk[0] = 0;
    for (u32 i = 0; i < n; ++i) {
        const u32 p = primes[i];
        if (p < 2u) return CZ_EINVAL;
        if (p >= NOALLOC_MAX_P) return CZ_ELIMIT;
        PrimeDesc P{};
        P.p = p;
        P.mask = p > 2u ? mask_of(p) : 0u;
        P.m = lcm_of_mask(P.mask);
        P.e = P.mask ? (p - 1u) / P.m : 0u;
        P.first_prof = nprof;
        P.nprof = popc(P.mask);
        P.route = P.nprof ? 1u : 0u;
        if (P.nprof) {
            const u32 nh = (p - 1u) / 2u;
            const u32 nseg = (nh + DENSE_SEG - 1u) / DENSE_SEG;
            const u32 nch = (nseg + DENSE_WARPS - 1u) / DENSE_WARPS;
            didx[nd] = i;
            summp[nd] = summ_slots;
            summ_slots += nch * P.nprof;
            chunk[nd + 1] = chunk[nd] + nch;
            for (u32 r = 2; r <= 9; ++r) {
                if (!(P.mask & (1u << (r - 2)))) continue;
                ProfDesc D{};
                D.prime = i; D.r = r; D.np = planes_for(r); D.npp = planes_stored(r);
                D.out_slot = nprof; D.local = nd;
                dlist[nprof] = nprof;
                hprof[nprof++] = D;
            }
            ++nd;
        }
        hp[i] = P;
    }
    if (out_cap < nprof) return CZ_EINVAL;
    if (nprof == 0) return CZ_OK;
    unsigned char *base = nullptr;
    int rc = noalloc_setup(&base);
    if (rc) return rc;
    constexpr NoallocLayout L = noalloc_layout();
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    auto h2d = [&](size_t off, const void *src, size_t bytes) {
        return cudaMemcpyAsync(base + off, src, bytes, cudaMemcpyHostToDevice, st) == cudaSuccess;
    };
    if (!h2d(L.primes, hp, sizeof(PrimeDesc) * n) || !h2d(L.profs, hprof, sizeof(ProfDesc) * nprof) ||
        !h2d(L.chunk, chunk, 4ull * (nd + 1)) || !h2d(L.summp, summp, 4ull * nd) || !h2d(L.didx, didx, 4ull * nd) ||
        !h2d(L.dlist, dlist, 4ull * nprof))
        return CZ_ECUDA;
    PrimeDesc *dP = reinterpret_cast<PrimeDesc *>(base + L.primes);
    ProfDesc *dD = reinterpret_cast<ProfDesc *>(base + L.profs);
    ProfState *dS = reinterpret_cast<ProfState *>(base + L.state);
    // setup_kernel re-initialises every ProfState this call uses
    if (!launch(setup_kernel, dim3((n + 127) / 128), dim3(128), 0, st, dP, dD, dS, n)) return CZ_ECUDA;
    u32 max_slots = 8;
    for (u32 i = 0; i < n; ++i) max_slots = std::max(max_slots, hash_slots(hp[i].m));
    DenseArgs da;
    da.primes = dP;
    da.dense_idx = reinterpret_cast<u32 *>(base + L.didx);
    da.profs = dD;
    da.chunk_prefix = reinterpret_cast<u32 *>(base + L.chunk);
    da.summ_prefix = reinterpret_cast<u32 *>(base + L.summp);
    da.nprimes = nd;
    da.nchunks = chunk[nd];
    da.summ = reinterpret_cast<Summ *>(base + L.summ);
    da.state = dS;
    da.seg = DENSE_SEG;
    if (!launch(dense_scan_kernel, dim3(std::max(1u, std::min(chunk[nd], 1184u))), dim3(DENSE_WARPS * 32),
                max_slots * 6u + 16u, st, da))
        return CZ_ECUDA;
    DenseMergeArgs ma;
    ma.primes = dP;
    ma.profs = dD;
    ma.chunk_prefix = da.chunk_prefix;
    ma.summ_prefix = da.summ_prefix;
    ma.nprimes = nd;
    ma.summ = da.summ;
    ma.state = dS;
    ma.prefix_out = reinterpret_cast<u32 *>(base + L.dpre);
    const u32 *dl = reinterpret_cast<const u32 *>(base + L.dlist);
    if (!launch(dense_merge_kernel, dim3((nprof + 7) / 8), dim3(256), 0, st, ma, dl, nprof)) return CZ_ECUDA;
    OutRecord *dO = reinterpret_cast<OutRecord *>(base + L.out);
    const u32 *dpre = ma.prefix_out;
    if (!launch(finalize_kernel, dim3((nprof + 127) / 128), dim3(128), 0, st, (const PrimeDesc *)dP,
                (const ProfDesc *)dD, (const ProfState *)dS, dpre, nprof, 0u, dO))
        return CZ_ECUDA;
    static_assert(sizeof(OutRecord) == sizeof(cz_profile), "record layout");
    if (cudaMemcpyAsync(out, dO, sizeof(OutRecord) * nprof, cudaMemcpyDeviceToHost, st) != cudaSuccess)
        return CZ_ECUDA;
    if (cudaStreamSynchronize(st) != cudaSuccess) return CZ_ECUDA;
    for (u32 g = 0; g < nprof; ++g)
        if (out[g].status) return CZ_EREFUSED;
    return CZ_OK;
}

// ---- reference-compatible adapter -------------------------------------------
//
// The reference's only in-process C ABI (src/census/engine32/src/baseline_bridge.cu:7,21-27):
// with full = 0 it serves exactly the order sets {2}, {2,4}, {3,6}, {2,3,6} and
// {2,3,4,6} (masks 1, 5, 18, 19, 23) and returns 2 for any other mask; with
// full = 1 it profiles every admissible order and reports those in the mask.
// Here the same rule holds, and a mask naming an order that does not divide
// p - 1 is refused with 2 as well (the reference reads an undefined colouring
// there).  cap (the reference's largest p, which sizes its buffers) is not
// needed: the handle grows its buffers on demand.
static cz_handle *g_base = nullptr;
static std::mutex g_base_mu;

void baseline_init(unsigned cap) {
    (void)cap;
    std::lock_guard<std::mutex> lk(g_base_mu);
    if (!g_base) cz_open(nullptr, &g_base);
}

int baseline_profile(unsigned p, unsigned mask, unsigned *out, unsigned *prefix, int full) {
    if (!full && mask != 1u && mask != 5u && mask != 18u && mask != 19u && mask != 23u) return 2;
    if (!out || !prefix || p < 3u) return 2;
    const u32 adm = mask_of(p);
    if (mask & ~adm) return 2;
    baseline_init(0);
    std::lock_guard<std::mutex> lk(g_base_mu);
    if (!g_base) return 2;
    std::vector<cz_profile> rec(popc(adm));
    u32 pp = p;
    if (cz_census(g_base, &pp, 1, CZ_AUTO | CZ_VERIFY, rec.data(), (u32)rec.size(), nullptr, nullptr)) return 2;
    for (const cz_profile &v : rec)
        if (mask & (1u << (v.r - 2))) { out[v.r] = v.M; prefix[v.r] = v.L; }
    return 0;
}

// ---- exact prime counts on the host -----------------------------------------
//
// pi(x) by the Lucy-Hedgehog recursion over the values floor(x / k): S(v)
// starts at v - 1 and, for each prime q <= sqrt(x) in turn, every v >= q^2
// loses S(v / q) - S(q - 1) (the integers whose least prime factor is q);
// O(x^(3/4)) time, O(sqrt x) memory -- a few ms at x = 2^32.  It plays the
// role of the reference's Meissel-Lehmer count (src/census/prime_count.cpp:11-24):
// interval buffers are sized exactly in one pass, without sieving ahead.
// Short intervals are counted by a segmented sieve instead.

namespace {

u64 isqrt64(u64 x) {
    u64 r = (u64)std::sqrt((double)x);
    while (r * r > x) --r;
    while ((r + 1) * (r + 1) <= x) ++r;
    return r;
}

u64 lucy_pi(u64 x) {
    if (x < 2) return 0;
    const u64 r = isqrt64(x);
    std::vector<u64> lo(r + 1), hi(r + 1);     // lo[v] = S(v), hi[k] = S(x / k)
    for (u64 v = 1; v <= r; ++v) lo[v] = v - 1;
    for (u64 k = 1; k <= r; ++k) hi[k] = x / k - 1;
    for (u64 q = 2; q <= r; ++q) {
        if (lo[q] == lo[q - 1]) continue;          // q composite
        const u64 sp = lo[q - 1], q2 = q * q;
        const u64 kmax = std::min(r, x / q2);
        for (u64 k = 1; k <= kmax; ++k) {
            const u64 kq = k * q;
            const u64 sub = kq <= r ? hi[kq] : lo[x / kq];
            hi[k] -= sub - sp;
        }
        for (u64 v = r; v >= q2; --v) lo[v] -= lo[v / q] - sp;
    }
    return hi[1];
}

// primes in [lo, hi) by a segmented sieve (hi - lo small)
u64 sieve_count(u64 lo, u64 hi) {
    if (hi <= 2) return 0;
    if (lo < 2) lo = 2;
    if (lo >= hi) return 0;
    const u64 r = isqrt64(hi - 1);
    std::vector<char> small(r + 1, 1), seg(hi - lo, 1);
    for (u64 q = 2; q <= r; ++q) {
        if (!small[q]) continue;
        for (u64 j = q * q; j <= r; j += q) small[j] = 0;
        u64 s = std::max(q * q, (lo + q - 1) / q * q);
        for (u64 j = s; j < hi; j += q) seg[j - lo] = 0;
    }
    u64 c = 0;
    for (char v : seg) c += (u64)v;
    return c;
}

}  // namespace

uint64_t cz_prime_count(uint64_t lo, uint64_t hi) {
    if (hi > (1ull << 33)) hi = 1ull << 33;
    if (lo >= hi) return 0;
    if (hi - lo <= (1ull << 22)) return sieve_count(lo, hi);
    return lucy_pi(hi - 1) - (lo >= 2 ? lucy_pi(lo - 1) : 0);
}

}  // extern "C"

#include "runtime.cuh"
