// census.cu -- host orchestration and C ABI of librabung_census.so for primes
// below 2^32 (census_wide.cu adds the same census for primes below 2^33).
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
// (cz_replay), optionally through a captured CUDA graph.  The planning and
// launch code is core.cuh, shared with the wide build; runtime.cuh, included
// at the end, adds the interval census and the serving runtime on top of
// these entry points.
#include "core.cuh"
#include "microbench.cuh"
#include "sieve.cuh"

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
    c->cta_per_profile = 1;
    c->epoch_rows = EPOCH_ROWS_DEFAULT;
    c->speculate = 1;
    c->plane_budget_mb = 24u * 1024u;
    c->dense_steps = DENSE_STEPS;
    const u32 sm[10] = {0, 0, 30, 20, 15, 15, 10, 0, 5, 10};   // measured per order
    for (int r = 0; r < 10; ++r) c->spec_margin10[r] = sm[r];
    const u32 at[10] = {0, 0, 11, 7, 6, 5, 5, 5, 5, 5};   // measured per order on a top block
    for (int r = 0; r < 10; ++r) c->anchor_t[r] = at[r];
    return CZ_OK;
}

int cz_open(const cz_config *cfg, cz_handle **out) {
    const int rc = handle_open(cfg, out);
    if (rc == CZ_OK)
        cudaFuncSetAttribute(sieve_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, SIEVE_MAX_WIDTH / 16 + 64);
    return rc;
}

void cz_close(cz_handle *h) { handle_close(h); }

const char *cz_last_error(const cz_handle *h) { return h ? h->err.c_str() : "null handle"; }

uint32_t cz_count_profiles(const uint32_t *primes, uint32_t n) { return count_profiles(primes, n); }

int cz_census(cz_handle *h, const uint32_t *primes, uint32_t n, uint32_t flags, cz_profile *out,
              uint32_t out_cap, uint32_t *a4_out, cz_stats *stats) {
    return census_entry(h, primes, n, flags, out, out_cap, a4_out, stats);
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
