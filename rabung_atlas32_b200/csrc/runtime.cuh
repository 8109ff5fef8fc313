// runtime.cuh -- host runtime above the census entry points: the census of a
// prime interval (device sieve + census) and the serving runtime.  Included
// once, at the end of census.cu.
//
// Serving design (the reference has no serving path; its supervisor feeds
// fixed blocks to worker processes, src/census/worker32.cu:10-45):
//  * one scheduler thread owns the GPU work; requests wait in arrival order;
//  * every admitted request stays resident until its records are final: its
//    sparse primes' descriptors, per-profile state, colour planes, records and
//    A4 live in device arrays sized at open (ranges handed out first-fit), so
//    admission is by free plane memory and free descriptor space;
//  * the anchor filter runs as one persistent kernel over the unfinished
//    profiles of every admitted request.  When requests arrive, the scheduler
//    sets the kernel's yield flag: its CTAs finish the work item in hand,
//    leave their profiles (the claim state stays in device memory) and exit;
//    the new requests are sieved, planned and tabled on the whole GPU, and the
//    kernel is relaunched over the old and new unfinished profiles together,
//    so an arrival waits one work item (tens of microseconds), not a batch;
//  * the last CTA to leave a finished profile certifies and writes its record
//    and counts the request down; a request's last profile raises its done
//    flag in mapped host memory, and the scheduler copies its records out
//    while the kernel keeps running;
//  * primes routed to the dense scan (small p), primes whose sparse record
//    needs the dense re-run, and requests larger than the whole plane arena
//    (in waves of one slot's planes) are handled by a second handle in the
//    window between launches; a caller's non-prime is refused on the host;
//    a profile whose speculative threshold missed is re-run there on the
//    anchor filter without speculation, as cz_census does.
#pragma once
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <thread>
#include <unordered_map>

namespace {

// census of `primes` into recs (and A4), on handle h
int census_into(cz_handle *h, const std::vector<uint32_t> &primes, uint32_t flags, std::vector<cz_profile> &recs,
                std::vector<uint32_t> &a4) {
    const uint32_t n = (uint32_t)primes.size();
    recs.assign(cz_count_profiles(primes.data(), n), cz_profile{});
    a4.assign((flags & CZ_A4) ? n : 0u, 0u);
    if (n == 0) return CZ_OK;
    return cz_census(h, primes.data(), n, flags, recs.data(), (uint32_t)recs.size(),
                     (flags & CZ_A4) ? a4.data() : nullptr, nullptr);
}

// first-fit ranges of [0, cap)
struct Ranges {
    std::map<u64, u64> free_;          // start -> length
    void init(u64 cap) { free_.clear(); if (cap) free_[0] = cap; }
    bool alloc(u64 n, u64 &off) {
        if (n == 0) { off = 0; return true; }
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second < n) continue;
            off = it->first;
            const u64 rest = it->second - n, start = it->first + n;
            free_.erase(it);
            if (rest) free_[start] = rest;
            return true;
        }
        return false;
    }
    void release(u64 off, u64 n) {
        if (n == 0) return;
        auto it = free_.emplace(off, n).first;
        auto nx = std::next(it);
        if (nx != free_.end() && it->first + it->second == nx->first) { it->second += nx->second; free_.erase(nx); }
        if (it != free_.begin()) {
            auto pv = std::prev(it);
            if (pv->first + pv->second == it->first) { pv->second += it->second; free_.erase(it); }
        }
    }
};

struct CzRequest {
    uint64_t id = 0;
    uint32_t lo = 0, count = 0, flags = 0;
    bool given = false;                 // primes supplied by the caller
    int rc = -1;                        // -1 while pending
    std::string err;
    std::vector<uint32_t> primes;
    std::vector<cz_profile> recs;
    std::vector<uint32_t> a4;
    // resident part (sparse primes)
    uint32_t slot = 0xFFFFFFFFu;        // request slot: pending counter and done flag
    u64 pbase = 0, np = 0, gbase = 0, ng = 0, wbase = 0, nw = 0;
    std::vector<uint32_t> list;         // global profile indices, launch order
    std::vector<uint8_t> sparse;        // per prime: 1 resident, 0 censused on the second handle
    std::vector<cz_profile> drecs;      // records of the other primes, in prime order
    std::vector<uint32_t> da4;
};

// the device ranges of one request, freed when no kernel can touch them
struct Held {
    u64 pbase, np, gbase, ng, wbase, nw;
    u32 slot;
};

constexpr u32 SRV_CAP_PRIMES = 1u << 20;       // resident primes
constexpr u32 SRV_CAP_PROFILES = 1u << 22;     // resident profiles
constexpr u32 SRV_CAP_SLOTS = 1u << 16;        // requests in flight
constexpr int SRV_MIN_LAUNCH_US = 5000;        // a launch runs this long before it yields to arrivals

}  // namespace

struct cz_server {
    cz_config cfg{};
    cz_handle *h = nullptr;             // stream, static tables; its buffers are unused
    cz_handle *aux = nullptr;           // sieve, plans, dense primes, dense re-runs
    PrimeDesc *d_primes = nullptr;
    ProfDesc *d_profs = nullptr;
    ProfState *d_state = nullptr;
    OutRecord *d_out = nullptr;
    u32 *d_a4 = nullptr, *d_list = nullptr, *d_sidx = nullptr, *d_next = nullptr, *d_pending = nullptr;
    u32 *d_yield = nullptr, *d_a4err = nullptr, *d_planes = nullptr;
    u32 *h_done = nullptr, *d_done = nullptr;   // mapped host flags, per request slot
    u32 *h_flag = nullptr;                      // pinned: [0] = 1 (yield), [1] = a4 error word
    u64 plane_words = 0;
    Ranges rp, rg, rw, rs;
    cudaStream_t cst = nullptr;                 // copies while the filter runs
    cudaEvent_t ev_kernel = nullptr;
    bool running = false, yielding = false;
    bool blocked = false;                       // the oldest waiting request needs space in-flight work holds
    std::chrono::steady_clock::time_point launch_t0, t_yield, t_end;
    bool ended = false;                         // a launch ended and the next has not started
    std::vector<CzRequest *> inflight, repair;
    std::vector<Held> deferred;                 // ranges of requests finished during the running launch
    std::thread sched;
    std::mutex m;
    std::condition_variable cv_work, cv_done;
    std::deque<CzRequest *> waiting;
    std::unordered_map<uint64_t, CzRequest *> reqs;
    std::deque<uint64_t> announced;     // completed, not yet returned by cz_next_done
    uint64_t next_id = 1, launches = 0, completed = 0;
    uint64_t yields = 0, n_respec = 0, n_fallback = 0, n_oversize = 0;
    double ms_drain = 0, ms_window = 0;         // yield flag -> kernel end; kernel end -> relaunch
    bool stop = false;
    std::string err;
};

namespace {

// publish a request's outcome; once it is announced the caller may release
// it (cz_poll deletes it), so the scheduler must not touch r afterwards
void finish(cz_server *s, CzRequest *r, int rc, const std::string &err = "") {
    {
        std::lock_guard<std::mutex> lk(s->m);
        r->rc = rc;
        r->err = err;
        if (rc) { r->recs.clear(); r->a4.clear(); }
        s->announced.push_back(r->id);
        ++s->completed;
    }
    s->cv_done.notify_all();
}

Held held(const CzRequest *r) { return Held{r->pbase, r->np, r->gbase, r->ng, r->wbase, r->nw, r->slot}; }

void release(cz_server *s, const Held &h) {
    s->rp.release(h.pbase, h.np);
    s->rg.release(h.gbase, h.ng);
    s->rw.release(h.wbase, h.nw);
    if (h.slot != 0xFFFFFFFFu) s->rs.release(h.slot, 1);
}

// ranges of a request no kernel is running for (admission window only)
void release(cz_server *s, CzRequest *r) {
    release(s, held(r));
    r->np = r->ng = r->nw = 0;
    r->slot = 0xFFFFFFFFu;
}

// records of a request in prime order: resident primes from the device
// arrays, the others from the second handle; primes needing the dense re-run
// are collected in *redo
int assemble(cz_server *s, CzRequest *r, std::vector<uint32_t> *redo) {
    std::vector<OutRecord> dev(r->ng);
    std::vector<u32> dva4(r->np);
    u32 a4err = 0;
    if (r->np && (r->flags & CZ_A4) &&
        cudaMemcpyAsync(&a4err, s->d_a4err + r->slot, 4, cudaMemcpyDeviceToHost, s->cst) != cudaSuccess)
        return CZ_ECUDA;
    if (r->ng && cudaMemcpyAsync(dev.data(), s->d_out + r->gbase, sizeof(OutRecord) * r->ng, cudaMemcpyDeviceToHost,
                                 s->cst) != cudaSuccess)
        return CZ_ECUDA;
    if ((r->flags & CZ_A4) && r->np &&
        cudaMemcpyAsync(dva4.data(), s->d_a4 + r->pbase, 4ull * r->np, cudaMemcpyDeviceToHost, s->cst) != cudaSuccess)
        return CZ_ECUDA;
    if (cudaStreamSynchronize(s->cst) != cudaSuccess) return CZ_ECUDA;
    if (a4err) { r->err = "refused: A4 point count not certified"; return CZ_EREFUSED; }
    r->recs.clear();
    r->a4.assign((r->flags & CZ_A4) ? r->primes.size() : 0u, 0u);
    size_t gi = 0, di = 0, pi = 0, dpi = 0;
    for (size_t i = 0; i < r->primes.size(); ++i) {
        const u32 k = r->primes[i] > 2u ? popc(mask_of(r->primes[i])) : 0u;
        if (r->sparse[i]) {
            for (u32 j = 0; j < k; ++j, ++gi) {
                const OutRecord &o = dev[gi];
                if (o.status) {
                    if (!(o.status & (ST_ROOT | ST_LABEL | ST_VERIFY))) {
                        if (redo && (redo->empty() || redo->back() != (u32)i)) redo->push_back((u32)i);
                    } else {
                        char buf[160];
                        snprintf(buf, sizeof buf, "refused: p=%u r=%u status=0x%x", o.p, o.r, o.status);
                        r->err = buf;
                        return CZ_EREFUSED;
                    }
                }
                r->recs.push_back(cz_profile{o.p, o.r, o.M, o.L, o.witness, o.status, o.K});
            }
            if (r->flags & CZ_A4) r->a4[i] = dva4[pi];
            ++pi;
        } else {
            for (u32 j = 0; j < k; ++j) r->recs.push_back(r->drecs[di++]);
            if (r->flags & CZ_A4) r->a4[i] = r->da4[dpi];
            ++dpi;
        }
    }
    return CZ_OK;
}

// re-run of the primes of r listed in redo (indices into r->primes) on the
// second handle, patching their records in place (the window between
// launches only): a prime whose only fault is a speculative miss (its best
// run stayed below the speculative threshold) runs on the anchor filter
// without speculation; any other fallback status runs on the dense scan
int repair(cz_server *s, CzRequest *r, const std::vector<u32> &redo) {
    size_t off = 0;
    std::vector<size_t> start(r->primes.size());
    for (size_t i = 0; i < r->primes.size(); ++i) {
        start[i] = off;
        off += r->primes[i] > 2u ? popc(mask_of(r->primes[i])) : 0u;
    }
    std::vector<u32> spec_i, dense_i;
    for (u32 i : redo) {
        bool only_spec = true;
        const u32 k = popc(mask_of(r->primes[i]));
        for (u32 j = 0; j < k; ++j)
            if (r->recs[start[i] + j].status & ~ST_SPEC) only_spec = false;
        (only_spec ? spec_i : dense_i).push_back(i);
    }
    auto rerun = [&](const std::vector<u32> &idx, uint32_t flags) -> int {
        if (idx.empty()) return CZ_OK;
        std::vector<u32> ps;
        for (u32 i : idx) ps.push_back(r->primes[i]);
        std::vector<cz_profile> recs;
        std::vector<uint32_t> a4;
        const int rc = census_into(s->aux, ps, flags, recs, a4);
        if (rc) { r->err = cz_last_error(s->aux); return rc; }
        size_t t = 0;
        for (u32 i : idx) {
            const u32 k = popc(mask_of(r->primes[i]));
            for (u32 j = 0; j < k; ++j) r->recs[start[i] + j] = recs[t++];
        }
        return CZ_OK;
    };
    const uint32_t keep = r->flags & ~(CZ_AUTO | CZ_A4);
    int rc = rerun(spec_i, keep | CZ_SPARSE | CZ_NOSPEC);
    if (!rc) rc = rerun(dense_i, keep | CZ_DENSE);
    {
        std::lock_guard<std::mutex> lk(s->m);
        s->n_respec += spec_i.size();
        s->n_fallback += dense_i.size();
    }
    return rc;
}

// requests whose done flag is up: records out (while the filter runs), then
// complete, or queue for a dense re-run in the next window
void poll_done(cz_server *s) {
    for (size_t i = 0; i < s->inflight.size();) {
        CzRequest *r = s->inflight[i];
        if (!*(volatile u32 *)&s->h_done[r->slot]) { ++i; continue; }
        s->inflight.erase(s->inflight.begin() + i);
        std::vector<u32> redo;
        const int rc = assemble(s, r, &redo);
        s->deferred.push_back(held(r));                 // its ranges are freed after this launch
        s->blocked = false;                             // its space frees when this launch ends
        if (rc) { finish(s, r, rc, r->err.empty() ? std::string("record copy failed") : r->err); continue; }                             // its space frees when this launch ends
        if (!redo.empty()) { s->repair.push_back(r); continue; }
        finish(s, r, CZ_OK);
    }
}

// requests out of flight whose records carry a fallback status: re-run those
// primes on the dense scan (the window between launches only)
void run_repairs(cz_server *s) {
    for (CzRequest *r : s->repair) {
        std::vector<u32> redo;
        size_t off = 0;
        for (size_t i = 0; i < r->primes.size(); ++i) {
            const u32 k = r->primes[i] > 2u ? popc(mask_of(r->primes[i])) : 0u;
            for (u32 j = 0; j < k; ++j)
                if (r->recs[off + j].status) { redo.push_back((u32)i); break; }
            off += k;
        }
        const int rc = repair(s, r, redo);
        finish(s, r, rc, rc ? r->err : std::string());
    }
    s->repair.clear();
}

// admit waiting requests while they fit; sieve, plan, upload, set up, table
// and A4 on the whole GPU (no filter kernel runs now)
void admit(cz_server *s) {
    std::vector<CzRequest *> batch;
    {
        std::lock_guard<std::mutex> lk(s->m);
        while (!s->waiting.empty() && batch.size() < 4096) { batch.push_back(s->waiting.front()); s->waiting.pop_front(); }
    }
    if (batch.empty()) return;
    cudaStream_t st = s->h->st;
    std::vector<u32> sidx;                              // global indices of new resident primes
    std::vector<CzRequest *> back;                      // did not fit now
    u32 table_smem = 0;
    std::vector<u32> pend_slot, pend_val;
    std::vector<CzRequest *> admitted;                  // requests given resident space in this window
    // a request that does not fit the empty server is refused; one that does
    // not fit now waits, with everything behind it, for space to free up
    auto no_room = [&](CzRequest *r) {
        if (s->inflight.empty() && s->deferred.empty() && admitted.empty())
            finish(s, r, CZ_EREFUSED, "refused: the request exceeds the server's prime, profile or plane capacity");
        else
            back.push_back(r);
    };
    for (size_t bi = 0; bi < batch.size(); ++bi) {
        CzRequest *r = batch[bi];
        if (!back.empty()) { back.push_back(r); continue; }
        if (!r->given) {
            std::vector<uint32_t> got(r->count);
            uint32_t found = 0;
            const int rc = cz_sieve(s->aux, &r->lo, &r->count, 1, got.data(), &found);
            if (rc) { finish(s, r, rc, cz_last_error(s->aux)); continue; }
            got.resize(found);
            r->primes.swap(got);
        }
        const u32 n = (u32)r->primes.size();
        if (n == 0) { r->recs.clear(); r->a4.clear(); finish(s, r, CZ_OK); continue; }
        if (r->given) {
            // a caller's non-prime is refused here: on the filter it would
            // match every window and run without a speculative threshold
            u32 bad = 0;
            bool composite = false;
            for (u32 p : r->primes)
                if (p > 2u && !is_prime_word(p)) { bad = p; composite = true; break; }
            if (composite) {
                finish(s, r, CZ_EREFUSED, "refused: p=" + std::to_string(bad) + " is not prime");
                continue;
            }
        }
        u32 mode = r->flags & CZ_AUTO;
        if (!mode) mode = CZ_AUTO;
        int rc = plan(s->aux, r->primes.data(), n, mode);
        if (rc) { finish(s, r, rc, s->aux->err); continue; }
        // the resident (sparse) part of the plan
        std::vector<PrimeDesc> hp;
        std::vector<ProfDesc> hg;
        std::vector<u32> slist_local;                   // plan's filter order, as local profile indices
        r->sparse.assign(n, 0u);
        u64 words = 0;
        for (u32 i = 0; i < n; ++i)
            if (s->aux->hp[i].route == 2u) r->sparse[i] = 1u;
        std::vector<u32> gmap(s->aux->nprof, 0xFFFFFFFFu);
        for (u32 i = 0; i < n; ++i) {
            if (!r->sparse[i]) continue;
            const PrimeDesc &P = s->aux->hp[i];
            for (u32 j = 0; j < P.nprof; ++j) {
                const ProfDesc &D = s->aux->hprof[P.first_prof + j];
                const u64 pw = ((u64)D.npp * (P.nwords + P.nwords2) + 7ull) & ~7ull;
                words = std::max<u64>(words, D.plane_off + pw);
            }
        }
        u64 np = 0;
        for (u32 i = 0; i < n; ++i) np += r->sparse[i];
        u64 ng = 0;
        for (u32 i = 0; i < n; ++i) if (r->sparse[i]) ng += s->aux->hp[i].nprof;
        // a request larger than the whole resident arena runs on the second
        // handle, in waves of at most one slot's planes, in this window
        const bool oversize = words > s->plane_words || np > SRV_CAP_PRIMES || ng > SRV_CAP_PROFILES;
        if (oversize) {
            {
                std::lock_guard<std::mutex> lk(s->m);
                ++s->n_oversize;
            }
            r->sparse.assign(n, 0u);
            np = ng = 0;
        }
        if (np) {
            u64 pb = 0, gb = 0, wb = 0, sl = 0;
            if (!s->rp.alloc(np, pb)) { no_room(r); continue; }
            if (!s->rg.alloc(ng, gb)) { s->rp.release(pb, np); no_room(r); continue; }
            if (!s->rw.alloc(words, wb)) { s->rp.release(pb, np); s->rg.release(gb, ng); no_room(r); continue; }
            if (!s->rs.alloc(1, sl)) {
                s->rp.release(pb, np); s->rg.release(gb, ng); s->rw.release(wb, words);
                no_room(r);
                continue;
            }
            r->pbase = pb; r->np = np; r->gbase = gb; r->ng = ng; r->wbase = wb; r->nw = words; r->slot = (u32)sl;
            u32 k = 0, gcount = 0;
            for (u32 i = 0; i < n; ++i) {
                if (!r->sparse[i]) continue;
                PrimeDesc P = s->aux->hp[i];
                const u32 f0 = P.first_prof;
                P.first_prof = (u32)(gb + gcount);
                for (u32 j = 0; j < P.nprof; ++j) {
                    ProfDesc D = s->aux->hprof[f0 + j];
                    D.prime = (u32)(pb + k);
                    D.out_slot = (u32)(gb + gcount + j);
                    D.plane_off += wb;
                    D.req = (u32)sl;
                    gmap[f0 + j] = (u32)(gb + gcount + j);
                    hg.push_back(D);
                }
                gcount += P.nprof;
                hp.push_back(P);
                sidx.push_back((u32)(pb + k));
                ++k;
            }
            for (u32 g : s->aux->h_slist)
                if (gmap[g] != 0xFFFFFFFFu) r->list.push_back(gmap[g]);
            table_smem = std::max(table_smem, s->aux->table_smem);
            cudaMemcpyAsync(s->d_primes + pb, hp.data(), sizeof(PrimeDesc) * np, cudaMemcpyHostToDevice, st);
            cudaMemcpyAsync(s->d_profs + gb, hg.data(), sizeof(ProfDesc) * ng, cudaMemcpyHostToDevice, st);
            setup_kernel<<<(u32)((np + 127) / 128), 128, 0, st>>>(s->d_primes + pb, s->d_profs, s->d_state, (u32)np);
            cudaMemsetAsync(s->d_a4err + sl, 0, 4, st);    // this request's A4 error word
            if (r->flags & CZ_A4)
                a4_kernel<<<(u32)((np + A4_WARPS - 1) / A4_WARPS), A4_WARPS * 32, 0, st>>>(s->d_primes + pb, (u32)np,
                                                                                     s->d_a4 + pb, s->d_a4err + sl);
            s->h_done[sl] = 0u;
            admitted.push_back(r);
            pend_slot.push_back((u32)sl);
            pend_val.push_back((u32)ng);
        }
        // the other primes on the second handle, in prime order: the dense
        // scan, or the whole oversize request in its own mode
        std::vector<uint32_t> other;
        for (u32 i = 0; i < n; ++i) if (!r->sparse[i]) other.push_back(r->primes[i]);
        rc = census_into(s->aux, other, oversize ? r->flags : ((r->flags & ~CZ_AUTO) | CZ_DENSE), r->drecs, r->da4);
        if (rc) { release(s, r); finish(s, r, rc, cz_last_error(s->aux)); continue; }
        if (!np) {
            const int arc = assemble(s, r, nullptr);
            finish(s, r, arc, arc ? r->err : std::string());
            continue;
        }
        s->inflight.push_back(r);
    }
    if (!sidx.empty()) {
        for (size_t i = 0; i < pend_slot.size(); ++i)
            cudaMemcpyAsync(s->d_pending + pend_slot[i], &pend_val[i], 4, cudaMemcpyHostToDevice, st);
        cudaMemcpyAsync(s->d_sidx, sidx.data(), 4ull * sidx.size(), cudaMemcpyHostToDevice, st);
        TableArgs ta;
        ta.primes = s->d_primes;
        ta.profs = s->d_profs;
        ta.state = s->d_state;
        ta.planes = s->d_planes;
        ta.sparse_primes = s->d_sidx;
        ta.nsparse = (u32)sidx.size();
        ta.small_primes = s->h->d_small;
        ta.n_small = s->h->n_small;
        ta.chain = s->h->d_chain;
        ta.chain_limit = CHAIN_LIMIT;
        table_kernel<<<std::min<u32>(ta.nsparse, (u32)s->h->sms), TABLE_THREADS, table_smem, st>>>(ta);
        if (cudaStreamSynchronize(st) != cudaSuccess) {
            for (CzRequest *r : s->inflight) { release(s, r); finish(s, r, CZ_ECUDA, "set-up kernels failed"); }
            s->inflight.clear();
        }
    }
    s->blocked = !back.empty();
    if (!back.empty()) {
        std::lock_guard<std::mutex> lk(s->m);
        for (auto it = back.rbegin(); it != back.rend(); ++it) s->waiting.push_front(*it);
    }
}

// launch the filter over the unfinished profiles of every request in flight
void launch(cz_server *s) {
    std::vector<u32> list;
    for (CzRequest *r : s->inflight) list.insert(list.end(), r->list.begin(), r->list.end());
    if (list.empty()) return;
    cudaStream_t st = s->h->st;
    cudaMemcpyAsync(s->d_list, list.data(), 4ull * list.size(), cudaMemcpyHostToDevice, st);
    cudaMemsetAsync(s->d_next, 0, 4, st);
    cudaMemsetAsync(s->d_yield, 0, 4, st);
    SparseArgs sa{};
    sa.primes = s->d_primes;
    sa.profs = s->d_profs;
    sa.state = s->d_state;
    sa.planes = s->d_planes;
    sa.prof_list = s->d_list;
    sa.nlist = (u32)list.size();
    sa.next = s->d_next;
    u32 grid = s->cfg.sparse_blocks ? s->cfg.sparse_blocks : (u32)CZ_SPARSE_MINB * (u32)s->h->sms;
    sa.group = std::max(std::max(1u, s->cfg.cta_per_profile), std::min(64u, grid / std::max(1u, sa.nlist)));
    sa.tune.screen = s->cfg.screen;
    sa.epoch_rows = s->cfg.epoch_rows;
    sa.yield = s->d_yield;
    sa.out = s->d_out;
    sa.verify = 1u;
    sa.req_pending = s->d_pending;
    sa.req_done = s->d_done;
    grid = std::min(grid, sa.nlist * sa.group);
    // the list copy above comes from pageable memory: it is staged before the
    // call returns, so `list` may go; the kernel runs on while the scheduler polls
    sparse_kernel<<<grid, SPARSE_WARPS * 32, TILE_WORDS * 4u, st>>>(sa);
}

void sched_loop(cz_server *s) {
    cudaSetDevice(s->h->dev);
    for (;;) {
        poll_done(s);
        bool have_waiting, stopping;
        {
            std::lock_guard<std::mutex> lk(s->m);
            have_waiting = !s->waiting.empty();
            stopping = s->stop;
        }
        if (s->running) {
            // yield to arrivals (unless the oldest waits for space still held)
            // and to dense re-runs, once the launch has run its minimum time
            const bool ripe = std::chrono::steady_clock::now() - s->launch_t0 >=
                              std::chrono::microseconds(SRV_MIN_LAUNCH_US);
            if ((stopping || (ripe && ((have_waiting && !s->blocked) || !s->repair.empty()))) && !s->yielding) {
                cudaMemcpyAsync(s->d_yield, &s->h_flag[0], 4, cudaMemcpyHostToDevice, s->cst);
                s->yielding = true;
                s->t_yield = std::chrono::steady_clock::now();
            }
            if (cudaEventQuery(s->ev_kernel) != cudaSuccess) {
                std::unique_lock<std::mutex> lk(s->m);
                s->cv_work.wait_for(lk, std::chrono::microseconds(100));
                continue;
            }
            cudaStreamSynchronize(s->cst);
            s->running = false;
            s->t_end = std::chrono::steady_clock::now();
            s->ended = true;
            if (s->yielding) {
                std::lock_guard<std::mutex> lk(s->m);
                ++s->yields;
                s->ms_drain += std::chrono::duration<double, std::milli>(s->t_end - s->t_yield).count();
            }
            poll_done(s);
            if (!s->yielding) {                        // a launch that ran to its end finished every profile
                for (CzRequest *r : s->inflight) {
                    s->deferred.push_back(held(r));
                    finish(s, r, CZ_EREFUSED, "refused: a profile did not finish");
                }
                s->inflight.clear();
            }
            s->yielding = false;
        }
        for (const Held &h : s->deferred) release(s, h);
        s->deferred.clear();
        if (stopping) return;
        run_repairs(s);
        admit(s);
        if (!s->inflight.empty()) {
            launch(s);
            cudaEventRecord(s->ev_kernel, s->h->st);
            s->running = true;
            s->launch_t0 = std::chrono::steady_clock::now();
            std::lock_guard<std::mutex> lk(s->m);
            ++s->launches;
            if (s->ended) s->ms_window += std::chrono::duration<double, std::milli>(s->launch_t0 - s->t_end).count();
            s->ended = false;
            continue;
        }
        s->ended = false;                              // idle: no window to count
        std::unique_lock<std::mutex> lk(s->m);
        s->cv_work.wait(lk, [s] { return s->stop || !s->waiting.empty(); });
    }
}

// waits on cv until pred() or the timeout (negative: no timeout); false on timeout
template <class Pred>
bool wait_for(std::condition_variable &cv, std::unique_lock<std::mutex> &lk, int32_t timeout_ms, Pred pred) {
    if (timeout_ms < 0) { cv.wait(lk, pred); return true; }
    return cv.wait_for(lk, std::chrono::milliseconds(timeout_ms), pred);
}

void server_free(cz_server *s) {
    cudaSetDevice(s->h ? s->h->dev : 0);
    void *dev[] = {s->d_primes, s->d_profs, s->d_state, s->d_out, s->d_a4, s->d_list, s->d_sidx, s->d_next,
                   s->d_pending, s->d_yield, s->d_a4err, s->d_planes};
    for (void *p : dev) if (p) cudaFree(p);
    if (s->h_done) cudaFreeHost(s->h_done);
    if (s->h_flag) cudaFreeHost(s->h_flag);
    if (s->ev_kernel) cudaEventDestroy(s->ev_kernel);
    if (s->cst) cudaStreamDestroy(s->cst);
    if (s->aux) cz_close(s->aux);
    if (s->h) cz_close(s->h);
    for (auto &kv : s->reqs) delete kv.second;
    delete s;
}

}  // namespace

extern "C" {

int cz_census_interval(cz_handle *h, uint64_t lo, uint64_t hi, uint32_t flags, uint32_t *primes_out,
                       uint32_t primes_cap, uint32_t *n_primes, cz_profile *out, uint32_t out_cap,
                       uint32_t *n_profiles, uint32_t *a4_out, cz_stats *stats) {
    if (!h || !n_primes || !n_profiles || lo > hi || hi > (1ull << 32)) return CZ_EINVAL;
    *n_primes = 0;
    *n_profiles = 0;
    // exact prime count first: a short buffer is reported with the needed
    // count before any device work
    const uint64_t count = cz_prime_count(lo, hi);
    if (count > primes_cap) {
        *n_primes = (uint32_t)std::min<uint64_t>(0xFFFFFFFFull, count);
        return CZ_ELIMIT;
    }
    std::vector<uint32_t> ps;
    ps.reserve(count);
    uint64_t cur = std::max<uint64_t>(lo, 2);
    while (cur < hi && ps.size() < count) {
        const uint32_t want = (uint32_t)std::min<uint64_t>(count - ps.size(), 32768u);
        std::vector<uint32_t> got(want);
        uint32_t found = 0, clo = (uint32_t)cur;
        const int rc = cz_sieve(h, &clo, &want, 1, got.data(), &found);
        if (rc) return rc;
        for (uint32_t i = 0; i < found && got[i] < hi; ++i) ps.push_back(got[i]);
        if (found < want || found == 0) break;
        cur = (uint64_t)got[found - 1] + 1u;
    }
    if (ps.size() != count) {
        h->err = "device sieve and prime count disagree on [" + std::to_string(lo) + ", " + std::to_string(hi) + ")";
        return CZ_EREFUSED;
    }
    *n_primes = (uint32_t)ps.size();
    if (!ps.empty() && !primes_out) return CZ_EINVAL;
    const uint32_t np = cz_count_profiles(ps.data(), (uint32_t)ps.size());
    *n_profiles = np;
    if (np > out_cap || (np && !out)) return CZ_ELIMIT;
    std::copy(ps.begin(), ps.end(), primes_out);
    if (ps.empty()) return CZ_OK;
    return cz_census(h, ps.data(), (uint32_t)ps.size(), flags, out, out_cap, a4_out, stats);
}

int cz_server_open(const cz_config *cfg, uint32_t slots, uint64_t slot_budget_bytes, cz_server **out) {
    if (!out || slots == 0 || slots > 16) return CZ_EINVAL;
    *out = nullptr;
    cz_server *s = new cz_server();
    if (cfg) s->cfg = *cfg; else cz_default_config(&s->cfg);
    const u64 per = slot_budget_bytes ? slot_budget_bytes : ((u64)s->cfg.plane_budget_mb << 20);
    // the second handle's waves (oversize requests) hold at most one slot's planes
    cz_config acfg = s->cfg;
    acfg.plane_budget_mb = (uint32_t)std::max<u64>(64, std::min<u64>(acfg.plane_budget_mb, per >> 20));
    int rc = cz_open(&s->cfg, &s->h);
    if (!rc) rc = cz_open(&acfg, &s->aux);
    if (rc) { server_free(s); return rc; }
    cudaSetDevice(s->h->dev);
    size_t fr = 0, tot = 0;
    cudaMemGetInfo(&fr, &tot);
    const u64 fixed = (u64)SRV_CAP_PRIMES * (sizeof(PrimeDesc) + 8) +
                      (u64)SRV_CAP_PROFILES * (sizeof(ProfDesc) + sizeof(ProfState) + sizeof(OutRecord) + 4) +
                      (u64)SRV_CAP_SLOTS * 4 + (4ull << 30);
    u64 planes = (u64)slots * per;
    if (fr > fixed && planes > (u64)fr - fixed) planes = (u64)fr - fixed;
    s->plane_words = planes / 4ull & ~7ull;
    bool ok = cudaMalloc(&s->d_primes, sizeof(PrimeDesc) * SRV_CAP_PRIMES) == cudaSuccess &&
              cudaMalloc(&s->d_profs, sizeof(ProfDesc) * SRV_CAP_PROFILES) == cudaSuccess &&
              cudaMalloc(&s->d_state, sizeof(ProfState) * SRV_CAP_PROFILES) == cudaSuccess &&
              cudaMalloc(&s->d_out, sizeof(OutRecord) * SRV_CAP_PROFILES) == cudaSuccess &&
              cudaMalloc(&s->d_a4, 4ull * SRV_CAP_PRIMES) == cudaSuccess &&
              cudaMalloc(&s->d_list, 4ull * SRV_CAP_PROFILES) == cudaSuccess &&
              cudaMalloc(&s->d_sidx, 4ull * SRV_CAP_PRIMES) == cudaSuccess &&
              cudaMalloc(&s->d_next, 64) == cudaSuccess && cudaMalloc(&s->d_yield, 64) == cudaSuccess &&
              cudaMalloc(&s->d_a4err, 4ull * SRV_CAP_SLOTS) == cudaSuccess &&
              cudaMalloc(&s->d_pending, 4ull * SRV_CAP_SLOTS) == cudaSuccess &&
              cudaMalloc(&s->d_planes, 4ull * std::max<u64>(8, s->plane_words)) == cudaSuccess &&
              cudaHostAlloc(&s->h_done, 4ull * SRV_CAP_SLOTS, cudaHostAllocMapped) == cudaSuccess &&
              cudaHostGetDevicePointer((void **)&s->d_done, s->h_done, 0) == cudaSuccess &&
              cudaHostAlloc(&s->h_flag, 64, cudaHostAllocDefault) == cudaSuccess &&
              cudaStreamCreateWithFlags(&s->cst, cudaStreamNonBlocking) == cudaSuccess &&
              cudaEventCreateWithFlags(&s->ev_kernel, cudaEventDisableTiming) == cudaSuccess;
    if (!ok) { server_free(s); return CZ_ECUDA; }
    s->h_flag[0] = 1u;
    std::memset(s->h_done, 0, 4ull * SRV_CAP_SLOTS);
    cudaMemset(s->d_yield, 0, 64);
    cudaMemset(s->d_a4err, 0, 4ull * SRV_CAP_SLOTS);
    s->rp.init(SRV_CAP_PRIMES);
    s->rg.init(SRV_CAP_PROFILES);
    s->rw.init(s->plane_words);
    s->rs.init(SRV_CAP_SLOTS);
    s->sched = std::thread(sched_loop, s);
    *out = s;
    return CZ_OK;
}

void cz_server_close(cz_server *s) {
    if (!s) return;
    {
        std::lock_guard<std::mutex> lk(s->m);
        s->stop = true;
    }
    s->cv_work.notify_all();
    s->cv_done.notify_all();
    if (s->sched.joinable()) s->sched.join();
    server_free(s);
}

int cz_submit(cz_server *s, uint32_t lo, uint32_t count, const uint32_t *primes, uint32_t flags,
              uint64_t *request_id) {
    if (!s || !request_id || count == 0 || count > (1u << 20)) return CZ_EINVAL;
    CzRequest *r = new CzRequest();
    r->lo = lo;
    r->count = count;
    r->flags = flags;
    if (primes) {
        r->given = true;
        r->primes.assign(primes, primes + count);
    }
    {
        std::lock_guard<std::mutex> lk(s->m);
        if (s->stop) { delete r; return CZ_EINVAL; }
        r->id = s->next_id++;
        s->reqs[r->id] = r;
        s->waiting.push_back(r);
        *request_id = r->id;
    }
    s->cv_work.notify_one();
    return CZ_OK;
}

int cz_next_done(cz_server *s, int32_t timeout_ms, uint64_t *request_id) {
    if (!s || !request_id) return CZ_EINVAL;
    std::unique_lock<std::mutex> lk(s->m);
    for (;;) {
        while (!s->announced.empty() && !s->reqs.count(s->announced.front())) s->announced.pop_front();
        if (!s->announced.empty()) {
            *request_id = s->announced.front();
            s->announced.pop_front();
            return CZ_OK;
        }
        if (s->stop) return CZ_EINVAL;
        if (!wait_for(s->cv_done, lk, timeout_ms, [s] { return s->stop || !s->announced.empty(); }))
            return CZ_EPENDING;
    }
}

int cz_poll(cz_server *s, uint64_t request_id, int32_t timeout_ms, uint32_t *primes_out, uint32_t primes_cap,
            uint32_t *n_primes, cz_profile *out, uint32_t out_cap, uint32_t *n_profiles, uint32_t *a4_out) {
    if (!s) return CZ_EINVAL;
    std::unique_lock<std::mutex> lk(s->m);
    auto it = s->reqs.find(request_id);
    if (it == s->reqs.end()) return CZ_EINVAL;
    CzRequest *r = it->second;
    if (!wait_for(s->cv_done, lk, timeout_ms, [s, r] { return s->stop || r->rc >= 0; }) || r->rc < 0)
        return CZ_EPENDING;
    if (n_primes) *n_primes = (uint32_t)r->primes.size();
    if (n_profiles) *n_profiles = (uint32_t)r->recs.size();
    if ((primes_out && r->primes.size() > primes_cap) || (out && r->recs.size() > out_cap) ||
        (a4_out && r->a4.size() > primes_cap))
        return CZ_ELIMIT;
    if (primes_out) std::copy(r->primes.begin(), r->primes.end(), primes_out);
    if (out) std::copy(r->recs.begin(), r->recs.end(), out);
    if (a4_out) std::copy(r->a4.begin(), r->a4.end(), a4_out);
    const int rc = r->rc;
    if (rc) s->err = r->err;
    s->reqs.erase(it);
    delete r;
    return rc;
}

int cz_server_info(cz_server *s, uint64_t *batches, uint64_t *completed, uint64_t *waiting) {
    if (!s) return CZ_EINVAL;
    std::lock_guard<std::mutex> lk(s->m);
    if (batches) *batches = s->launches;
    if (completed) *completed = s->completed;
    if (waiting) *waiting = s->waiting.size();
    return CZ_OK;
}

int cz_server_stats(cz_server *s, cz_server_counters *out) {
    if (!s || !out) return CZ_EINVAL;
    std::lock_guard<std::mutex> lk(s->m);
    *out = cz_server_counters{};
    out->launches = s->launches;
    out->yields = s->yields;
    out->completed = s->completed;
    out->waiting = s->waiting.size();
    out->respec_primes = s->n_respec;
    out->fallback_primes = s->n_fallback;
    out->oversize_requests = s->n_oversize;
    out->ms_drain = s->ms_drain;
    out->ms_window = s->ms_window;
    return CZ_OK;
}

const char *cz_server_last_error(cz_server *s) {
    if (!s) return "no server";
    std::lock_guard<std::mutex> lk(s->m);
    return s->err.c_str();
}

}  // extern "C"
