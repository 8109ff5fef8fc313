// runtime.cuh -- host runtime above the census entry points: the census of a
// prime interval (device sieve + census) and the serving loop (request queue,
// continuous batching over slots, admission by device memory, per-request
// results held until polled).  Included once, at the end of census.cu; it
// uses only the C ABI of include/rabung_census.h and the plane-pool estimate.
//
// Serving design:
//  * one worker thread per slot, each owning one handle (one CUDA stream), so
//    batches of different slots overlap on the device;
//  * a free slot admits waiting requests in arrival order while their
//    estimated colour-plane pools fit min(slot budget, free HBM - reserve)
//    (always at least one request) and their flags match the first one's;
//  * the batch's intervals are sieved in one device call, the primes of all
//    its requests censused in one call (one persistent filter launch), and
//    the records split back per request in submission order;
//  * a refused merged call is re-run request by request, so only the request
//    that caused the refusal is refused.
#pragma once
#include <chrono>
#include <condition_variable>
#include <deque>
#include <thread>
#include <unordered_map>

namespace {

struct CzRequest {
    uint64_t id = 0;
    uint32_t lo = 0, count = 0, flags = 0;
    bool given = false;                 // primes supplied by the caller
    int rc = -1;                        // -1 while pending
    std::string err;
    std::vector<uint32_t> primes;
    std::vector<cz_profile> recs;
    std::vector<uint32_t> a4;
    uint64_t est = 0;                   // colour-plane pool estimate, bytes
};

// plane-pool estimate of a request for `count` primes from lo: the pool of one
// prime near the top of the interval (prime number theorem with slack) times
// the count
uint64_t interval_estimate(const cz_config &c, uint32_t lo, uint32_t count, uint32_t flags) {
    const double span = (double)count * std::max(1.0, std::log((double)lo + 2.0)) * 1.3;
    const double top = std::min(4294967291.0, (double)lo + span);
    return plane_bytes(c, (uint32_t)top, flags) * (uint64_t)count;
}

// census of `primes` into r (records and A4), on handle h
int census_into(cz_handle *h, const std::vector<uint32_t> &primes, uint32_t flags, std::vector<cz_profile> &recs,
                std::vector<uint32_t> &a4) {
    const uint32_t n = (uint32_t)primes.size();
    recs.assign(cz_count_profiles(primes.data(), n), cz_profile{});
    a4.assign((flags & CZ_A4) ? n : 0u, 0u);
    if (n == 0) return CZ_OK;
    return cz_census(h, primes.data(), n, flags, recs.data(), (uint32_t)recs.size(),
                     (flags & CZ_A4) ? a4.data() : nullptr, nullptr);
}

}  // namespace

struct cz_server {
    cz_config cfg{};
    std::vector<cz_handle *> slots;
    std::vector<std::thread> threads;
    std::mutex m;
    std::condition_variable cv_work, cv_done;
    std::deque<CzRequest *> waiting;
    std::unordered_map<uint64_t, CzRequest *> reqs;
    std::deque<uint64_t> announced;     // completed, not yet returned by cz_next_done
    uint64_t next_id = 1, budget = 0, reserve = 2ull << 30;
    uint32_t max_batch = 4096;
    bool stop = false;
    uint64_t batches = 0, completed = 0;
    std::string err;
};

namespace {

void run_batch(cz_server *s, cz_handle *h, std::vector<CzRequest *> &b) {
    // device sieve of every interval of the batch, one call
    std::vector<uint32_t> lo, cnt;
    std::vector<CzRequest *> sv;
    for (CzRequest *r : b)
        if (!r->given) { lo.push_back(r->lo); cnt.push_back(r->count); sv.push_back(r); }
    if (!sv.empty()) {
        uint64_t tot = 0;
        for (uint32_t c : cnt) tot += c;
        std::vector<uint32_t> out(std::max<uint64_t>(1, tot)), found(sv.size());
        const int rc = cz_sieve(h, lo.data(), cnt.data(), (uint32_t)sv.size(), out.data(), found.data());
        uint64_t off = 0;
        for (size_t i = 0; i < sv.size(); ++i) {
            if (rc) { sv[i]->rc = rc; sv[i]->err = cz_last_error(h); continue; }
            sv[i]->primes.assign(out.begin() + off, out.begin() + off + found[i]);
            off += cnt[i];
        }
    }
    std::vector<CzRequest *> live;
    std::vector<uint32_t> flat;
    for (CzRequest *r : b)
        if (r->rc < 0) { live.push_back(r); flat.insert(flat.end(), r->primes.begin(), r->primes.end()); }
    if (live.empty()) return;
    const uint32_t flags = live.front()->flags;
    std::vector<cz_profile> recs;
    std::vector<uint32_t> a4;
    const int rc = census_into(h, flat, flags, recs, a4);
    if (rc == CZ_OK) {
        size_t pp = 0, rp = 0;
        for (CzRequest *r : live) {
            const uint32_t np = cz_count_profiles(r->primes.data(), (uint32_t)r->primes.size());
            r->recs.assign(recs.begin() + rp, recs.begin() + rp + np);
            if (flags & CZ_A4) r->a4.assign(a4.begin() + pp, a4.begin() + pp + r->primes.size());
            rp += np;
            pp += r->primes.size();
            r->rc = CZ_OK;
        }
        return;
    }
    for (CzRequest *r : live) {            // attribute the refusal: each request alone
        const int rr = live.size() == 1 ? rc : census_into(h, r->primes, flags, r->recs, r->a4);
        r->rc = rr;
        if (rr) { r->err = cz_last_error(h); r->recs.clear(); r->a4.clear(); }
    }
}

void slot_loop(cz_server *s, size_t k) {
    cz_handle *h = s->slots[k];
    for (;;) {
        uint64_t fr = 0, tot = 0;
        cz_mem_info(h, &fr, &tot);
        std::vector<CzRequest *> batch;
        {
            std::unique_lock<std::mutex> lk(s->m);
            s->cv_work.wait(lk, [s] { return s->stop || !s->waiting.empty(); });
            if (s->stop) return;
            const uint64_t cap = std::min<uint64_t>(s->budget, fr > s->reserve ? fr - s->reserve : 0);
            const uint32_t flags = s->waiting.front()->flags;
            uint64_t used = 0;
            for (auto it = s->waiting.begin(); it != s->waiting.end() && batch.size() < s->max_batch;) {
                CzRequest *r = *it;
                if (r->flags != flags || (!batch.empty() && used + r->est > cap)) { ++it; continue; }
                batch.push_back(r);
                used += r->est;
                it = s->waiting.erase(it);
            }
            ++s->batches;
        }
        run_batch(s, h, batch);
        {
            std::lock_guard<std::mutex> lk(s->m);
            for (CzRequest *r : batch) { s->announced.push_back(r->id); ++s->completed; }
        }
        s->cv_done.notify_all();
    }
}

// waits on cv until pred() or the timeout (negative: no timeout); false on timeout
template <class Pred>
bool wait_for(std::condition_variable &cv, std::unique_lock<std::mutex> &lk, int32_t timeout_ms, Pred pred) {
    if (timeout_ms < 0) { cv.wait(lk, pred); return true; }
    return cv.wait_for(lk, std::chrono::milliseconds(timeout_ms), pred);
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
    s->budget = slot_budget_bytes ? slot_budget_bytes : ((uint64_t)s->cfg.plane_budget_mb << 20);
    for (uint32_t k = 0; k < slots; ++k) {
        cz_handle *h = nullptr;
        const int rc = cz_open(&s->cfg, &h);
        if (rc) {
            for (cz_handle *x : s->slots) cz_close(x);
            delete s;
            return rc;
        }
        s->slots.push_back(h);
    }
    for (size_t k = 0; k < s->slots.size(); ++k) s->threads.emplace_back(slot_loop, s, k);
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
    for (std::thread &t : s->threads) t.join();
    for (auto &kv : s->reqs) delete kv.second;
    for (cz_handle *h : s->slots) cz_close(h);
    delete s;
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
        for (uint32_t p : r->primes) r->est += plane_bytes(s->cfg, p, flags);
    } else {
        r->est = interval_estimate(s->cfg, lo, count, flags);
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
    if (batches) *batches = s->batches;
    if (completed) *completed = s->completed;
    if (waiting) *waiting = s->waiting.size();
    return CZ_OK;
}

const char *cz_server_last_error(cz_server *s) {
    if (!s) return "no server";
    std::lock_guard<std::mutex> lk(s->m);
    return s->err.c_str();
}

}  // extern "C"
